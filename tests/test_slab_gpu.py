"""The X3 slab decomposition on the GPU (grim_b200/slab.py): a decomposed
torus run gives the single-handle run's primitives bit for bit.  One rank
exchanges with itself (the periodic ring closes on it); two ranks share
this one GPU and move their halos through host memory over gloo (no kernel
of one rank waits on the other: every exchange happens between launches)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from grim_b200 import config as C
from grim_b200.problems import torus as T

pytestmark = pytest.mark.gpu

SHAPE = dict(N1=64, N2=32, N3=8)  # two slabs of 4 planes
STEPS = 3


def _cfg(mode):
    return T.torus_config(**SHAPE, newtonMode=mode, perZoneConvergence=1 if mode else 0)


def _initial(cfg):
    from grim_b200.timestepper import timeStepper
    ts = timeStepper(cfg)
    P, _ = T.torus_prims(cfg, ts.getGeometry(C.CENTER))
    return ts, P


def _single(cfg, P, ts):
    ts.primOld.setVars(P)
    ts.problemInit()
    for _ in range(STEPS):
        ts.timeStep()
    s3, s2, s1 = C.interior_slices(cfg)
    return ts.primOld.getVars()[:, s3, s2, s1], ts.time


@pytest.mark.parametrize("mode", [C.NEWTON_PARITY_FD64, C.NEWTON_MIXED32])
def test_one_rank_slab_equals_the_plain_step(mode):
    from grim_b200.slab import SlabTimeStepper
    cfg = _cfg(mode)
    ts, P = _initial(cfg)
    ref, tref = _single(cfg, P, ts)
    sl = SlabTimeStepper(cfg)
    sl.setGlobalPrims(P)
    sl.ts.problemInit()
    for _ in range(STEPS):
        sl.timeStep()
    assert not np.isnan(ref).any()
    assert np.array_equal(sl.gatherInterior(), ref)
    assert sl.time == tref


def _rank(rank, world, port, mode, P, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from grim_b200.slab import SlabTimeStepper
        sl = SlabTimeStepper(_cfg(mode), device=0)
        sl.setGlobalPrims(P)
        sl.ts.problemInit()
        for _ in range(STEPS):
            sl.timeStep()
        g = sl.gatherInterior()
        if rank == 0:
            np.save(out, g)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_rank_slabs_equal_the_plain_step(tmp_path):
    cfg = _cfg(C.NEWTON_PARITY_FD64)
    ts, P = _initial(cfg)
    ref, _ = _single(cfg, P, ts)
    del ts
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    out = str(tmp_path / "g.npy")
    mp.start_processes(_rank, args=(2, port, C.NEWTON_PARITY_FD64, P, out), nprocs=2, start_method="spawn")
    assert not np.isnan(ref).any()
    assert np.array_equal(np.load(out), ref)


def _obs_rank(rank, world, port, cfg, P, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from grim_b200.slab import SlabTimeStepper
        sl = SlabTimeStepper(cfg, device=0)
        sl.setGlobalPrims(P)
        sl.ts.problemInit()
        for _ in range(STEPS):
            sl.timeStep()
        recs = sl.observations()
        now = sl.torusObservers()
        if rank == 0:
            np.save(out, np.array([[r["time"]] + [r[k] for k in OBS] for r in recs]
                                  + [[sl.time] + [now[k] for k in OBS]]))
        dist.barrier()
    finally:
        dist.destroy_process_group()


OBS = ("BaryonMass", "EMag", "ETh", "rhoMax", "betaMin", "MdotIn", "MdotOut", "UnboundMdotOut",
       "RelativisticUnboundMdotOut")


def test_two_rank_slab_observers_equal_the_single_handle(tmp_path):
    """The torus observers recorded by a two-slab run, combined over the
    ranks (sums for the integrals and boundary fluxes, max rhoMax, min
    betaMin), equal the single handle's records: sums to 1e-13 of their
    magnitude (the partial sums are added in another order), extrema and
    record times exactly."""
    cfg = dict(_cfg(C.NEWTON_PARITY_FD64), ObserveEveryDt=1e-12)
    ts, P = _initial(cfg)
    _single(cfg, P, ts)
    ref = [[r["time"]] + [r[k] for k in OBS] for r in ts.observations()]
    now = ts.torusObservers()
    ref.append([ts.time] + [now[k] for k in OBS])
    ref = np.array(ref)
    del ts
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    out = str(tmp_path / "obs.npy")
    mp.start_processes(_obs_rank, args=(2, port, cfg, P, out), nprocs=2, start_method="spawn")
    got = np.load(out)
    assert got.shape == ref.shape and ref.shape[0] >= STEPS + 1
    np.testing.assert_array_equal(got[:, 0], ref[:, 0])
    for k, name in enumerate(OBS, start=1):
        if name in ("rhoMax", "betaMin"):
            np.testing.assert_array_equal(got[:, k], ref[:, k], err_msg=name)
        else:
            scale = np.max(np.abs(ref[:, k])) + 1e-300
            assert np.max(np.abs(got[:, k] - ref[:, k])) <= 1e-13 * scale, name
