"""Host logic of the X3 slab decomposition (grim_b200/slab.py) on CPU:
the slab configurations and the halo wiring, the latter over gloo with two
ranks exchanging tensors (no GPU)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from grim_b200 import config as C
from grim_b200 import slab
from grim_b200.problems import torus as T


def test_slab_config_periodic_and_bounded():
    cfg = T.torus_config(N1=16, N2=8, N3=16)
    for world in (1, 2, 4):
        for r in range(world):
            loc = slab.slab_config(cfg, r, world)
            assert loc["N3"] == 16 // world and loc["N3Global"] == 16
            assert loc["boundaryBack"] == C.EXCHANGE and loc["boundaryFront"] == C.EXCHANGE
            assert loc["X3Start"] == cfg["X3Start"] and loc["X3End"] == cfg["X3End"]
    b = dict(cfg, boundaryBack=C.OUTFLOW, boundaryFront=C.OUTFLOW)
    loc0, loc1 = slab.slab_config(b, 0, 2), slab.slab_config(b, 1, 2)
    assert loc0["boundaryBack"] == C.OUTFLOW and loc0["boundaryFront"] == C.EXCHANGE
    assert loc1["boundaryBack"] == C.EXCHANGE and loc1["boundaryFront"] == C.OUTFLOW
    assert slab.neighbours(0, 2, False) == (None, 1) and slab.neighbours(1, 2, False) == (0, None)
    assert slab.neighbours(0, 3, True) == (2, 1)
    with pytest.raises(ValueError):
        slab.slab_config(cfg, 0, 3)  # 16 planes over 3 ranks
    with pytest.raises(ValueError):
        slab.slab_config(cfg, 0, 8)  # 2 planes per slab


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, periodic, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        lower, upper = slab.neighbours(rank, world, periodic)
        mk = lambda v: torch.full((2, 3, 4, 5), float(v), dtype=torch.float64)
        send_lo, send_hi = mk(10 * rank + 1), mk(10 * rank + 2)
        recv_lo, recv_hi = mk(-1), mk(-1)
        slab.exchange_planes(send_lo, send_hi, recv_lo, recv_hi, lower, upper, rank)
        out[rank] = (float(recv_lo[0, 0, 0, 0]), float(recv_hi[0, 0, 0, 0]))
        # the two reductions of a step
        t = torch.tensor([float(rank + 1)], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        assert float(t) == world
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,periodic", [(2, True), (3, True), (3, False)])
def test_halo_wiring_gloo(world, periodic):
    """recv_lo holds the lower neighbour's high interior planes, recv_hi the
    upper neighbour's low ones; physical ends receive nothing."""
    out = mp.get_context("spawn").Manager().dict()
    mp.start_processes(_worker, args=(world, _free_port(), periodic, out), nprocs=world, start_method="spawn")
    for r in range(world):
        lower, upper = slab.neighbours(r, world, periodic)
        lo, hi = out[r]
        assert lo == (10 * lower + 2 if lower is not None else -1.0), (r, lo)
        assert hi == (10 * upper + 1 if upper is not None else -1.0), (r, hi)


def test_combine_observer_rows():
    """Integrals and boundary fluxes add over slabs, rhoMax is the largest
    slab maximum, betaMin the smallest slab minimum (ObserversTorus.hpp)."""
    a = np.arange(1., 10.)
    b = np.array([10., 20., 30., 0.5, 7., 40., 50., 60., 70.])
    out = slab.combine_observer_rows([a, b])
    want = a + b
    want[3] = max(a[3], b[3])
    want[4] = min(a[4], b[4])
    np.testing.assert_array_equal(out, want)
    # records (rows of 9) combine row by row
    recs = slab.combine_observer_rows([np.stack([a, b]), np.stack([b, a])])
    np.testing.assert_array_equal(recs[0], want)
    np.testing.assert_array_equal(recs[1], want)


def _obs_worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = np.full((2, 9), float(rank + 1))
        mine[:, 4] = 10. - rank  # betaMin: smallest on the last rank
        rows = slab.all_gather_rows(mine, world)
        out[rank] = slab.combine_observer_rows(rows).tolist()
    finally:
        dist.destroy_process_group()


def test_observer_rows_gathered_over_gloo():
    """Two ranks gather each other's observer records in rank order and
    agree on the combined values."""
    out = mp.get_context("spawn").Manager().dict()
    mp.start_processes(_obs_worker, args=(2, _free_port(), out), nprocs=2, start_method="spawn")
    for r in range(2):
        got = np.array(out[r])
        assert got.shape == (2, 9)
        np.testing.assert_array_equal(got[:, 0], 3.)  # 1 + 2
        np.testing.assert_array_equal(got[:, 3], 2.)  # max
        np.testing.assert_array_equal(got[:, 4], 9.)  # min
