"""Ragged batch (grim_batch_*): independent problems of different grid
sizes stepped together, one compacted Newton launch per iteration over all
problems' unconverged zones.

Each problem of a batch must advance exactly as the same problem stepped
alone with the same Newton form (compacted worklists, mixed FP32 Jacobian /
FP64 residual): the per-zone code is the same, so the states agree to the
last bits up to FMA contraction choices of the two kernels (1e-13
relative); the graph-captured batch step replays the eager one bit for bit.
"""
import numpy as np
import pytest

from grim_b200 import config as C
from grim_b200 import problems as PR
from tests.helpers import interior

pytestmark = pytest.mark.gpu

RTOL, ATOL = 1e-10, 1e-24
SIZES = (16, 40, 24, 64)


def _cfgs():
    out = []
    for k, n in enumerate(SIZES):
        recon = (C.MINMOD, C.PPM, C.WENO5, C.MINMOD)[k]
        out.append(PR.fast_mode_config(N=n, reconstruction=recon, nonlinearsolve_rtol=RTOL,
                                       nonlinearsolve_atol=ATOL, maxNonLinearIter=5))
    return out


def _prims(cfg, k):
    P = PR.fast_mode_prims(cfg)
    X1, X2, _ = C.cell_centers(cfg)
    P[1] = P[1] + 1e-2 * (k + 1) * np.sin(2 * np.pi * (X1 + 2 * X2))  # uneven Newton work
    return P


def _batch(graph):
    from grim_b200.timestepper import Batch
    cfgs = _cfgs()
    B = Batch(cfgs)
    B.setNewtonMode(C.NEWTON_MIXED32, RTOL)
    for k, (cfg, ts) in enumerate(zip(cfgs, B.problems)):
        ts.primOld.setVars(_prims(cfg, k))
    B.enableGraph(graph)
    B.timeSteps(5)
    B.synchronize()
    return cfgs, B


def test_batch_matches_problems_stepped_alone():
    from grim_b200.timestepper import timeStepper
    cfgs, B = _batch(False)
    for k, (cfg, tb) in enumerate(zip(cfgs, B.problems)):
        ts = timeStepper(cfg)
        ts.setNewtonMode(C.NEWTON_MIXED32, 2, RTOL)
        ts.primOld.setVars(_prims(cfg, k))
        for _ in range(5):
            ts.timeStep()
        a, b = interior(cfg, tb.primOld.getVars()), interior(cfg, ts.primOld.getVars())
        assert np.max(np.abs(a - b) / (np.abs(b) + 1e-300)) <= 1e-13, k
        assert tb.time == ts.time
        st = tb.stats()
        assert st["unconverged"] == [0, 0] and st["nonFinite"] == 0
        assert st["newtonIters"][0] >= 1
        hist = tb.newtonHistogram()
        assert sum(hist[0]) == cfg["N1"] * cfg["N2"] and sum(hist[1]) == cfg["N1"] * cfg["N2"]


def test_batch_graph_replay_is_bitwise():
    cfgs, B1 = _batch(False)
    _, B2 = _batch(True)
    for cfg, a, b in zip(cfgs, B1.problems, B2.problems):
        assert np.array_equal(a.primOld.getVars(), b.primOld.getVars())
