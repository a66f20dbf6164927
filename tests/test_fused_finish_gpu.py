"""The stage finish fused into the per-zone mixed Newton.

With ideal MHD and the per-zone mixed Newton, each stage's Newton writes
its zone's finished state (the copy into primHalfStep / primOld, the torus
floors, the next dt term and the non-finite count of the full stage) and a
pass over the ghost zones does the rest; GRIM_DEBUG_SEPARATE_FINISH runs
the finish as one pass of its own over every zone instead.  Both give the
same bits: primOld, prim, primHalfStep, time, dt, the Newton histogram and
the counters, on the torus (floors; a NaN planted in the interior takes
fullStepDiagnostics' reset), Orszag-Tang and the linear fast mode (the dt
term formed in the finish).
"""
import numpy as np
import pytest

from grim_b200 import _lib
from grim_b200 import config as C
from grim_b200 import problems as PR

pytestmark = pytest.mark.gpu

TOL = dict(nonlinearsolve_atol=1e-24, nonlinearsolve_rtol=1e-10, nonlinearsolve_ulps=8.)


def _pair(cfg, P, init=False, graph=True):
    from grim_b200.timestepper import timeStepper
    out = []
    for separate in (0, 1):
        ts = timeStepper(cfg)
        ts.setNewtonMode(C.NEWTON_MIXED32, 1, cfg["nonlinearsolve_rtol"])
        ts.setDebug(_lib.DEBUG_SEPARATE_FINISH, separate)
        ts.primOld.setVars(P)
        if init:
            ts.problemInit()
        ts.enableGraph(graph)
        out.append(ts)
    return out


def _same(a, b, steps):
    for _ in range(steps):
        a.timeStep()
        b.timeStep()
    for g in ("primOld", "prim", "primHalfStep"):
        x, y = getattr(a, g).getVars(), getattr(b, g).getVars()
        assert np.array_equal(x, y, equal_nan=True), g
    assert a.time == b.time and a.dt == b.dt
    assert a.newtonHistogram() == b.newtonHistogram()
    sa, sb = a.stats(), b.stats()
    for key in ("unconverged", "newtonIters", "nonFinite"):
        assert sa[key] == sb[key], (key, sa[key], sb[key])
    return sa


def _torus(shape, **kw):
    from grim_b200.problems import torus as T
    from grim_b200.timestepper import timeStepper
    cfg = dict(T.torus_config(**shape), **TOL, **kw)
    P, _ = T.torus_prims(cfg, timeStepper(cfg).getGeometry(C.CENTER))
    return cfg, P


@pytest.mark.parametrize("shape,graph", [(dict(N1=64, N2=32, N3=8), False), (dict(N1=64, N2=32, N3=8), True),
                                         (dict(N1=256, N2=128, N3=64), True)])
def test_torus(shape, graph):
    cfg, P = _torus(shape)
    a, b = _pair(cfg, P, init=True, graph=graph)
    _same(a, b, 3)


def test_torus_nan_reset():
    """A NaN planted in one interior zone: the full stage's finish resets
    it (to zero, then the floors) in both forms, decided per zone in the
    fused one and by the grid's NaN count in the separate pass."""
    cfg, P = _torus(dict(N1=64, N2=32, N3=8))
    a, b = _pair(cfg, P, init=True, graph=False)
    for ts in (a, b):
        Q = ts.primOld.getVars()
        g = cfg["numGhost"]
        Q[1, g + 3, g + 10, g + 20] = np.nan
        ts.primOld.setVars(Q)
    _same(a, b, 1)
    assert np.isfinite(a.primOld.getVars()).all()


def test_orszag_tang():
    cfg = PR.orszag_tang_config(N=256, maxNonLinearIter=4, **TOL)
    a, b = _pair(cfg, PR.orszag_tang_prims(cfg))
    _same(a, b, 5)


def test_fast_mode_dt_from_the_finish():
    """elemOldFromFullStep: the next step's dt comes from the full stage's
    finish, formed in the Newton for the interior and in the ghost pass for
    the ghosts."""
    cfg = PR.fast_mode_config(N=64, **TOL)
    assert cfg["elemOldFromFullStep"] == 1
    a, b = _pair(cfg, PR.fast_mode_prims(cfg))
    _same(a, b, 6)
