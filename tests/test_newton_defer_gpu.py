"""The deferred-tail Newton (perZoneConvergence 3): one persistent kernel
whose warps run the first maxNonLinearIter - 1 updates of 32 zones
together and gather the zones still above tolerance, 32 at a time, for the
last update.  Each zone's arithmetic is the per-zone kernel's
(perZoneConvergence 1), so the two give the same bits: the state, dt, the
Newton histogram and the unconverged count, on the torus (MKS, derefine,
cylindrify, floors; the benchmarked 256x128x64 grid and a small one),
Orszag-Tang and a tolerance no zone meets (every zone through the final
test).  The EMHD problems run the per-zone kernel under setting 3.
"""
import numpy as np
import pytest

from grim_b200 import config as C
from grim_b200 import problems as PR

pytestmark = pytest.mark.gpu

TOL = dict(nonlinearsolve_atol=1e-24, nonlinearsolve_rtol=1e-10, nonlinearsolve_ulps=8.)


def _pair(cfg, P, init=False, graph=True):
    from grim_b200.timestepper import timeStepper
    out = []
    for mode in (1, 3):
        ts = timeStepper(cfg)
        ts.setNewtonMode(C.NEWTON_MIXED32, mode, cfg["nonlinearsolve_rtol"])
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
    assert np.array_equal(a.primOld.getVars(), b.primOld.getVars())
    assert a.time == b.time and a.dt == b.dt
    assert np.array_equal(a.newtonHistogram(), b.newtonHistogram())
    sa, sb = a.stats(), b.stats()
    for key in ("unconverged", "newtonIters", "nonFinite"):
        assert sa[key] == sb[key], (key, sa[key], sb[key])
    return sa


def _torus(shape, **kw):
    from grim_b200.problems import torus as T
    from grim_b200.timestepper import timeStepper
    cfg = dict(T.torus_config(**shape), **kw)
    P, _ = T.torus_prims(cfg, timeStepper(cfg).getGeometry(C.CENTER))
    return cfg, P


@pytest.mark.parametrize("shape", [dict(N1=64, N2=32, N3=8), dict(N1=256, N2=128, N3=64)])
def test_torus_same_bits_as_the_per_zone_kernel(shape):
    cfg, P = _torus(shape, **TOL)
    a, b = _pair(cfg, P, init=True)
    _same(a, b, 4)
    h = b.newtonHistogram()
    # zones did take the deferred last update
    assert h[0][cfg["maxNonLinearIter"]] + h[1][cfg["maxNonLinearIter"]] > 0


def test_unconverged_zones_take_the_final_test():
    """A tolerance below the rounding of the residual: every zone runs to
    the cap and through the final test in both kernels."""
    cfg, P = _torus(dict(N1=64, N2=32, N3=8), nonlinearsolve_atol=0., nonlinearsolve_rtol=1e-30,
                    nonlinearsolve_ulps=0., maxNonLinearIter=2)
    a, b = _pair(cfg, P, init=True, graph=False)
    st = _same(a, b, 2)
    assert min(st["unconverged"]) > 0


def test_orszag_tang_same_bits():
    cfg = PR.orszag_tang_config(N=256, maxNonLinearIter=4, **TOL)
    a, b = _pair(cfg, PR.orszag_tang_prims(cfg))
    _same(a, b, 5)


def test_emhd_runs_the_per_zone_kernel():
    cfg = PR.emhd_stratified_config(N=64, maxNonLinearIter=4, **TOL)
    a, b = _pair(cfg, PR.emhd_stratified_prims(cfg))
    _same(a, b, 3)
