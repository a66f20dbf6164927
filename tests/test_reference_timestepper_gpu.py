"""The reference's fluid element and timestepper Python objects
(physicsPy.fluidElementPy, timeStepperPy.timeStepperPy) restated over the
library (grim_b200/refpy), and the two library calls under them that the
other parity tests do not reach: grim_element_fluxes (fluidElement::
computeFluxes along any direction, physics.cpp:185-217) and
grim_get_stage_grid (the consOld, divFluxes and sourcesExplicit grids a
stage leaves, timestep.cpp:26-79, 180-237), each against the oracle.  The
last test restates src/timestepper/test_CT.py, which steps a periodic grid
and prints div B of primHalfStep and primOld after every step, as an
assertion that both stay at their initial rounding level.
"""
import numpy as np
import pytest

from grim_b200 import _lib
from grim_b200 import config as C
from grim_b200 import problems as PR
from grim_b200.problems import torus as T
from oracle.oracle import PRIM_HALF
from tests.helpers import interior, pair, scaled_err

pytestmark = pytest.mark.gpu


def _torus_pair():
    """A 64x32x8 torus (MKS, derefine, cylindrify) with the oracle's
    geometry loaded into the library handle, after the initial floors (at
    32x16x8 the initial state keeps NaN zones at the inner edge, in the
    oracle as in the library)."""
    cfg = T.torus_config(N1=64, N2=32, N3=8)
    ts, orc = pair(cfg)
    for loc in (C.CENTER, C.LEFT, C.BOTTOM, C.RIGHT, C.TOP):
        o = orc.geometry(loc)
        ts.setGeometry(loc, o["gCov"], o["gCon"], o["g"], o["alpha"], x=o["x"],
                       gamma=o["gamma"] if loc == C.CENTER else None)
    P, _ = T.torus_prims(cfg, orc.geometry(C.CENTER))
    orc.set_prims(P)
    orc.problem_init()
    P = orc.get_prims()
    ts.primOld.setVars(P)
    return cfg, ts, orc, P


def _emhd_pair():
    cfg = PR.linear_modes_config(N=24)
    ts, orc = pair(cfg)
    P = orc.apply_boundaries(PR.linear_modes_prims(cfg, amplitude=1e-3))
    ts.primOld.setVars(P)
    orc.set_prims(P)
    return cfg, ts, orc, P


@pytest.mark.parametrize("case", ["torus", "emhd"])
def test_element_fluxes_match_the_oracle(case):
    """grim_element_fluxes along X0 (the conserved variables) and X1..X3 at
    every zone equals the oracle's fluidElement::computeFluxes to rounding
    (the parity build: no FMA contraction on either side)."""
    cfg, ts, orc, P = _torus_pair() if case == "torus" else _emhd_pair()
    for d in range(4):
        got = ts.elementFluxes(P, d)
        want = orc.element_fluxes(P, d)
        assert np.isfinite(want).all()
        assert scaled_err(got, want) <= 1e-14, (d, scaled_err(got, want))
    assert np.array_equal(ts.elementFluxes(P, 0), ts.conserved(P))


@pytest.mark.parametrize("case", ["torus", "emhd"])
def test_stage_grids_match_the_oracle(case):
    """After the half stage's set-up (and, for the linear mode, the full
    stage's on a perturbed primHalfStep) consOld, divFluxes and
    sourcesExplicit agree with the oracle's over the interior: to 1e-13 of
    each row's magnitude (Christoffel and EMHD source sums in another
    order)."""
    cfg, ts, orc, P = _torus_pair() if case == "torus" else _emhd_pair()
    stages = [C.HALF_STEP] if case == "torus" else [C.HALF_STEP, C.FULL_STEP]
    for stage in stages:
        if stage == C.FULL_STEP:
            Ph = P * (1. + 1e-4 * np.random.default_rng(2).standard_normal(P.shape))
            ts.primHalfStep.setVars(Ph)
            orc.set_prims(Ph, which=PRIM_HALF)
        ts.stageSetup(stage)
        orc.stage_setup(stage)
        for which in (_lib.STAGE_CONS_OLD, _lib.STAGE_DIV_FLUXES, _lib.STAGE_SOURCES_EXPLICIT):
            got = interior(cfg, ts.stageGrid(which))
            want = interior(cfg, orc.stage_grid(which))
            if which == _lib.STAGE_SOURCES_EXPLICIT:
                assert np.max(np.abs(want)) > 0, "sources expected in this case"
            assert scaled_err(got, want) <= 1e-13, (stage, which, scaled_err(got, want))


def test_fluid_element_py_computes_the_fluxes_of_its_grid():
    """physicsPy.fluidElementPy(prim, geom).computeFluxes(geom, direction,
    flux) fills flux with the element's fluxes along the four-vector index
    `direction`, as physicsPy.pyx:31-42 does (gridPy.X1 = 0 therefore gives
    the conserved variables, as it does in the reference)."""
    from grim_b200.refpy import geometryPy, gridPy, physicsPy
    cfg = PR.fast_mode_config(N=16)
    P = PR.fast_mode_prims(cfg)
    prim = gridPy.gridPy(16, 16, 1, 2, 8, 3, True, True, False)
    prim.setVars(P)
    X = gridPy.coordinatesGridPy(16, 16, 1, 2, 3, 0., 1., 0., 1., 0., 1.)
    X.getCoords(gridPy.CENTER)
    geom = geometryPy.geometryPy(geometryPy.MINKOWSKI, 0., 1., X)
    elem = physicsPy.fluidElementPy(prim, geom)
    flux = gridPy.gridPy(16, 16, 1, 2, 8, 3)
    assert elem.computeFluxes(geom, gridPy.X1, flux) == (0, 0)
    from oracle.oracle import Oracle
    orc = Oracle(C.make_config(N1=16, N2=16, dim=2))
    assert scaled_err(flux.getVars(), orc.element_fluxes(P, gridPy.X1)) <= 1e-15
    elem.computeFluxes(geom, 2, flux)
    assert scaled_err(flux.getVars(), orc.element_fluxes(P, 2)) <= 1e-15


def _test_ct_stepper(N=32):
    from grim_b200.refpy import boundaryPy, geometryPy, timeStepperPy
    per = boundaryPy.PERIODIC
    ts = timeStepperPy.timeStepperPy(N, N, 1, 2, 8, 3, 0., 0.002, per, per, per, per, per, per,
                                     geometryPy.MINKOWSKI, 0.5, 0.7, 0., 1., 0., 1., 0., 1.)
    return ts


def test_timestepper_py_fluxes_emfs_and_divergence_match_the_oracle():
    """computeDivOfFluxes leaves fluxesX1/X2 (field rows replaced by the
    constrained-transport values), emfX3 and divFluxes as the oracle's
    computeDivOfFluxes leaves its own, on the interior faces and edges."""
    ts = _test_ct_stepper(N=24)
    cfg = ts._ts.cfg
    from oracle.oracle import Oracle
    orc = Oracle(cfg)
    P = orc.apply_boundaries(PR.fast_mode_prims(PR.fast_mode_config(N=24), amplitude=1e-2))
    ts.primOld.setVars(P)
    ts.computeDivOfFluxes(ts.primOld)
    od, of, oe = orc.div_fluxes(P)
    assert scaled_err(interior(cfg, ts.divFluxes.getVars()), interior(cfg, od)) <= 1e-13
    for d, g in enumerate((ts.fluxesX1, ts.fluxesX2)):
        assert scaled_err(interior(cfg, g.getVars()), interior(cfg, of[d])) <= 1e-13, d
    assert scaled_err(interior(cfg, ts.emfX3.getVars()), interior(cfg, oe[2:3])) <= 1e-14


def test_timestepper_py_restates_test_ct():
    """src/timestepper/test_CT.py: step a periodic grid and compute div B of
    primHalfStep and primOld after every step.  Flux-CT keeps the corner
    divergence where the initial state put it: every value stays within
    1e-12 of the field's scale of its initial one."""
    ts = _test_ct_stepper()
    cfg = PR.fast_mode_config(N=32)
    P = PR.fast_mode_prims(cfg, amplitude=1e-2)
    ts.primOld.setVars(P)
    ts.computeDivB(ts.primOld)
    g = 3
    div0 = ts.divB.getVars()[0, 0, g:32 + g, g:32 + g].copy()
    scale = np.max(np.abs(P[5:8])) * 32
    for n in range(10):
        ts.timeStep()
        for grid in (ts.primHalfStep, ts.primOld):
            ts.computeDivB(grid)
            d = ts.divB.getVars()[0, 0, g:32 + g, g:32 + g]
            assert np.max(np.abs(d - div0)) <= 1e-12 * scale, (n, np.max(np.abs(d - div0)) / scale)
    assert ts.sourcesExplicit.getVars().shape == (5, 1, 38, 38)
