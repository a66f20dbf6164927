"""The workloads at the sizes and lengths they are specified at, each with
the fast form's error against the FP64 parity path stated.

The fast form (FP32 tangent Jacobian and solve refined by the FP64
residual, per-zone convergence, FMA arithmetic) and the FP64 parity path
(the reference's FD-Jacobian Newton, no FMA contraction) run the same
steps at the same Newton tolerance: relative residual 1e-10 with the
absolute floor |R| <= 1e-12 and the rounding floor of 8 ulps of the
residual's largest term (every zone converges in every form).  Their
difference per variable, max |fast - fp64| over the interior divided by
max |fp64|, is the error this module states; each bound is about 10x the
value measured on a B200, and the measured values are in the docstrings.

  * Orszag-Tang 512^2, WENO5, HLL, 200 steps; the parity path against the
    oracle for the first 5 steps of the same grid;
  * the stratified EMHD problem 256^2 (dof 10), MP5, HLL, 200 steps;
  * the 3D torus 256x128x64, PPM, LLF, 500 steps (the whole step as a CUDA
    graph in both forms): no non-finite zone, error per variable.
"""
import numpy as np
import pytest

from grim_b200 import config as C
from grim_b200 import problems as PR
from tests.helpers import interior, scaled_err

pytestmark = pytest.mark.gpu

TOL = dict(nonlinearsolve_atol=1e-24, nonlinearsolve_rtol=1e-10, nonlinearsolve_ulps=8.)


def _run(cfg, P, steps, mode, problem_init=False):
    from grim_b200.timestepper import timeStepper
    ts = timeStepper(cfg)
    if mode != C.NEWTON_PARITY_FD64:
        ts.setNewtonMode(mode, 1, cfg["nonlinearsolve_rtol"])
    ts.primOld.setVars(P)
    if problem_init:
        ts.problemInit()
    ts.enableGraph(True)
    unconv = 0
    for _ in range(steps):
        ts.timeStep()
    st = ts.stats()
    unconv += sum(st["unconverged"])
    assert st["nonFinite"] == 0
    return ts, unconv


def _per_variable(cfg, a, b):
    return [scaled_err(a[v:v + 1], b[v:v + 1]) for v in range(a.shape[0])]


def test_orszag_tang_512_for_200_steps():
    """The fast form differs from the FP64 path by at most ERR_OT of each
    variable's scale after 200 steps (measured on a B200: 1.9e-10 in rho,
    2-3e-11 in u, the velocities and the field); neither leaves a zone
    unconverged at the last step."""
    cfg = PR.orszag_tang_config(N=512, maxNonLinearIter=4, **TOL)
    P = PR.orszag_tang_prims(cfg)
    fast, u1 = _run(cfg, P, 200, C.NEWTON_MIXED32)
    ref, u2 = _run(cfg, P, 200, C.NEWTON_PARITY_FD64)
    assert u1 == 0 and u2 == 0
    a, b = interior(cfg, fast.primOld.getVars()), interior(cfg, ref.primOld.getVars())
    err = _per_variable(cfg, a, b)
    assert max(err) <= ERR_OT, err
    assert abs(fast.time - ref.time) <= 1e-12 * ref.time


def test_orszag_tang_512_parity_path_against_the_oracle():
    """The full 512^2 grid, 5 steps at the reference's tolerances: the FP64
    parity path and the oracle agree to 1e-12 of each variable's scale."""
    from oracle.oracle import Oracle
    cfg = PR.orszag_tang_config(N=512)
    P = PR.orszag_tang_prims(cfg)
    ts, _ = _run(cfg, P, 5, C.NEWTON_PARITY_FD64)
    orc = Oracle(cfg)
    orc.set_prims(P)
    orc.time_step(5)
    g, o = interior(cfg, ts.primOld.getVars()), interior(cfg, orc.get_prims())
    assert scaled_err(g, o) <= 1e-12
    assert abs(ts.time - orc.time) <= 1e-15 * orc.time


def test_emhd_stratified_256_mp5_for_200_steps():
    """The fast form (FP32 forward-tangent Jacobian of the EMHD residual)
    differs from the FP64 path by at most ERR_EMHD of each variable's scale
    after 200 steps, q and deltaP included (measured: 3.0e-11 in q,
    1.3e-11 in u1, at most 4e-12 elsewhere)."""
    cfg = PR.emhd_stratified_config(N=256, maxNonLinearIter=4, **TOL)
    P = PR.emhd_stratified_prims(cfg)
    fast, u1 = _run(cfg, P, 200, C.NEWTON_MIXED32)
    ref, u2 = _run(cfg, P, 200, C.NEWTON_PARITY_FD64)
    assert u1 == 0 and u2 == 0
    a, b = interior(cfg, fast.primOld.getVars()), interior(cfg, ref.primOld.getVars())
    err = _per_variable(cfg, a, b)
    assert max(err) <= ERR_EMHD, err


def test_torus_256x128x64_for_500_steps():
    """The benchmarked torus for the 500 steps it is specified with, both
    forms as CUDA graphs: every zone finite, every zone converged; the fast
    form differs from the FP64 path by at most ERR_TORUS of each variable's
    scale (measured: 4.8e-8 in u1, 4.2e-8 in u2, 4.4e-8 in u3, 1.5e-10 in
    rho, 4e-11 in u, at most 3.5e-10 in the field)."""
    from grim_b200.problems import torus as T
    from grim_b200.timestepper import timeStepper
    cfg = T.torus_config(**TOL)
    P, _ = T.torus_prims(cfg, timeStepper(cfg).getGeometry(C.CENTER))
    fast, u1 = _run(cfg, P, 500, C.NEWTON_MIXED32, problem_init=True)
    ref, u2 = _run(cfg, P, 500, C.NEWTON_PARITY_FD64, problem_init=True)
    assert u1 == 0 and u2 == 0
    a, b = interior(cfg, fast.primOld.getVars()), interior(cfg, ref.primOld.getVars())
    assert np.all(np.isfinite(a)) and np.all(np.isfinite(b))
    err = _per_variable(cfg, a, b)
    assert max(err) <= ERR_TORUS, err


# bounds: about 10x the measured differences
ERR_OT = 2e-9
ERR_EMHD = 3e-10
ERR_TORUS = 5e-7
