"""The ragged batch and adjoint workload at its specified size: 16
independent 2D ideal linear-mode problems of 64^2 .. 512^2 (seeded random
sizes and wavevectors, amplitude 1e-4), 100 implicit steps.

  * the batch (one CUDA graph per batch step, one compacted Newton launch
    per iteration over every problem's unconverged zones) advances each
    problem as the same problem stepped alone (1e-13 relative), with every
    zone converged;
  * a small batch against the oracle (the reference's method);
  * per problem, the reverse adjoint of its final L2 energy with respect to
    its initial primitives, checkpoints every 10 steps, checked against
    central differences of the same forward map at 1e-6 along sampled
    directions of every problem (see that test for why directions, and
    for the scheme and amplitude);
  * the adjoint through a torch.autograd.Function (the test harness's
    wrapper of the C ABI) gives the same gradient, and torch's gradcheck
    passes on a small problem.
"""
import numpy as np
import pytest
import torch

from grim_b200 import config as C
from grim_b200 import problems as PR
from tests.adjoint_harness import TimeSteps, energy, energy_lambda, interior_mask, prepare
from tests.helpers import interior, scaled_err

pytestmark = pytest.mark.gpu

TOL = dict(nonlinearsolve_atol=1e-24, nonlinearsolve_rtol=1e-10, nonlinearsolve_ulps=8., maxNonLinearIter=4)
STEPS = 100
BG = PR.LM_BACKGROUND_IDEAL


def test_ragged_batch_of_16_problems_for_100_steps():
    from grim_b200.timestepper import Batch, timeStepper
    probs = PR.ragged_batch(**TOL)
    assert len(probs) == 16 and min(c["N1"] for c, _ in probs) >= 64 and max(c["N1"] for c, _ in probs) <= 512
    B = Batch([cfg for cfg, _ in probs])
    B.setNewtonMode(C.NEWTON_MIXED32, TOL["nonlinearsolve_rtol"])
    for (cfg, P), ts in zip(probs, B.problems):
        ts.primOld.setVars(P)
    B.enableGraph(True)
    B.timeSteps(STEPS)
    B.synchronize()
    for (cfg, P), tb in zip(probs, B.problems):
        st = tb.stats()
        assert st["unconverged"] == [0, 0] and st["nonFinite"] == 0
        alone = timeStepper(cfg)
        alone.setNewtonMode(C.NEWTON_MIXED32, 2, TOL["nonlinearsolve_rtol"])
        alone.primOld.setVars(P)
        alone.enableGraph(True)
        alone.timeSteps(STEPS)
        a, b = interior(cfg, tb.primOld.getVars()), interior(cfg, alone.primOld.getVars())
        assert np.max(np.abs(a - b) / (np.abs(b) + 1e-300)) <= 1e-13, cfg["N1"]
        assert tb.time == alone.time


def test_small_batch_against_the_oracle():
    """Three problems of the batch family (16^2, 24^2, 32^2) stepped 5 times
    as a batch (exact FP64 tangent Jacobian, per-zone convergence) and by
    the oracle (the reference's FD-Jacobian Newton, global break) at the
    same relative tolerance 1e-10 with maxNonLinearIter 6: the two
    converged solutions agree to 1e-10 of each variable's scale."""
    from grim_b200.timestepper import Batch
    from oracle.oracle import Oracle
    tol = dict(nonlinearsolve_atol=1e-24, nonlinearsolve_rtol=1e-10, maxNonLinearIter=6)
    probs = [(PR.fast_mode_config(N=n, **tol), None) for n in (16, 24, 32)]
    rng = np.random.default_rng(9)
    out = []
    for cfg, _ in probs:
        X1, X2, _ = C.cell_centers(cfg)
        k1, k2 = (int(x) for x in rng.integers(1, 5, 2))
        ph = rng.uniform(0, 2 * np.pi, 8)
        out.append((cfg, np.stack([BG[v] + 1e-4 * np.cos(2 * np.pi * (k1 * X1 + k2 * X2) + ph[v])
                                   for v in range(8)])))
    B = Batch([cfg for cfg, _ in out])
    B.setNewtonMode(C.NEWTON_TANGENT64, tol["nonlinearsolve_rtol"])
    for (cfg, P), ts in zip(out, B.problems):
        ts.primOld.setVars(P)
    B.timeSteps(5)
    B.synchronize()
    for (cfg, P), tb in zip(out, B.problems):
        o = Oracle(cfg)
        o.set_prims(P)
        o.time_step(5)
        assert abs(tb.time - o.time) <= 1e-14 * o.time
        assert scaled_err(interior(cfg, tb.primOld.getVars()), interior(cfg, o.get_prims())) <= 1e-10


def _adjoint_stepper(cfg):
    from grim_b200.timestepper import timeStepper
    ts = timeStepper(cfg)
    ts.setNewtonMode(C.NEWTON_TANGENT64, 1, 0.0)
    return ts


def test_per_problem_adjoint_of_the_final_energy():
    """Each of the 16 problems (their sizes, wavevectors and phases): the
    adjoint of L = 1/2 sum (P_final - bg)^2 over 100 steps (checkpoints
    every 10, dt fixed, the Newton converged to rounding with the exact
    FP64 Jacobian) is
      * the same bits with checkpoints every 10 or every 100 steps (the
        recomputed segments are the forward run's);
      * checked against central differences of the same forward map along
        three directions of the initial interior (the gradient itself and
        two random unit vectors): (L(P + h d) - L(P - h d)) / 2h matches
        <grad, d> to 1e-6 of |grad| at h = 1e-6 or 1e-7.

    Directions rather than single entries: over 100 steps the map is only
    piecewise smooth (limiter branches, HLL's min / max of the face states'
    speeds, which nearly tie on every face of a near-uniform state), and a
    one-entry difference of 1e-6 crosses enough branch switches downstream
    that its error grows with the step count (measured on this family:
    1e-6 at 6 steps, up to 1e-5 .. 1e-2 at 100 steps, falling as h falls),
    while the rounding of L, O(N^2 amplitude^2), keeps h from going lower.
    A unit direction spreads the same step over every zone (1e-9 per zone
    on a 368^2 grid), and <grad, d> sums the whole gradient, so both errors
    fall far below 1e-6.  The entrywise check is
    test_adjoint_matches_central_fd (24^2, 6 steps).  The family runs with
    WENO5 / HLL at amplitude 1e-2 here (minmod / LLF at 1e-4 in the batch
    test): the adjoint code is the same for every reconstruction and
    Riemann solver (their local Jacobians come from one forward-tangent
    pass), and WENO5's weights are smooth."""
    probs = PR.ragged_batch(amplitude=1e-2, reconstruction=C.WENO5, riemannSolver=C.HLL, maxNonLinearIter=6,
                            nonlinearsolve_atol=0.0)
    rng = np.random.default_rng(15)
    worst = []
    for cfg, P in probs:
        ts = _adjoint_stepper(cfg)
        prepare(ts, cfg, P)
        ts.adjointForward(STEPS, 10)
        lam = energy_lambda(cfg, ts.primOld.getVars(), BG)
        grad = ts.adjointBackward(lam)
        prepare(ts, cfg, P)
        ts.adjointForward(STEPS, STEPS)
        assert np.array_equal(ts.adjointBackward(lam), grad), cfg["N1"]
        inner = interior_mask(cfg, grad.shape)
        gnorm = float(np.sqrt(np.sum(grad[inner] ** 2)))
        dirs = [grad / gnorm]
        for _ in range(2):
            d = np.zeros_like(grad)
            d[inner] = rng.standard_normal(int(inner.sum()))
            dirs.append(d / np.sqrt(np.sum(d ** 2)))

        def L(Q):
            prepare(ts, cfg, Q)
            ts.timeSteps(STEPS)
            return energy(cfg, ts.primOld.getVars(), BG)

        for d in dirs:
            want = float(np.sum(grad * d))
            fd = [(L(P + h * d) - L(P - h * d)) / (2 * h) for h in (1e-6, 1e-7)]
            err = min(abs(f - want) for f in fd) / gnorm
            worst.append(err)
            assert err <= 1e-6, (cfg["N1"], want, fd, gnorm)
    assert len(worst) == 48


def test_autograd_wrapper_gives_the_adjoint_gradient():
    """loss.backward() through TimeSteps equals grim_adjoint_backward's
    gradient bit for bit, on the smallest problem of the batch (80^2), 20
    steps."""
    cfg, P = PR.ragged_batch(maxNonLinearIter=6, nonlinearsolve_atol=0.0)[15]
    ts = _adjoint_stepper(cfg)
    p0 = torch.from_numpy(P.copy()).requires_grad_(True)
    pf = TimeSteps.apply(p0, ts, cfg, 20, 10)
    bg = torch.tensor(BG, dtype=torch.float64)[:, None, None, None]
    g = cfg["numGhost"]
    loss = 0.5 * ((pf[:, :, g:g + cfg["N2"], g:g + cfg["N1"]] - bg) ** 2).sum()
    loss.backward()
    ref = _adjoint_stepper(cfg)
    prepare(ref, cfg, P)
    ref.adjointForward(20, 10)
    want = ref.adjointBackward(energy_lambda(cfg, ref.primOld.getVars(), BG))
    assert np.array_equal(p0.grad.numpy(), want)
    assert abs(float(loss.detach()) - energy(cfg, ref.primOld.getVars(), BG)) <= 1e-15 * float(loss.detach())


def test_gradcheck_of_the_wrapper_on_a_small_problem():
    """torch.autograd.gradcheck of TimeSteps in its fast mode (the Jacobian
    projected on random input and output directions, ghosts included) on an
    8^2 problem over 3 steps, WENO5 / HLL, a smooth 1e-2 perturbation with
    random phases, at gradcheck's FP64 step 1e-6 and tolerances 1e-5
    absolute, 1e-3 relative.  Entry by entry the map is only piecewise
    smooth: HLL's min / max of the two face states' speeds nearly tie on
    every face of a near-uniform state, and a plain cosine sampled on 8
    zones puts zones symmetric about its extrema, where the limiters'
    candidate slopes tie exactly (a kink at the point); the entrywise check
    with its screens for both is test_adjoint_matches_central_fd."""
    cfg = PR.fast_mode_config(N=8, reconstruction=C.WENO5, riemannSolver=C.HLL, maxNonLinearIter=6,
                              nonlinearsolve_atol=0.0)
    X1, X2, _ = C.cell_centers(cfg)
    rng = np.random.default_rng(21)
    ph = rng.uniform(0, 2 * np.pi, (8, 2))
    P = np.stack([BG[v] + 1e-2 * np.sin(2 * np.pi * X1 + ph[v, 0]) * np.cos(2 * np.pi * X2 + ph[v, 1])
                  for v in range(8)])
    ts = _adjoint_stepper(cfg)
    p0 = torch.from_numpy(P).requires_grad_(True)
    assert torch.autograd.gradcheck(lambda x: TimeSteps.apply(x, ts, cfg, 3, 2), (p0,), eps=1e-6, atol=1e-5,
                                    rtol=1e-3, fast_mode=True)
