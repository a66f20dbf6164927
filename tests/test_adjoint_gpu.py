"""Adjoint (reverse) sweep of whole implicit timesteps, through the C ABI.

The gradient of L = 1/2 sum_interior (P_final - P_background)^2 with
respect to the initial primitives, from grim_adjoint_backward after a
checkpointed grim_adjoint_forward, against central finite differences of
the same forward map (dt held fixed, Newton converged to roundoff with the
exact FP64 tangent Jacobian) at a relative tolerance of 1e-6 in FP64.
The workload is the ideal-MHD linear-mode problem family of the batched
adjoint configuration: 2D, Minkowski, periodic, minmod / PPM reconstruction,
LLF / HLL fluxes, flux-CT, random smooth 1e-2 perturbations; the same in
3D (periodic in all three directions, the three edge EMFs of flux-CT); and
the torus grid's metric (modified Kerr-Schild) and boundaries (outflow,
mirror, periodic) without the torus problem hooks.
"""
import numpy as np
import pytest

from grim_b200 import config as C
from grim_b200 import problems as PR
from tests.adjoint_harness import fd_check, fd_check_richardson
from tests.helpers import interior

pytestmark = pytest.mark.gpu

BG = np.array([1.0, 2.0, 0.0, 0.0, 0.0, 0.1, 0.3, 0.0])


def _state(cfg, seed, amp=1e-2):
    rng = np.random.default_rng(seed)
    X1, X2, _ = C.cell_centers(cfg)
    P = np.zeros((8,) + X1.shape)
    for v in range(8):
        k1, k2 = rng.integers(1, 3, 2)
        ph = rng.uniform(0, 2 * np.pi, 2)
        P[v] = BG[v] + amp * (np.sin(2 * np.pi * k1 * X1 + ph[0]) * np.cos(2 * np.pi * k2 * X2 + ph[1]))
    return P


def _stepper(cfg, P):
    from grim_b200.timestepper import timeStepper
    ts = timeStepper(cfg)
    ts.setNewtonMode(C.NEWTON_TANGENT64, 1, 0.0)
    ts.primOld.setVars(P)
    ts.primOld.communicate()  # ghosts = periodic images of the interior
    ts.setTime(0.0, cfg["dt"])
    ts.setFixedDt(True)
    return ts


def _loss(cfg, P, nsteps):
    ts = _stepper(cfg, P)
    for _ in range(nsteps):
        ts.timeStep()
    Q = interior(cfg, ts.primOld.getVars())
    return 0.5 * np.sum((Q - BG[:, None, None, None]) ** 2)


def _adjoint(cfg, P, nsteps, every):
    ts = _stepper(cfg, P)
    ts.adjointForward(nsteps, every)
    Pf = ts.primOld.getVars()
    lam = np.zeros_like(Pf)
    sl = (slice(None),) + tuple(slice(0, n) for n in Pf.shape[1:])
    lam[sl] = Pf - BG[:, None, None, None]
    g = cfg["numGhost"]
    mask = np.zeros(Pf.shape[1:], bool)
    mask[:, g:g + cfg["N2"], g:g + cfg["N1"]] = True
    lam[:, ~mask] = 0.0
    grad = ts.adjointBackward(lam)
    assert np.array_equal(ts.primOld.getVars(), Pf)  # the stepper is left at the final state
    return grad


@pytest.mark.parametrize("recon,riemann", [(C.MINMOD, C.LOCAL_LAX_FRIEDRICH), (C.PPM, C.HLL)])
def test_adjoint_matches_central_fd(recon, riemann):
    """The forward map is piecewise smooth: the limiters (minmod's slope
    choice, PPM's monotonicity corrections) and the Riemann solvers' max /
    min of the two face states' speeds switch branch where two candidates
    tie, and the adjoint is the derivative of the branch taken.  A central
    difference whose bracket contains such a switch measures an average of
    two branches, so the 1e-6 check applies where the map is smooth over the
    bracket: the differences at h = 1e-6 and h = 1e-7 agree (to the 1e-7
    difference's roundoff) and the second differences show no slope jump at
    the point itself (a switch within 1e-7 of the point sits in both
    brackets); there the adjoint matches one of the central differences to
    1e-6.  At least 10 of 64 random picks must
    qualify."""
    N, nsteps = 24, 6
    cfg = PR.fast_mode_config(N=N, reconstruction=recon, riemannSolver=riemann, maxNonLinearIter=6,
                              nonlinearsolve_atol=0.0)
    P = _state(cfg, 11)
    grad = _adjoint(cfg, P, nsteps, every=4)
    g = cfg["numGhost"]
    gi = interior(cfg, grad)
    assert np.all(grad[:, 0, :g, :] == 0) and np.all(grad[:, 0, :, :g] == 0)
    scale = np.max(np.abs(gi))
    rng = np.random.default_rng(5)

    L0 = _loss(cfg, P, nsteps)

    def shifted(v, j, i, h):
        Q = P.copy()
        Q[v, 0, j + g, i + g] += h
        return _loss(cfg, Q, nsteps)

    # a slope jump D at the point (a switch closer than 1e-7, inside both
    # brackets) makes the second differences (p - 2 L0 + m) / h equal D at
    # every h, a smooth map makes them h L''; fd_check screens on both
    picks = [(n % 8,) + tuple(int(x) for x in rng.integers(0, N, 2)) for n in range(64)]
    smooth, bad = fd_check(shifted, L0, gi[:, 0], picks, scale)
    assert not bad, bad
    assert smooth >= 10, smooth


def test_adjoint_checkpoint_interval_does_not_change_the_gradient():
    """Checkpoints every step or every third step give the same bits: the
    recomputed segments reproduce the forward run, and every accumulation of
    the reverse sweep is a fixed-order gather (no atomics)."""
    cfg = PR.fast_mode_config(N=16, maxNonLinearIter=6, nonlinearsolve_atol=0.0)
    P = _state(cfg, 3)
    a = _adjoint(cfg, P, 5, every=1)
    b = _adjoint(cfg, P, 5, every=3)
    assert np.array_equal(a, b)


def test_adjoint_refuses_unsupported_configurations():
    """A 1D grid and a slab of a decomposed grid are outside the adjoint's
    scope (GRIM_ENOTSUP)."""
    from grim_b200.timestepper import timeStepper
    for cfg in (PR.fast_mode_config(N=32, dim=1), PR.fast_mode_config(N=8, N3=8, dim=3, N3Global=16)):
        ts = timeStepper(cfg)
        with pytest.raises(Exception):
            ts.adjointForward(2, 1)


def _with_images(ts, P):
    ts.primOld.setVars(P)
    ts.primOld.communicate()
    return ts.primOld.getVars()


@pytest.mark.parametrize("recon,riemann", [(C.MINMOD, C.LOCAL_LAX_FRIEDRICH), (C.PPM, C.HLL)])
def test_stencil_transpose_matches_fd(recon, riemann):
    """The transpose of the flux divergence (reconstruction, Riemann, flux-CT,
    divergence; ghosts as periodic images) against central differences of
    <gbar, divF(P)> from grim_compute_div_fluxes."""
    cfg = PR.fast_mode_config(N=16, reconstruction=recon, riemannSolver=riemann)
    from grim_b200.timestepper import timeStepper
    ts = timeStepper(cfg)
    P = _with_images(ts, _state(cfg, 2))
    g = cfg["numGhost"]
    rng = np.random.default_rng(1)
    gbar = np.zeros_like(P)
    gbar[:, :, g:g + 16, g:g + 16] = rng.standard_normal((8, 1, 16, 16))
    vjp = ts.adjointStencil(P, gbar)

    def f(Q):
        return float(np.sum(gbar * ts.computeDivOfFluxes(Q)[0]))

    h = 1e-6
    for v in range(8):
        j, i = rng.integers(0, 16, 2)
        Pp, Pm = P.copy(), P.copy()
        Pp[v, 0, j + g, i + g] += h
        Pm[v, 0, j + g, i + g] -= h
        fd = (f(_with_images(ts, Pp)) - f(_with_images(ts, Pm))) / (2 * h)
        ad = vjp[v, 0, j + g, i + g]
        assert abs(fd - ad) <= 1e-6 * max(abs(ad), 1e-3 * np.max(np.abs(vjp))), (v, j, i, fd, ad)


# ---- 3D periodic ------------------------------------------------------------
def _cfg3(N=12, **kw):
    return PR.fast_mode_config(N=N, N3=N, dim=3, **kw)


def _state3(cfg, seed, amp=1e-2):
    rng = np.random.default_rng(seed)
    X1, X2, X3 = C.cell_centers(cfg)
    P = np.zeros((8,) + X1.shape)
    for v in range(8):
        k1, k2, k3 = rng.integers(1, 3, 3)
        ph = rng.uniform(0, 2 * np.pi, 3)
        P[v] = BG[v] + amp * (np.sin(2 * np.pi * k1 * X1 + ph[0]) * np.cos(2 * np.pi * k2 * X2 + ph[1])
                              * np.cos(2 * np.pi * k3 * X3 + ph[2]))
    return P


def _adjoint3(cfg, P, nsteps, every):
    ts = _stepper(cfg, P)
    ts.adjointForward(nsteps, every)
    Pf = ts.primOld.getVars()
    lam = np.zeros_like(Pf)
    sl = (slice(None),) + tuple(C.interior_slices(cfg))
    lam[sl] = Pf[sl] - BG[:, None, None, None]
    return ts.adjointBackward(lam)


@pytest.mark.parametrize("recon,riemann", [(C.MINMOD, C.LOCAL_LAX_FRIEDRICH), (C.PPM, C.HLL)])
def test_stencil_transpose_matches_fd_3d(recon, riemann):
    """The 3D stencil transpose (three face directions, the three edge EMFs
    of flux-CT, ghosts as periodic images in every direction) against
    central differences of <gbar, divF(P)> (an exactly rounded sum).  The
    map is piecewise smooth (the limiters; the Riemann solvers' min / max of
    speeds, which tie often around a fluid at rest), so the entries are
    screened and checked as in the whole-run test: at least 12 of 40
    random picks must qualify, and every one that does must match."""
    import math
    N = 10
    cfg = _cfg3(N, reconstruction=recon, riemannSolver=riemann)
    from grim_b200.timestepper import timeStepper
    ts = timeStepper(cfg)
    P = _with_images(ts, _state3(cfg, 2))
    g = cfg["numGhost"]
    rng = np.random.default_rng(1)
    gbar = np.zeros_like(P)
    gbar[:, g:g + N, g:g + N, g:g + N] = rng.standard_normal((8, N, N, N))
    vjp = ts.adjointStencil(P, gbar)

    def f(Q):
        return math.fsum((gbar * ts.computeDivOfFluxes(Q)[0]).ravel().tolist())

    def shifted(v, k, j, i, h):
        Q = P.copy()
        Q[v, k + g, j + g, i + g] += h
        return f(_with_images(ts, Q))

    picks = [(n % 8,) + tuple(int(x) for x in rng.integers(0, N, 3)) for n in range(40)]
    smooth, bad = fd_check(shifted, f(P), interior(cfg, vjp), picks, float(np.max(np.abs(vjp))))
    assert not bad, bad
    assert smooth >= 12, smooth


def test_adjoint_matches_central_fd_3d():
    """Whole checkpointed runs in 3D (12^3, 4 steps, checkpoints every 2),
    screened and checked as the 2D runs are."""
    N, nsteps = 12, 4
    cfg = _cfg3(N, reconstruction=C.PPM, riemannSolver=C.HLL, maxNonLinearIter=6, nonlinearsolve_atol=0.0)
    P = _state3(cfg, 7)
    grad = _adjoint3(cfg, P, nsteps, every=2)
    g = cfg["numGhost"]
    gi = interior(cfg, grad)
    assert np.all(grad[:, :g] == 0) and np.all(grad[:, :, :g] == 0) and np.all(grad[:, :, :, :g] == 0)
    scale = np.max(np.abs(gi))
    L0 = _loss(cfg, P, nsteps)

    def shifted(v, k, j, i, h):
        Q = P.copy()
        Q[v, k + g, j + g, i + g] += h
        return _loss(cfg, Q, nsteps)

    rng = np.random.default_rng(9)
    picks = [(n % 8,) + tuple(int(x) for x in rng.integers(0, N, 3)) for n in range(40)]
    smooth, bad = fd_check(shifted, L0, gi, picks, scale)
    assert not bad, bad
    assert smooth >= 8, smooth


def test_adjoint_checkpoint_interval_does_not_change_the_gradient_3d():
    cfg = _cfg3(10, maxNonLinearIter=6, nonlinearsolve_atol=0.0)
    P = _state3(cfg, 3)
    a = _adjoint3(cfg, P, 4, every=1)
    b = _adjoint3(cfg, P, 4, every=3)
    assert np.array_equal(a, b)


# ---- modified Kerr-Schild, outflow / mirror / periodic ------------------------
def _mks_cfg(N1=16, N2=16, N3=8, recon=C.PPM, riemann=C.LOCAL_LAX_FRIEDRICH, **kw):
    """The torus grid's metric and boundaries (spin 0.9375, MKS with the
    horizon derefinement and cylindrification, outflow in X1, mirror in X2,
    periodic in X3) on a small grid out to r = 40, without the torus
    problem hooks (floors, inflow check, pole fix, flux filter)."""
    import math
    from grim_b200.problems import torus as T
    return T.torus_config(N1=N1, N2=N2, N3=N3, problem=C.PROBLEM_NONE, X1End=math.log(40.), reconstruction=recon,
                          riemannSolver=riemann, dt=2e-3, maxNonLinearIter=8, nonlinearsolve_atol=0.0, **kw)


MKS_BG = np.array([1.0, 0.5, 0.0, 0.0, 0.0, 0.05, 0.02, 0.01])


def _mks_state(cfg, seed, amp=1e-2):
    """rho ~ 1, u ~ 0.5, small velocities and field, smooth in X1, X2, X3"""
    rng = np.random.default_rng(seed)
    X1, X2, X3 = C.cell_centers(cfg)
    bg = MKS_BG
    P = np.zeros((8,) + X1.shape)
    for v in range(8):
        k1, k2, k3 = rng.integers(1, 3, 3)
        ph = rng.uniform(0, 2 * np.pi, 3)
        P[v] = bg[v] + amp * (np.sin(2 * np.pi * k1 * X1 / 3. + ph[0]) * np.cos(2 * np.pi * k2 * X2 + ph[1])
                              * np.cos(k3 * X3 + ph[2]))
    return P


def _mks_stepper(cfg, P):
    from grim_b200.timestepper import timeStepper
    ts = timeStepper(cfg)
    ts.setNewtonMode(C.NEWTON_TANGENT64, 1, 0.0)
    ts.primOld.setVars(P)
    ts.primOld.communicate()
    ts.setTime(0.0, cfg["dt"])
    ts.setFixedDt(True)
    return ts


def _mks_loss(cfg, P, nsteps):
    """L = 1/2 sum over the interior of (P_final - background)^2, exactly
    rounded (the screen of fd_check counts two ulps of L per evaluation)"""
    from tests.adjoint_harness import energy
    ts = _mks_stepper(cfg, P)
    for _ in range(nsteps):
        ts.timeStep()
    assert ts.stats()["nonFinite"] == 0
    return energy(cfg, ts.primOld.getVars(), MKS_BG)


def test_stencil_transpose_matches_fd_mks():
    """The stencil transpose with the face metric and the outflow / mirror /
    periodic ghost fill of the torus grid, against central differences of
    <gbar, divF(P)> (ghosts from the boundary fill), screened as above."""
    import math
    cfg = _mks_cfg(N1=12, N2=12, N3=6)
    from grim_b200.timestepper import timeStepper
    ts = timeStepper(cfg)
    P = _with_images(ts, _mks_state(cfg, 4))
    g = cfg["numGhost"]
    rng = np.random.default_rng(2)
    gbar = np.zeros_like(P)
    sl = (slice(None),) + tuple(C.interior_slices(cfg))
    gbar[sl] = rng.standard_normal(gbar[sl].shape)
    vjp = ts.adjointStencil(P, gbar)

    def f(Q):
        return math.fsum((gbar * ts.computeDivOfFluxes(Q)[0]).ravel().tolist())

    def shifted(v, k, j, i, h):
        Q = P.copy()
        Q[v, k + g, j + g, i + g] += h
        return f(_with_images(ts, Q))

    # the boundary zones (whose ghosts copy them) are picked on purpose
    picks = [(n % 8, int(rng.integers(0, 6)), int(rng.choice([0, 1, 5, 10, 11])), int(rng.choice([0, 4, 11])))
             for n in range(32)]
    smooth, bad = fd_check(shifted, f(P), interior(cfg, vjp), picks, float(np.max(np.abs(vjp))))
    assert not bad, bad
    assert smooth >= 10, smooth


def test_adjoint_matches_central_fd_mks():
    """Whole checkpointed runs on the torus grid's metric and boundaries
    (12x12x6, 3 steps, checkpoints every 2): the geometric source's
    transpose, the face metric, the MKS conserved variables and field
    update, the outflow / mirror ghost fill.  The grid starts at r = 2.5:
    from the torus grid's inner edge (inside the horizon) this fluid at
    rest, with no floors or inflow check, turns non-finite in the first
    three columns within a step (measured), and the check needs a finite
    forward map."""
    import math
    cfg = _mks_cfg(N1=12, N2=12, N3=6, X1Start=math.log(2.5))
    P = _mks_state(cfg, 6)
    nsteps = 3
    ts = _mks_stepper(cfg, P)
    ts.adjointForward(nsteps, 2)
    Pf = ts.primOld.getVars()
    lam = np.zeros_like(Pf)
    sl = (slice(None),) + tuple(C.interior_slices(cfg))
    lam[sl] = Pf[sl] - MKS_BG[:, None, None, None]
    grad = ts.adjointBackward(lam)
    g = cfg["numGhost"]
    gi = interior(cfg, grad)
    L0 = _mks_loss(cfg, P, nsteps)

    def shifted(v, k, j, i, h):
        Q = P.copy()
        Q[v, k + g, j + g, i + g] += h
        return _mks_loss(cfg, Q, nsteps)

    rng = np.random.default_rng(3)
    picks = [(n % 8, int(rng.integers(0, 6)), int(rng.choice([0, 1, 6, 10, 11])), int(rng.choice([0, 5, 11])))
             for n in range(32)]
    smooth, bad = fd_check(shifted, L0, gi, picks, float(np.max(np.abs(gi))))
    if bad:
        raise AssertionError("entries off the central differences: %s" % str(bad))
    assert smooth >= 10, smooth


# ---- the torus problem: floors, inflow check, pole fix, flux filter ------------
def test_adjoint_matches_central_fd_torus():
    """Whole checkpointed runs of the torus problem itself (Fishbone-Moncrief
    torus in its atmosphere, 16x12x6 from r = 2.5 to 100, 3 steps,
    checkpoints every 2): the
    floors after each stage (their local Jacobian at each stage's Newton
    solution), the inflow check and the pole fix at the start of each stage
    and the flux filter, on top of the MKS transposes.  The floors make the
    map piecewise smooth at the atmosphere's floor values; the screen of
    fd_check skips picks at a switch.  The two rows next to each pole are
    overwritten from the third by the pole fix before anything reads them,
    so the gradient of their fluid variables is exactly zero.  From the
    torus grid's inner edge (inside the horizon) this coarse grid's first
    columns go non-finite and are reset to the floors every step (measured);
    the reset's zones carry no derivative, and the central differences need
    a map without resets, hence r >= 2.5 here."""
    import math
    from grim_b200.problems import torus as T
    from grim_b200.timestepper import timeStepper
    cfg = T.torus_config(N1=16, N2=12, N3=6, dt=1e-3, maxNonLinearIter=8, nonlinearsolve_atol=0.0,
                         X1Start=math.log(2.5), X1End=math.log(100.))
    init = timeStepper(cfg)
    P, _ = T.torus_prims(cfg, init.getGeometry(C.CENTER))
    init.primOld.setVars(P)
    init.problemInit()  # the field loop, the perturbation, the floors
    P0 = init.primOld.getVars()
    g = cfg["numGhost"]
    sl = (slice(None),) + tuple(C.interior_slices(cfg))
    assert np.isfinite(P0[sl]).all()
    # the initial torus is exactly axisymmetric, with exactly zero field
    # outside the loop: every X3 face sits at a switch of the limiters and of
    # the Riemann solver's speed min / max, where a central difference
    # averages two branches; a seeded 1e-3 perturbation of every variable
    # moves the state off those switches
    rng0 = np.random.default_rng(17)
    Q = P0[sl]
    Q[:5] *= 1. + 1e-3 * rng0.uniform(-1., 1., Q[:5].shape)
    # the atmosphere is at rest: its velocities are exactly zero, where the
    # reconstruction's limiters and the speed extrema sit at their switches;
    # an additive perturbation moves them off
    Q[2:5] += 1e-5 * rng0.uniform(-1., 1., Q[2:5].shape)
    Q[5:] += 1e-6 * rng0.uniform(-1., 1., Q[5:].shape)
    P0[sl] = Q
    ref = np.array(P0[sl])

    def stepper(P):
        ts = _mks_stepper(cfg, P)
        return ts

    def loss(P):
        ts = stepper(P)
        for _ in range(nsteps):
            ts.timeStep()
            # no zone went through the NaN reset
            assert np.isfinite(ts.prim.getVars()[sl]).all()
        d = (ts.primOld.getVars()[sl] - ref).ravel()
        return 0.5 * math.fsum((d * d).tolist())

    nsteps = 3
    ts = stepper(P0)
    ts.adjointForward(nsteps, 2)
    Pf = ts.primOld.getVars()
    lam = np.zeros_like(Pf)
    lam[sl] = Pf[sl] - ref
    gi = interior(cfg, ts.adjointBackward(lam))
    assert np.isfinite(gi).all()
    assert np.all(gi[:5, :, :2, :] == 0.) and np.all(gi[:5, :, -2:, :] == 0.)
    L0 = loss(P0)

    def shifted(v, k, j, i, h):
        Q = P0.copy()
        Q[v, k + g, j + g, i + g] += h
        return loss(Q)

    rng = np.random.default_rng(5)
    picks = [(n % 8, int(rng.integers(0, 6)), int(rng.integers(2, 10)), int(rng.choice([0, 1, 3, 6, 9, 15])))
             for n in range(40)]
    smooth, bad = fd_check(shifted, L0, gi, picks, float(np.max(np.abs(gi))))
    if bad:
        raise AssertionError("entries off the central differences: %s" % str(bad))
    assert smooth >= 8, smooth


def test_adjoint_matches_central_fd_torus_emhd():
    """The torus problem with conduction and viscosity (its closure: tau
    from the dynamical time limited by the q and deltaP bounds; the floors'
    q and deltaP limiters, their local Jacobian at each stage's Newton
    solution; the pole fix's scaled and mirrored q and deltaP) on the run of
    the ideal torus test (16x12x6 from r = 2.5, 3 steps, checkpoints every
    2), against Richardson-extrapolated central differences as for the
    other EMHD runs."""
    import math
    from grim_b200.problems import torus as T
    from grim_b200.timestepper import timeStepper
    cfg = T.torus_config(N1=16, N2=12, N3=6, emhd=True, dt=1e-3, maxNonLinearIter=8, nonlinearsolve_atol=0.0,
                         X1Start=math.log(2.5), X1End=math.log(100.))
    init = timeStepper(cfg)
    P, _ = T.torus_prims(cfg, init.getGeometry(C.CENTER))
    init.primOld.setVars(P)
    init.problemInit()
    P0 = init.primOld.getVars()
    g = cfg["numGhost"]
    sl = (slice(None),) + tuple(C.interior_slices(cfg))
    assert np.isfinite(P0[sl]).all()
    dof, nf = C.var_counts(cfg)
    # off the axisymmetric ties (as in the ideal torus test), and q, deltaP
    # off their initial zeros (a fraction of the pressure)
    rng0 = np.random.default_rng(17)
    Q = P0[sl]
    Q[:5] *= 1. + 1e-3 * rng0.uniform(-1., 1., Q[:5].shape)
    Q[2:5] += 1e-5 * rng0.uniform(-1., 1., Q[2:5].shape)  # off the atmosphere's zero velocities
    pres = (cfg["adiabaticIndex"] - 1.) * Q[1]
    Q[5:nf] = 1e-3 * pres * rng0.uniform(-1., 1., Q[5:nf].shape)
    Q[nf:] += 1e-6 * rng0.uniform(-1., 1., Q[nf:].shape)
    P0[sl] = Q
    ref = np.array(P0[sl])

    def loss(P):
        ts = _mks_stepper(cfg, P)
        for _ in range(nsteps):
            ts.timeStep()
            if not np.isfinite(ts.prim.getVars()[sl]).all():
                # a zone the NaN reset replaces: off the map the adjoint
                # differentiates (the check skips the pick)
                return math.nan
        d = (ts.primOld.getVars()[sl] - ref).ravel()
        return 0.5 * math.fsum((d * d).tolist())

    nsteps = 3
    ts = _mks_stepper(cfg, P0)
    ts.adjointForward(nsteps, 2)
    Pf = ts.primOld.getVars()
    lam = np.zeros_like(Pf)
    lam[sl] = Pf[sl] - ref
    gi = interior(cfg, ts.adjointBackward(lam))
    assert np.isfinite(gi).all()
    assert np.all(gi[:nf, :, :2, :] == 0.) and np.all(gi[:nf, :, -2:, :] == 0.)
    L0 = loss(P0)
    assert math.isfinite(L0)

    def shifted(v, k, j, i, h):
        Q = P0.copy()
        Q[v, k + g, j + g, i + g] += h
        return loss(Q)

    # X1 columns from the fourth on: in the first three the density (a few
    # 1e-5) crosses the floors within the differences' +-4e-6, and the
    # differences settle on the adjoint only below h = 1e-8 (measured)
    rng = np.random.default_rng(5)
    picks = [(n % dof, int(rng.integers(0, 6)), int(rng.integers(2, 10)), int(rng.choice([3, 6, 9, 12, 15])))
             for n in range(40)]
    smooth, bad = fd_check_richardson(shifted, L0, gi, picks, float(np.max(np.abs(gi))), rtol=1e-5)
    if bad:
        raise AssertionError("entries off the central differences: %s" % str(bad))
    assert smooth >= 10, smooth


# ---- extended MHD: conduction and viscosity ------------------------------------
def _emhd_cfg(N=12, cond=1, visc=1, **kw):
    """The damped EMHD linear-mode problem's set-up (Minkowski, periodic, the
    high-order terms, constant-tau closure), WENO5 / HLL, Newton run to
    roundoff (8 updates of the exact FP64 tangent)."""
    return PR.linear_modes_config(N=N, conduction=cond, viscosity=visc, reconstruction=C.WENO5, riemannSolver=C.HLL,
                                  maxNonLinearIter=8, nonlinearsolve_atol=0.0, **kw)


def _emhd_state(cfg, seed, amp=1e-2):
    """the linear mode at amplitude amp plus seeded smooth perturbations of
    every variable"""
    rng = np.random.default_rng(seed)
    P = PR.linear_modes_prims(cfg, amplitude=amp)
    X1, X2, _ = C.cell_centers(cfg)
    for v in range(P.shape[0]):
        k1, k2 = rng.integers(1, 3, 2)
        ph = rng.uniform(0, 2 * np.pi, 2)
        P[v] += 0.3 * amp * np.sin(2 * np.pi * k1 * X1 + ph[0]) * np.cos(2 * np.pi * k2 * X2 + ph[1])
    return P


@pytest.mark.parametrize("cond,visc", [(1, 1), (1, 0), (0, 1)])
def test_stencil_transpose_matches_fd_emhd(cond, visc):
    """The stencil transpose with the EMHD variables (q, deltaP in the
    reconstruction, the Riemann solver's fluxes and speeds), against
    Richardson-extrapolated central differences of <gbar, divF(P)>."""
    import math
    N = 12
    cfg = _emhd_cfg(N, cond, visc)
    from grim_b200.timestepper import timeStepper
    ts = timeStepper(cfg)
    P = _with_images(ts, _emhd_state(cfg, 2))
    g = cfg["numGhost"]
    rng = np.random.default_rng(1)
    gbar = np.zeros_like(P)
    sl = (slice(None),) + tuple(C.interior_slices(cfg))
    gbar[sl] = rng.standard_normal(gbar[sl].shape)
    vjp = ts.adjointStencil(P, gbar)

    def f(Q):
        return math.fsum((gbar * ts.computeDivOfFluxes(Q)[0]).ravel().tolist())

    def shifted(v, j, i, h):
        Q = P.copy()
        Q[v, 0, j + g, i + g] += h
        return f(_with_images(ts, Q))

    dof = P.shape[0]
    picks = [(n % dof,) + tuple(int(x) for x in rng.integers(0, N, 2)) for n in range(3 * dof)]
    smooth, bad = fd_check_richardson(shifted, f(P), interior(cfg, vjp)[:, 0], picks, float(np.max(np.abs(vjp))))
    assert not bad, bad
    assert smooth >= 2 * dof, smooth


@pytest.mark.parametrize("cond,visc", [(1, 1), (1, 0), (0, 1)])
def test_adjoint_matches_central_fd_emhd(cond, visc):
    """Whole checkpointed EMHD runs (12^2, 3 steps, checkpoints every 2): the
    stage adjoint through the EMHD residual (its time-derivative and
    implicit-source terms, the row normalisation of q and deltaP), the
    stage constants' dependence on the old state (elemOld) and on the
    stage's reference element, and the EMHD source's gradients of u_mu and
    T over the neighbouring zones."""
    import math
    N, nsteps = 12, 3
    cfg = _emhd_cfg(N, cond, visc)
    P0 = _emhd_state(cfg, 6)
    g = cfg["numGhost"]
    sl = (slice(None),) + tuple(C.interior_slices(cfg))
    bg = P0[sl].mean(axis=(1, 2, 3))

    def loss(P):
        ts = _stepper(cfg, P)
        for _ in range(nsteps):
            ts.timeStep()
        d = (ts.primOld.getVars()[sl] - bg[:, None, None, None]).ravel()
        return 0.5 * math.fsum((d * d).tolist())

    ts = _stepper(cfg, P0)
    ts.adjointForward(nsteps, 2)
    Pf = ts.primOld.getVars()
    lam = np.zeros_like(Pf)
    lam[sl] = Pf[sl] - bg[:, None, None, None]
    gi = interior(cfg, ts.adjointBackward(lam))[:, 0]
    assert np.isfinite(gi).all()
    L0 = loss(P0)

    def shifted(v, j, i, h):
        Q = P0.copy()
        Q[v, 0, j + g, i + g] += h
        return loss(Q)

    rng = np.random.default_rng(4)
    dof = P0.shape[0]
    picks = [(n % dof,) + tuple(int(x) for x in rng.integers(0, N, 2)) for n in range(3 * dof)]
    # the EMHD map's third derivatives put the plain 1e-6 difference's
    # truncation error near 1e-6 (measured): Richardson-extrapolated
    # differences instead.  The forward map itself moves by up to 1e-5 of
    # these derivatives between 8 and 15 Newton updates (measured: the EMHD
    # Newton converges to its own floor, not to roundoff), and the adjoint
    # is the derivative of the exact solution map, so the check is at 1e-5
    # here (the stencil transpose, with no Newton in it, holds at 1e-6)
    smooth, bad = fd_check_richardson(shifted, L0, gi, picks, float(np.max(np.abs(gi))), rtol=1e-5)
    if bad:
        raise AssertionError("entries off the central differences: %s" % str(bad))
    assert smooth >= 2 * dof, smooth
