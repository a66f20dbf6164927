"""The 3D Fishbone-Moncrief torus in modified Kerr-Schild coordinates
(src/problem/torus): geometry, initial floors and timesteps of the CUDA
path against the CPU oracle.

Tolerances: the metric (transcendental functions of CUDA vs glibc, 1-2 ulp)
to 1e-12 relative; the Christoffel symbols, central differences with
eps = 1e-5 of that metric, to 1e-6 of each component's scale; the
primitives after the initial floors and after timesteps to 1e-12 of each
variable's scale, with the oracle's geometry loaded into the GPU handle so
the comparison isolates the timestep.
"""
import numpy as np
import pytest

from grim_b200 import config as C
from grim_b200.problems import torus as T
from tests.helpers import interior, scaled_err

pytestmark = pytest.mark.gpu

SHAPE = dict(N1=64, N2=32, N3=8)


def _pair():
    from grim_b200.timestepper import timeStepper
    from oracle.oracle import Oracle
    cfg = T.torus_config(**SHAPE)
    return cfg, timeStepper(cfg), Oracle(cfg)


def _natural_err(a, b, keep):
    """max over zones of |a_ij - b_ij| / sqrt(|b_ii b_jj|) for each (i, j):
    the error of a metric entry measured against the size the diagonal sets
    for it, so that an off-diagonal entry that passes near zero is not held
    to its own (vanishing) magnitude; the scale is floored at 1e-6 of its
    largest value on the grid.  Only zones where keep is true count."""
    out = np.zeros((4, 4))
    for i, j in np.ndindex(4, 4):
        s = np.sqrt(np.abs(b[i, i] * b[j, j]))
        # floor: g_33 ~ sin^2(theta) vanishes on the polar faces
        s = np.maximum(s, 1e-6 * np.nanmax(s))
        m = ~np.isnan(b[i, j]) & (s > 0) & keep
        out[i, j] = np.max(np.abs(a[i, j][m] - b[i, j][m]) / s[m])
    return out


def test_mks_geometry_matches_oracle():
    """The metric entries agree to 1e-9 of their natural scale
    sqrt(|g_ii g_jj|) per zone, g = sqrt(-det g) and alpha to 1e-9 relative. dr/dX and
    dtheta/dX are central differences (eps = 1e-5) of exp/acos/asin
    compositions, which turn the last-ulp differences between CUDA's and
    glibc's functions into ~1e-11 of a derivative; the Christoffels, second
    differences, agree to 1e-5 of their component's scale (at least 1e-3:
    components that vanish analytically carry FD noise of ~1e-11).

    Zones on the polar axis (|sin theta| < 1e-6: the X2 = 0 and X2 = 1
    faces) are left out of the per-zone relative checks: theta there is
    zero analytically and both sides get ~1e-8 from cancellation in the
    cylindrified map, so g_33 ~ sin^2 theta and g^33 ~ 1/sin^2 theta have
    no meaningful relative error; theta itself must agree to 1e-15 there."""
    cfg, ts, orc = _pair()
    for loc in (C.CENTER, C.LEFT, C.BOTTOM):
        g = ts.getGeometry(loc)
        o = orc.geometry(loc)
        th = np.asarray(o["x"][1])
        keep = ~(np.abs(np.sin(th)) < 1e-6)
        for key in ("gCov", "gCon"):
            a, b = np.asarray(g[key]), np.asarray(o[key])
            assert np.array_equal(np.isnan(a), np.isnan(b)), (loc, key)
            err = _natural_err(a, b, keep)
            assert err.max() <= 1e-9, (loc, key, err)
        for key in ("g", "alpha"):
            a, b = np.asarray(g[key]), np.asarray(o[key])
            assert np.array_equal(np.isnan(a), np.isnan(b)), (loc, key)
            m = ~np.isnan(b) & keep
            assert np.max(np.abs(a[m] - b[m]) / np.abs(b[m])) <= 1e-9, (loc, key)
        xa, xb = np.asarray(g["x"][:2]), np.asarray(o["x"][:2])
        assert np.allclose(xa[:, keep], xb[:, keep], rtol=1e-13, atol=0, equal_nan=True), loc
        polar = ~keep & ~np.isnan(th)
        assert np.all(np.abs(xa[1][polar] - xb[1][polar]) <= 1e-15), loc
        if loc == C.CENTER:
            a, b = g["gamma"], o["gamma"]
            for idx in np.ndindex(4, 4, 4):
                m = ~np.isnan(b[idx])
                s = np.abs(b[idx][m]).max()
                # components that vanish analytically are FD noise (~1e-11)
                assert np.max(np.abs(a[idx][m] - b[idx][m])) <= 1e-5 * max(s, 1e-3), idx


def _load_oracle_geometry(ts, orc):
    for loc in (C.CENTER, C.LEFT, C.BOTTOM, C.RIGHT, C.TOP):
        o = orc.geometry(loc)
        ts.setGeometry(loc, o["gCov"], o["gCon"], o["g"], o["alpha"], x=o["x"],
                       gamma=o["gamma"] if loc == C.CENTER else None)


def test_torus_init_and_steps_match_oracle():
    cfg, ts, orc = _pair()
    _load_oracle_geometry(ts, orc)
    P, info = T.torus_prims(cfg, orc.geometry(C.CENTER))
    assert np.isfinite(info["BFactor"]) and not np.isnan(P).any()
    ts.primOld.setVars(P)
    orc.set_prims(P)
    ts.problemInit()
    orc.problem_init()
    g0 = ts.primOld.getVars()
    o0 = orc.get_prims()
    assert scaled_err(interior(cfg, g0), interior(cfg, o0)) <= 1e-12
    for n in range(3):
        ts.timeStep()
        orc.time_step(1)
        assert abs(ts.dt - orc.dt) <= 1e-13 * orc.dt, n
        g = interior(cfg, ts.primOld.getVars())
        o = interior(cfg, orc.get_prims())
        assert not np.isnan(g).any()
        assert scaled_err(g, o) <= 1e-12, (n, scaled_err(g, o))
    st = ts.stats()
    assert st["nonFinite"] == 0


def test_torus_observers_match_oracle():
    """ObserversTorus.hpp on the same primOld (the oracle's, after the
    initial floors and two steps): the per-zone integrands are the same
    arithmetic on both sides, so the sums agree to their summation order
    (1e-13 of their magnitude) and the extrema exactly."""
    cfg, ts, orc = _pair()
    _load_oracle_geometry(ts, orc)
    P, _ = T.torus_prims(cfg, orc.geometry(C.CENTER))
    orc.set_prims(P)
    orc.problem_init()
    orc.time_step(2)
    ts.primOld.setVars(orc.get_prims())
    g = ts.torusObservers()
    o = orc.torus_observers()
    assert g["BaryonMass"] > 0 and g["ETh"] > 0 and g["EMag"] > 0
    for k, b in o.items():
        a = g[k]
        if k in ("rhoMax", "betaMin"):
            assert a == b, (k, a, b)
        else:
            assert abs(a - b) <= 1e-13 * max(abs(b), 1e-300), (k, a, b)


def test_observations_recorded_by_the_steps():
    """With ObserveEveryDt set, every step whose time crosses a multiple of
    it (problem.cpp:754) leaves one record {time, observers}; the last one
    equals grim_torus_observers on the state that step left."""
    from grim_b200.timestepper import timeStepper
    cfg = T.torus_config(**SHAPE, ObserveEveryDt=0.004)
    ts = timeStepper(cfg)
    from oracle.oracle import Oracle
    orc = Oracle(cfg)
    _load_oracle_geometry(ts, orc)
    P, _ = T.torus_prims(cfg, orc.geometry(C.CENTER))
    ts.primOld.setVars(P)
    ts.problemInit()
    E = cfg["ObserveEveryDt"]
    due = []
    last = None
    for n in range(6):
        t0 = ts.time
        ts.timeStep()
        t1, dt = ts.time, ts.dt
        if np.floor(t1 / E) != np.floor((t1 - dt) / E):
            due.append(t1)
            last = ts.torusObservers()
        assert abs((t1 - t0) - dt) <= 1e-15 * t1
    recs = ts.observations()
    assert len(due) >= 2 and len(recs) == len(due)
    assert [r["time"] for r in recs] == due
    for k, v in last.items():
        assert recs[-1][k] == v, k


def test_torus_emhd_steps_match_oracle():
    """The torus with conduction and viscosity (nf = 7, the torus closure of
    problem.cpp:7-55 and the MKS EMHD gradients): initial floors and three
    steps of the FP64 parity path against the oracle, with the oracle's
    geometry in the handle.  The stage pieces agree bit for bit (flux
    divergence, the half stage's residual and its Newton solution); the
    closure's exp and pow differ from glibc's in the last ulp, and this
    configuration (FD Jacobian with eps = 4e-8, three iterations, global
    break) carries such differences far: the oracle itself, started from a
    state one ulp away, moves by up to 1e-5 of a variable's scale in three
    steps.  Each variable must stay within 10x that sensitivity."""
    from grim_b200.timestepper import timeStepper
    from oracle.oracle import Oracle
    cfg = T.torus_config(**SHAPE, emhd=True)
    ts, orc, orc2 = timeStepper(cfg), Oracle(cfg), Oracle(cfg)
    _load_oracle_geometry(ts, orc)
    P, _ = T.torus_prims(cfg, orc.geometry(C.CENTER))
    ts.primOld.setVars(P)
    for o in (orc, orc2):
        o.set_prims(P)
        o.problem_init()
    ts.problemInit()
    assert scaled_err(interior(cfg, ts.primOld.getVars()), interior(cfg, orc.get_prims())) == 0.
    Q = orc2.get_prims()
    Q[:5] = np.nextafter(Q[:5], np.inf)  # one ulp up in the fluid variables
    orc2.set_prims(Q)
    for n in range(3):
        ts.timeStep()
        orc.time_step(1)
        orc2.time_step(1)
        assert abs(ts.dt - orc.dt) <= 1e-12 * orc.dt, n
        g = interior(cfg, ts.primOld.getVars())
        o = interior(cfg, orc.get_prims())
        o2 = interior(cfg, orc2.get_prims())
        assert not np.isnan(g).any()
        for v in range(g.shape[0]):
            err = scaled_err(g[v:v + 1], o[v:v + 1])
            sens = scaled_err(o2[v:v + 1], o[v:v + 1])
            assert err <= 10. * sens + 1e-12, (n, v, err, sens)
    assert np.max(np.abs(interior(cfg, ts.primOld.getVars())[5:7])) > 0


def test_torus_2d_steps_match_oracle():
    """The axisymmetric torus (dim = 2, 64x32): initial floors and three
    steps against the oracle to 1e-12 of each variable's scale, the 2D
    paths of the MKS stencil (flux-CT with EMF3 only, zero-padded
    divergence, Christoffel sources)."""
    from grim_b200.timestepper import timeStepper
    from oracle.oracle import Oracle
    cfg = T.torus_config(N1=64, N2=32, N3=1, dim=2)
    ts, orc = timeStepper(cfg), Oracle(cfg)
    _load_oracle_geometry(ts, orc)
    P, info = T.torus_prims(cfg, orc.geometry(C.CENTER))
    assert np.isfinite(info["BFactor"])
    ts.primOld.setVars(P)
    orc.set_prims(P)
    ts.problemInit()
    orc.problem_init()
    assert scaled_err(interior(cfg, ts.primOld.getVars()), interior(cfg, orc.get_prims())) <= 1e-12
    for n in range(3):
        ts.timeStep()
        orc.time_step(1)
        assert abs(ts.dt - orc.dt) <= 1e-13 * orc.dt, n
        g = interior(cfg, ts.primOld.getVars())
        o = interior(cfg, orc.get_prims())
        assert not np.isnan(g).any()
        assert scaled_err(g, o) <= 1e-12, (n, scaled_err(g, o))


def _torus_stepper(mode, **kw):
    from grim_b200.timestepper import timeStepper
    cfg = dict(T.torus_config(**SHAPE), newtonMode=mode, perZoneConvergence=1, nonlinearsolve_rtol=1e-10,
               nonlinearsolve_atol=1e-24, **kw)
    ts = timeStepper(cfg)
    P, _ = T.torus_prims(cfg, ts.getGeometry(C.CENTER))
    ts.primOld.setVars(P)
    ts.problemInit()
    return cfg, ts


def _column_err(a, b, keep):
    """max over kept zones and columns of max_i |a[z,i,j] - b[z,i,j]| / max_i |b[z,i,j]|"""
    scale = np.max(np.abs(b), axis=-2, keepdims=True) + 1e-300
    return float(np.max((np.abs(a - b) / scale)[keep]))


def test_closed_form_jacobian_on_kerr_schild():
    """The closed-form ideal-MHD Jacobian the fast Newton uses on every torus
    step (physics.cpp:53-217 differentiated by hand) on the 64x32x8 torus,
    MKS with derefine and cylindrify, at the half stage's Newton guess:
      * against the generic forward-tangent pass of the residual (dual
        numbers, FP64): 1e-10 of each zone's column scale;
      * against a central difference of the FP64 residual with the step
        h_j = 1e-6 |P_j| for rho and u (the atmosphere holds them near
        1e-12: a larger step crosses the element's floors, a kink) and
        1e-6 max(|P_j|, 1e-2) for the velocities: 1e-6 of the column scale
        (O(h^2) plus roundoff / h);
      * the mixed Newton's FP32 Jacobian (the same closed form on FP32
        geometry) against the FP64 one: 3e-5 of the column scale, the
        stated error of the Jacobian the FP64 residual then corrects."""
    from grim_b200.timestepper import timeStepper as TS
    cfg, ts = _torus_stepper(C.NEWTON_PARITY_FD64)
    ts.stageSetup(C.HALF_STEP)
    guess = ts.prim.getVars()
    s3, s2, s1 = C.interior_slices(cfg)
    J64 = ts.jacobianForm(guess, TS.JAC_FAST64)
    Jdual = ts.jacobianForm(guess, TS.JAC_DUAL64)
    J32 = ts.jacobianForm(guess, TS.JAC_FAST32)
    assert np.array_equal(J64, ts.jacobianTangent(guess))
    keep = np.zeros(ts.zshape + (1, 1), bool)
    keep[s3, s2, s1] = True
    keep = np.broadcast_to(keep, J64.shape)
    assert np.all(np.isfinite(J64[keep]))
    assert _column_err(J64, Jdual, keep) <= 1e-10
    assert _column_err(J32, J64, keep) <= 3e-5
    nf = C.var_counts(cfg)[1]
    Jfd = np.zeros_like(J64)
    for j in range(nf):
        h = 1e-6 * (np.abs(guess[j]) if j < 2 else np.maximum(np.abs(guess[j]), 1e-2))
        h = np.where(h > 0, h, 1e-8)  # ghost zones (not compared) may hold zeros
        gp, gm = guess.copy(), guess.copy()
        gp[j] += h
        gm[j] -= h
        Jfd[..., :, j] = np.moveaxis((ts.computeResidual(gp) - ts.computeResidual(gm)) / (2 * h), 0, -1)
    assert _column_err(J64, Jfd, keep) <= 1e-6


def test_torus_fast_steps_match_parity_path():
    """The fast form of the torus step (FP32 closed-form Jacobian, FP64
    residual, per-zone convergence, FMA arithmetic, its fused floors / dt /
    NaN-count passes) against the FD64 parity path at the same relative
    tolerance and the torus's 3 Newton iterations, which leave zones above
    tolerance in both forms (about 5x more in the parity form), so the two
    differ by those zones' residuals, 1.5e-6 of the velocities' scale on a
    B200: three steps agree to 1e-5 of each variable's scale, with the same
    dt to 1e-9."""
    _, ref = _torus_stepper(C.NEWTON_PARITY_FD64)
    cfg, fast = _torus_stepper(C.NEWTON_MIXED32)
    for n in range(3):
        ref.timeStep()
        fast.timeStep()
        assert abs(fast.dt - ref.dt) <= 1e-9 * ref.dt, n
    a = interior(cfg, fast.primOld.getVars())
    b = interior(cfg, ref.primOld.getVars())
    assert not np.isnan(a).any()
    err = scaled_err(a, b)
    assert err <= 1e-5, err
    assert fast.stats()["nonFinite"] == 0


@pytest.mark.parametrize("mode", [C.NEWTON_PARITY_FD64, C.NEWTON_MIXED32])
def test_torus_nan_count_and_reset(mode):
    """fullStepDiagnostics (torus/problem.cpp:719-746): the count of interior
    zones of the full stage's Newton result that hold a NaN, then the reset
    of those zones before the floors.  The fast per-zone Newton counts them
    as it writes them, the parity path in a pass of its own.  A NaN planted
    in one interior zone's velocity spreads through the two stages'
    stencils; after the step's first three segments the count equals the
    NaN zones of the Newton result, and the finished step leaves the
    interior finite.  (A NaN density would not spread here: the element
    floors rho with fmax, which returns the floor for a NaN.)"""
    import ctypes
    import torch
    from grim_b200 import _lib
    from grim_b200.slab import SCALAR_NANFLAG, SEG_FULL, SEG_HALF, SEG_POST, SEG_PRE
    from grim_b200.timestepper import Grid
    cfg, ts = _torus_stepper(mode)
    P = ts.primOld.getVars()
    P[2, 3 + SHAPE["N3"] // 2, 3 + SHAPE["N2"] // 2, 3 + SHAPE["N1"] // 3] = np.nan
    ts.primOld.setVars(P)
    L = _lib.lib()
    for seg in (SEG_PRE, SEG_HALF, SEG_FULL):
        _lib.check(L.grim_step_segment(ts._h, seg), "step_segment")
    buf = torch.zeros(1, dtype=torch.int64, device="cuda")
    _lib.check(L.grim_scalar_get(ts._h, SCALAR_NANFLAG, ctypes.c_void_p(buf.data_ptr())), "scalar_get")
    ts.synchronize()
    count = int(buf.item())
    bad = int(np.isnan(interior(cfg, Grid(ts, _lib.PRIM).getVars())).any(axis=0).sum())
    assert count == bad and bad > 1, (count, bad)
    _lib.check(L.grim_step_segment(ts._h, SEG_POST), "step_segment")
    assert not np.isnan(interior(cfg, ts.primOld.getVars())).any()


def test_torus_full_size_fast_steps_properties():
    """At the bench's full size (256x128x64), three steps of the fast form
    (corner EMFs formed in the epilogue's flux half, FMA arithmetic):
    the corner divergence of sqrt(-g) B that flux-CT conserves (the 8 zones
    around each corner; computeDivB is the 2D form) stays at roundoff,
    below 1e-12 of |B| / dX1 at the corners away from the boundaries and
    the pole rows (the oracle holds it at ~7e-14 of that on the 64x32x8
    torus); the interior stays finite with no non-finite count; and two
    handles stepping the same state give the same bits (no order-dependent
    arithmetic in the step)."""
    from grim_b200.timestepper import timeStepper
    cfg = dict(T.torus_config(N1=256, N2=128, N3=64), newtonMode=C.NEWTON_MIXED32, perZoneConvergence=1,
               nonlinearsolve_rtol=1e-10, nonlinearsolve_atol=1e-24)
    a = timeStepper(cfg)
    P, _ = T.torus_prims(cfg, a.getGeometry(C.CENTER))
    b = timeStepper(cfg)
    for ts in (a, b):
        ts.primOld.setVars(P)
        ts.problemInit()
    for _ in range(3):
        a.timeStep()
        b.timeStep()
    Pa, Pb = a.primOld.getVars(), b.primOld.getVars()
    ia = interior(cfg, Pa)
    assert np.isfinite(ia).all()
    assert np.array_equal(Pa, Pb)
    assert a.stats()["nonFinite"] == 0 and a.dt > 0
    g = a.getGeometry(C.CENTER)["g"]
    dX = [(cfg["X1End"] - cfg["X1Start"]) / cfg["N1"], (cfg["X2End"] - cfg["X2Start"]) / cfg["N2"],
          (cfg["X3End"] - cfg["X3Start"]) / cfg["N3"]]
    d = _corner_divb_3d(Pa, g, dX)[3:-3, 5:-5, 3:-3]
    scale = float(np.max(np.abs(ia[5:8]))) * cfg["N1"]
    assert np.max(np.abs(d)) <= 1e-12 * scale, (float(np.max(np.abs(d))), scale)


def _corner_divb_3d(P, g, dX):
    """div(sqrt(-g) B) at the corner below-left-front of zone (k+1, j+1,
    i+1) for array index (k, j, i): each direction's difference summed over
    the 4 zone pairs around the corner."""
    def sh(x, dk, dj, di):
        return x[1 - dk:x.shape[0] - dk, 1 - dj:x.shape[1] - dj, 1 - di:x.shape[2] - di]
    b1, b2, b3 = (g * P[5 + d] for d in range(3))
    d1 = sum(sh(b1, dk, dj, 0) - sh(b1, dk, dj, 1) for dk in (0, 1) for dj in (0, 1)) / (4 * dX[0])
    d2 = sum(sh(b2, dk, 0, di) - sh(b2, dk, 1, di) for dk in (0, 1) for di in (0, 1)) / (4 * dX[1])
    d3 = sum(sh(b3, 0, dj, di) - sh(b3, 1, dj, di) for dj in (0, 1) for di in (0, 1)) / (4 * dX[2])
    return d1 + d2 + d3
