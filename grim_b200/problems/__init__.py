"""Initial conditions and configs of the workloads the timestep is run on.

Initial conditions are set-up code (the reference's
``timeStepper::initialConditions`` hooks, src/problem/<name>/problem.cpp),
evaluated once on the host in FP64 with numpy and uploaded with
``set_prims``; they are not part of the timed path.

Workloads:
  * ``linear_modes``  -- the reference's damped EMHD eigenmode
    (linear_modes/params.cpp:45-69, problem.cpp:10-216), with its analytic
    solution; the known-answer check of the whole timestep.
  * ``fast_mode``     -- 2D ideal GRMHD, Minkowski 128^2 periodic, seeded
    1e-4 sinusoidal perturbation along k=(2pi,2pi), minmod/LLF.
  * ``orszag_tang``   -- 2D Orszag-Tang vortex 512^2, WENO5/HLL
    (ICs as orzag_tang/problem.cpp:3-34, u^i = gamma v^i).
  * ``emhd_stratified`` -- 2D EMHD 256^2, stratified density, tau(y) profile,
    MP5 reconstruction.
  * ``torus``         -- 3D Fishbone-Moncrief torus in MKS (torus/*).
  * ``ragged_batch``  -- 16 independent 2D ideal linear-mode problems of
    64^2 .. 512^2 (seeded), the batching and adjoint workload.
"""
import math

import numpy as np

from .. import config as C


def _blank(cfg):
    dof, _ = C.var_counts(cfg)
    return np.zeros((dof,) + tuple(reversed(C.total_dims(cfg))))


# --------------------------------------------------------------------------
# linear_modes: src/problem/linear_modes/params.cpp:4-105, problem.cpp:3-216
# --------------------------------------------------------------------------
LM_AW = 1.e-8
LM_K1 = 2. * math.pi
LM_K2 = 4. * math.pi
LM_GAMMA = -0.5533585207638141
LM_OMEGA = -3.6262571286888425
# eigenvector (cos, sin) coefficients, problem.cpp:164-185
LM_EIG = dict(
    RHO=(-0.518522524082246, 0.1792647678001878),
    U=(0.5516170736393813, 0.),
    U1=(0.008463122479547856, -0.011862022608466367),
    U2=(-0.16175466371870734, 0.034828080823603294),
    B1=(-0.05973794979640743, 0.03351707506150924),
    B2=(0.02986897489820372, -0.016758537530754618),
    Q=(0.5233486841539436, -0.04767672501939603),
    DP=(0.2909106062057657, -0.02159452055336572),
)
LM_BACKGROUND = dict(RHO=1., U=2., U1=0., U2=0., U3=0., B1=0.1, B2=0.3, B3=0., Q=0., DP=0.)


def linear_modes_config(N=64, **kw):
    base = dict(N1=N, N2=N, N3=1, dim=2, conduction=1, viscosity=1,
                highOrderTermsConduction=1, highOrderTermsViscosity=1,
                adiabaticIndex=4. / 3, reconstruction=C.MINMOD, riemannSolver=C.HLL,
                CourantFactor=0.9, dt=0.5 / N, closure=C.CLOSURE_CONST_TAU,
                closureTau0=1., elemOldFromFullStep=1)
    base.update(kw)
    return C.make_config(**base)


def linear_modes_prims(cfg, amplitude=LM_AW):
    """linear_modes/problem.cpp:115-216 (Minkowski: x = X)."""
    X1, X2, _ = C.cell_centers(cfg)
    idx = C.var_index(cfg)
    P = _blank(cfg)
    phase = LM_K1 * X1 + LM_K2 * X2
    cphi, sphi = np.cos(phase), np.sin(phase)
    for name, v in idx.items():
        P[v] = LM_BACKGROUND[name]
    for name, (cc, ss) in LM_EIG.items():
        if name in idx:
            P[idx[name]] = P[idx[name]] + amplitude * cphi * cc + amplitude * sphi * ss
    G = cfg["adiabaticIndex"]
    rho, u = P[idx["RHO"]], P[idx["U"]]
    pressure = (G - 1.) * u
    temperature = pressure / rho
    cs = np.sqrt(G * pressure / (rho + G * u))
    if "Q" in idx and cfg["highOrderTermsConduction"]:
        P[idx["Q"]] = P[idx["Q"]] / temperature / np.sqrt(rho * cfg["ConductionAlpha"] * cs * cs)
    if "DP" in idx and cfg["highOrderTermsViscosity"]:
        P[idx["DP"]] = P[idx["DP"]] / np.sqrt(temperature * rho * cfg["ViscosityAlpha"] * cs * cs)
    return P


def linear_modes_analytic(cfg, time, amplitude=LM_AW):
    """Analytic primitives (rho, u, u1, u2, q, dP, B1, B2) at ``time``;
    linear_modes/problem.cpp:223-296.  q and dP are the physical (not
    tilde) values."""
    X1, X2, _ = C.cell_centers(cfg)
    phase = LM_K1 * X1 + LM_K2 * X2 + LM_OMEGA * time
    cphi, sphi = np.cos(phase), np.sin(phase)
    damp = math.exp(LM_GAMMA * time)
    out = {}
    for name, (cc, ss) in LM_EIG.items():
        out[name] = LM_BACKGROUND[name] + (amplitude * cphi * cc + amplitude * sphi * ss) * damp
    return out


# finalTime of the run behind the published error table of Linear modes.ipynb
# (cell 1, N = 32..512).  params.cpp:18 sets finalTime = 2 but the published
# numbers are those of the run stopped at the first step past t = 0.5
# (grim.cpp:41, `while (time < finalTime)`): the table is reproduced there to
# its printed digits and at no other end time.
LM_PUBLISHED_FINAL_TIME = 0.5


def linear_modes_errors(cfg, P, time, amplitude=LM_AW):
    """The diagnostic the reference prints after every full step
    (linear_modes/problem.cpp:118-213): per variable, the Euclidean norm
    (af::norm's default) of the flattened difference between the element's
    value and the analytic mode at ``time``, over the whole local array
    including the ghost zones (elemOld is set on the ghosted grid), divided
    by N1*N2*N3.  q and deltaP are the element's physical values.  ``P`` is
    primOld after the step, ghosts as the step left them."""
    idx = C.var_index(cfg)
    an = linear_modes_analytic(cfg, time, amplitude)
    q, dP = emhd_physical(cfg, P)
    rho = np.maximum(P[idx["RHO"]], cfg["rhoFloorInFluidElement"])
    u = np.maximum(P[idx["U"]], cfg["uFloorInFluidElement"])
    num = dict(RHO=rho, U=u, U1=P[idx["U1"]], U2=P[idx["U2"]], B1=P[idx["B1"]],
               B2=P[idx["B2"]], Q=q, DP=dP)
    vol = float(cfg["N1"]) * float(cfg["N2"]) * float(cfg["N3"])
    return {k: float(np.linalg.norm((num[k] - an[k]).ravel())) / vol for k in num}


def emhd_physical(cfg, P):
    """(q, deltaP) from the tilde primitives, physics.cpp:120-148."""
    idx = C.var_index(cfg)
    G = cfg["adiabaticIndex"]
    rho = np.maximum(P[idx["RHO"]], cfg["rhoFloorInFluidElement"])
    u = np.maximum(P[idx["U"]], cfg["uFloorInFluidElement"])
    pressure = (G - 1.) * u
    T = np.maximum(pressure / rho, cfg["temperatureFloorInFluidElement"])
    cs = np.sqrt(G * pressure / (rho + G * u))
    q = P[idx["Q"]] * T * np.sqrt(rho * cfg["ConductionAlpha"] * cs * cs) \
        if cfg["highOrderTermsConduction"] else P[idx["Q"]]
    dP = P[idx["DP"]] * np.sqrt(T * rho * cfg["ViscosityAlpha"] * cs * cs) \
        if cfg["highOrderTermsViscosity"] else P[idx["DP"]]
    return q, dP


# --------------------------------------------------------------------------
# fast_mode: 2D ideal GRMHD linear wave, Minkowski 128^2 periodic
# --------------------------------------------------------------------------
def fast_mode_config(N=128, **kw):
    base = dict(N1=N, N2=N, N3=1, dim=2, conduction=0, viscosity=0,
                adiabaticIndex=4. / 3, reconstruction=C.MINMOD,
                riemannSolver=C.LOCAL_LAX_FRIEDRICH, CourantFactor=0.5,
                dt=0.5 / N, maxNonLinearIter=3, maxLineSearchIters=3,
                nonlinearsolve_atol=1e-20, JacobianAssembleEpsilon=4e-8,
                elemOldFromFullStep=1)
    base.update(kw)
    return C.make_config(**base)


def fast_mode_prims(cfg, seed=1, amplitude=1e-4):
    """Background rho=1, u=2, u^i=0, B=(0.1,0.3,0); each of rho,u,u1,u2,u3,B3
    gets amplitude*a_v*cos(2pi(x+y)+phi_v) with a_v~U[-1,1], phi_v~U[0,2pi)
    (numpy PCG64, ``seed``); dB1 = -dB2 keeps div B = 0 for k=(2pi,2pi)."""
    rng = np.random.default_rng(seed)
    X1, X2, _ = C.cell_centers(cfg)
    idx = C.var_index(cfg)
    P = _blank(cfg)
    bg = dict(RHO=1., U=2., U1=0., U2=0., U3=0., B1=0.1, B2=0.3, B3=0.)
    for k, v in bg.items():
        P[idx[k]] = v
    phase = 2 * math.pi * (X1 + X2)
    for name in ("RHO", "U", "U1", "U2", "U3", "B3", "B2"):
        a = rng.uniform(-1., 1.)
        phi = rng.uniform(0., 2 * math.pi)
        d = amplitude * a * np.cos(phase + phi)
        P[idx[name]] = P[idx[name]] + d
        if name == "B2":
            P[idx["B1"]] = P[idx["B1"]] - d
    return P


# --------------------------------------------------------------------------
# orszag_tang: orzag_tang/problem.cpp:3-34 (u^i = gamma v^i)
# --------------------------------------------------------------------------
def orszag_tang_config(N=512, **kw):
    base = dict(N1=N, N2=N, N3=1, dim=2, conduction=0, viscosity=0,
                adiabaticIndex=5. / 3, reconstruction=C.WENO5, riemannSolver=C.HLL,
                CourantFactor=0.5, dt=0.5 / N, elemOldFromFullStep=1,
                nonlinearsolve_atol=1e-20)
    base.update(kw)
    return C.make_config(**base)


def orszag_tang_prims(cfg):
    X1, X2, _ = C.cell_centers(cfg)
    idx = C.var_index(cfg)
    P = _blank(cfg)
    G = cfg["adiabaticIndex"]
    rho = 25. / (36. * math.pi) + 0. * X1
    p = 5. / (12. * math.pi) + 0. * X1
    v1 = -0.5 * np.sin(2 * math.pi * X2)
    v2 = 0.5 * np.sin(2 * math.pi * X1)
    gam = 1. / np.sqrt(1. - v1 * v1 - v2 * v2)
    B0 = 1. / math.sqrt(4. * math.pi)
    P[idx["RHO"]] = rho
    P[idx["U"]] = p / (G - 1.)
    P[idx["U1"]] = gam * v1
    P[idx["U2"]] = gam * v2
    P[idx["U3"]] = 0.
    P[idx["B1"]] = -B0 * np.sin(2 * math.pi * X2)
    P[idx["B2"]] = B0 * np.sin(4 * math.pi * X1)
    P[idx["B3"]] = 0.
    return P


# --------------------------------------------------------------------------
# emhd_stratified: 2D EMHD 256^2, rho ~ exp(-y/H), tau(y), MP5
# --------------------------------------------------------------------------
EMHD_T0 = 0.1       # temperature P/rho of the background (stated choice)
EMHD_B = 0.1        # |B| of the uniform field, at 30 degrees in the x-y plane


def emhd_stratified_config(N=256, **kw):
    base = dict(N1=N, N2=N, N3=1, dim=2, conduction=1, viscosity=1,
                highOrderTermsConduction=1, highOrderTermsViscosity=1,
                adiabaticIndex=4. / 3, reconstruction=C.MP5, riemannSolver=C.HLL,
                CourantFactor=0.5, dt=0.5 / N, closure=C.CLOSURE_TAU_PROFILE,
                closureTau0=0.1, closureTau1=1.0, elemOldFromFullStep=1,
                boundaryTop=C.OUTFLOW, boundaryBottom=C.OUTFLOW,
                nonlinearsolve_atol=1e-20)
    base.update(kw)
    return C.make_config(**base)


def emhd_stratified_prims(cfg, seed=3, H=0.5, amplitude=1e-3):
    rng = np.random.default_rng(seed)
    X1, X2, _ = C.cell_centers(cfg)
    idx = C.var_index(cfg)
    P = _blank(cfg)
    G = cfg["adiabaticIndex"]
    rho = np.exp(-X2 / H)
    u = rho * EMHD_T0 / (G - 1.)
    u = u * (1. + amplitude * rng.uniform(-0.5, 0.5, size=u.shape))
    P[idx["RHO"]] = rho
    P[idx["U"]] = u
    th = math.radians(30.)
    P[idx["B1"]] = EMHD_B * math.cos(th)
    P[idx["B2"]] = EMHD_B * math.sin(th)
    return P


# --------------------------------------------------------------------------
# ragged batch: independent 2D ideal linear-mode problems of different sizes
# --------------------------------------------------------------------------
LM_BACKGROUND_IDEAL = (1.0, 2.0, 0.0, 0.0, 0.0, 0.1, 0.3, 0.0)


def ragged_batch(seed=5, count=16, amplitude=1e-4, **kw):
    """[(config, prims)] of ``count`` problems: 2D ideal MHD, Minkowski,
    periodic unit squares, N = 16 U{4..32} (64 .. 512, seeded PCG64), a
    wave 2 pi (k1 x + k2 y) with k1, k2 in U{1..4} and ``amplitude`` (1e-4)
    in every primitive (random phase per variable) on the background
    rho = 1, u = 2, B = (0.1, 0.3, 0); minmod, LLF, flux-CT
    (fast_mode_config); ``kw`` sets further config fields (Newton
    tolerances, the scheme)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        n = int(rng.integers(4, 33)) * 16
        cfg = fast_mode_config(N=n, **kw)
        X1, X2, _ = C.cell_centers(cfg)
        k1, k2 = (int(x) for x in rng.integers(1, 5, 2))
        ph = rng.uniform(0, 2 * math.pi, 8)
        P = np.stack([LM_BACKGROUND_IDEAL[v] + amplitude * np.cos(2 * math.pi * (k1 * X1 + k2 * X2) + ph[v])
                      for v in range(8)])
        out.append((cfg, P))
    return out
