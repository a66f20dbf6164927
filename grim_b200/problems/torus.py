"""Fishbone-Moncrief torus in modified Kerr-Schild coordinates: config and
initial conditions (src/problem/torus/params.cpp:3-148,
src/problem/torus/problem.cpp:56-540).

The initial conditions are evaluated on the host in FP64 from the
geometry the caller passes (the stepper's own metric), once, before the
timed run.  The reference draws the 4% perturbation of u with PETSc's
RAND48 generator; here numpy's PCG64 with a seed stands in for it.
"""
import math

import numpy as np

from .. import config as C


def torus_config(N1=256, N2=128, N3=64, spin=0.9375, r_in=6., r_max=12., emhd=False, **kw):
    """cfg4: a=0.9375, r_in=6, r_max=12, 256x128x64, PPM, LLF, flux-CT."""
    Rin = 0.85 * (1. + math.sqrt(1. - spin * spin))
    Rout = 3000.
    base = dict(
        N1=N1, N2=N2, N3=N3, dim=3, metric=C.MODIFIED_KERR_SCHILD, blackHoleSpin=spin, hSlope=0.3,
        X1Start=math.log(Rin), X1End=math.log(Rout), X2Start=0. + 1.e-8, X2End=1. - 1.e-8,
        X3Start=0., X3End=2. * math.pi,
        DerefineThetaHorizon=1, DoCylindrify=1, X1cyl=math.log(4. * Rin), X2cyl=1. / N2,
        boundaryLeft=C.OUTFLOW, boundaryRight=C.OUTFLOW, boundaryTop=C.MIRROR, boundaryBottom=C.MIRROR,
        boundaryFront=C.PERIODIC, boundaryBack=C.PERIODIC,
        conduction=1 if emhd else 0, viscosity=1 if emhd else 0,
        highOrderTermsConduction=1, highOrderTermsViscosity=1,
        ConductionAlpha=1., ViscosityAlpha=1., ConductionClosureFactor=1., ViscosityClosureFactor=1.,
        adiabaticIndex=5. / 3, reconstruction=C.PPM, riemannSolver=C.LOCAL_LAX_FRIEDRICH,
        maxNonLinearIter=3, maxLineSearchIters=3, nonlinearsolve_atol=1.e-3,
        JacobianAssembleEpsilon=4.e-8, linesearchfloor=1.e-24,
        CourantFactor=0.9, maxDtIncrement=1.3, dt=0.005,
        closure=C.CLOSURE_TORUS, problem=C.PROBLEM_TORUS, elemOldFromFullStep=1,
        MaxLorentzFactor=10., RhoFloorAmpl=1.e-3, UFloorAmpl=1.e-5, RhoFloorSlope=-2.5,
        UFloorSlope=-2.5, BsqrOverRhoMax=10., BsqrOverUMax=500.,
    )
    base.update(kw)
    cfg = C.make_config(**base)
    cfg["_torus"] = dict(InnerEdgeRadius=r_in, PressureMaxRadius=r_max, MinPlasmaBeta=100.,
                         MagneticLoops=1., Adiabat=1.e-3, InitialPerturbationAmplitude=4.e-2)
    return cfg


# Fishbone & Moncrief (1976) helpers, torus/problem.cpp:56-143
def _delta(a, r):
    return r * r - 2 * r + a * a


def _sigma(a, r, th):
    return r * r + a * a * np.cos(th) * np.cos(th)


def _A(a, r, th):
    return (r * r + a * a) ** 2 - _delta(a, r) * a * a * np.sin(th) * np.sin(th)


def l_fm(a, r):
    return (math.sqrt(1. / r ** 3) * (r ** 4 + r * r * a * a - 2. * r * a * a - a * math.sqrt(r) * (r * r - a * a))
            / (r * r - 3 * r + 2. * a * math.sqrt(r)))


def _lnh_terms(a, r, th, l):
    D, S, A = _delta(a, r), _sigma(a, r, th), _A(a, r, th)
    t1 = 0.5 * np.log((1. + np.sqrt(1. + (4. * l * l * S * S * D) / (A * np.sin(th) * A * np.sin(th)))) / (S * D / A))
    t2 = -0.5 * np.sqrt(1. + (4. * l * l * S * S * D) / (A * A * np.sin(th) * np.sin(th)))
    t3 = -2 * a * r * l / A
    return t1 + t2 + t3


def ln_h(a, r, th, r_in, r_max):
    l = l_fm(a, r_max)
    return _lnh_terms(a, r, th, l) - _lnh_terms(a, r_in, math.pi / 2., l)


def torus_fluid(cfg, geo, seed=4):
    """rho, u, u^1..3 (before the field), problem.cpp:145-355.  ``geo`` is a
    dict with x (r, theta), alpha, gCon of the zone centres."""
    tp = cfg["_torus"]
    a = cfg["blackHoleSpin"]
    G = cfg["adiabaticIndex"]
    K = tp["Adiabat"]
    r = geo["x"][0]
    th = geo["x"][1]
    _, X2, _ = C.cell_centers(cfg)
    lapse = geo["alpha"]
    beta = [geo["gCon"][0][m] for m in (1, 2, 3)]
    rng = np.random.default_rng(seed)
    rand = rng.uniform(0., 1., size=r.shape)
    with np.errstate(all="ignore"):
        lnh = np.where(r >= tp["InnerEdgeRadius"], ln_h(a, r, th, tp["InnerEdgeRadius"], tp["PressureMaxRadius"]), 1.)
        inside = ~((lnh < 0.) | (r < tp["InnerEdgeRadius"]))
        h = np.exp(lnh)
        rho = np.where(inside, ((h - 1) * (G - 1.) / (K * G)) ** (1. / (G - 1.)), cfg["rhoFloorInFluidElement"])
        u = np.where(inside, K * rho ** G / (G - 1.) * (1. + tp["InitialPerturbationAmplitude"] * (rand - 0.5)),
                     cfg["uFloorInFluidElement"])
        # Boyer-Lindquist u_phi -> MKS u^i
        A, S, D = _A(a, r, th), _sigma(a, r, th), _delta(a, r)
        l = l_fm(a, tp["PressureMaxRadius"])
        e2chi = S * S * D / (A * A * np.sin(th) * np.sin(th))
        uphi_cov = np.sqrt((-1. + np.sqrt(1. + 4 * l * l * e2chi)) / 2.)
        uphi_con = 2. * a * r * np.sqrt(1. + uphi_cov * uphi_cov) / np.sqrt(A * S * D) + \
            np.sqrt(S / A) * uphi_cov / np.sin(th)
        mu = 1 + a * a * np.cos(th) * np.cos(th) / (r * r)
        g00 = -(1. - 2. / (r * mu))
        g03 = -2. * a * np.sin(th) * np.sin(th) / (r * mu)
        g33 = r * r * np.sin(th) * np.sin(th) * (1. + a * a / (r * r) + 2. * a * a * np.sin(th) * np.sin(th) / (r * r * r * mu))
        AA = g00
        BB = 2. * (g03 * uphi_con)
        CC = 1. + g33 * uphi_con * uphi_con
        u0 = -(BB + np.sqrt(BB * BB - 4. * AA * CC)) / (2. * AA)
        uKS = [u0 + 2. * r / D * 0., 0., 0., uphi_con]
        # transformBLToMKS: uKS^0 = u0 + 2r/D u^1_BL (= 0), uKS^3 = u3 + a/D u^1_BL (= 0)
        uKS = [u0, 0. * r, 0. * r, uphi_con]
        hfac = math.pi + (1. - cfg["hSlope"]) * math.pi * np.cos(2. * math.pi * X2)
        uMKS = [uKS[0], uKS[1] / r, uKS[2] / hfac, uKS[3]]
        U = [uMKS[m + 1] + lapse ** 2 * beta[m] * uMKS[0] for m in range(3)]
    U = [np.where(inside, U[m], 0.) for m in range(3)]
    return rho, u, U


def torus_prims(cfg, geo, seed=4):
    """Primitives after the field set-up and beta normalisation, before the
    floors (problem.cpp:145-525).  ``geo`` (centre) needs x, alpha, g, gCon,
    gCov.  The floors and the first fullStepDiagnostics run on the GPU."""
    idx = C.var_index(cfg)
    dof, nf = C.var_counts(cfg)
    rho, u, U = torus_fluid(cfg, geo, seed)
    # ArrayFire's max/min reductions skip NaN (the cylindrified map is
    # undefined in some inner ghost zones)
    rhoMax = np.nanmax(rho)
    rho = rho / rhoMax
    u = u / rhoMax
    # vector potential from the density averaged over the 4 (6) neighbours
    sh = lambda a, s1, s2, s3: np.roll(a, shift=(s3, s2, s1), axis=(0, 1, 2))  # af::shift
    ravg = sh(rho, 1, 0, 0) + sh(rho, -1, 0, 0) + sh(rho, 0, 1, 0) + sh(rho, 0, -1, 0)
    if cfg["dim"] > 2:
        ravg = (ravg + sh(rho, 0, 0, 1) + sh(rho, 0, 0, -1)) / 6.
    else:
        ravg = ravg / 4.
    tp = cfg["_torus"]
    Avec = np.maximum(ravg - 0.2, 0.) * np.cos(geo["x"][1] * (tp["MagneticLoops"] - 1))
    g = geo["g"]
    dX1 = (cfg["X1End"] - cfg["X1Start"]) / cfg["N1"]
    dX2 = (cfg["X2End"] - cfg["X2Start"]) / cfg["N2"]
    B1 = (sh(Avec, 0, -1, 0) - Avec + sh(Avec, -1, -1, 0) - sh(Avec, -1, 0, 0)) / (2. * dX2 * g)
    B2 = (Avec - sh(Avec, -1, 0, 0) + sh(Avec, 0, -1, 0) - sh(Avec, -1, -1, 0)) / (2. * dX1 * g)
    mask = np.zeros_like(rho)
    mask[C.interior_slices(cfg)] = 1.
    B1 = B1 * mask
    B2 = B2 * mask
    P = np.zeros((dof,) + rho.shape)
    P[idx["RHO"]], P[idx["U"]] = rho, u
    P[idx["U1"]], P[idx["U2"]], P[idx["U3"]] = U
    P[idx["B1"]], P[idx["B2"]] = B1, B2
    P = communicate(cfg, P)
    # beta normalisation (SANE): min over the grid of 2(P+1e-13)/(b^2+1e-18)
    bsq, pg = b2_and_pressure(cfg, P, geo)
    beta = 2. * (pg + 1.e-13) / (bsq + 1.e-18)
    BFactor = math.sqrt(np.nanmin(beta) / tp["MinPlasmaBeta"])
    for v in ("B1", "B2", "B3"):
        P[idx[v]] = P[idx[v]] * BFactor
    return P, dict(rhoMax=float(rhoMax), BFactor=BFactor)


def communicate(cfg, P):
    """grid::communicate semantics: periodic wrap, other ghosts zero."""
    Q = P.copy()
    g = cfg["numGhost"]
    dims = [(cfg["N1"], cfg["boundaryLeft"] == C.PERIODIC, 3), (cfg["N2"], cfg["boundaryBottom"] == C.PERIODIC, 2),
            (cfg["N3"], cfg["boundaryBack"] == C.PERIODIC, 1)]
    n3, n2, n1 = P.shape[1:]
    idxs = []
    zero = np.zeros(P.shape[1:], dtype=bool)
    for d, (N, per, axis) in enumerate(dims):
        if d >= cfg["dim"]:
            idxs.append(np.arange(P.shape[axis]))
            continue
        x = np.arange(N + 2 * g)
        inner = (x >= g) & (x < N + g)
        src = np.where(inner, x, g + (x - g) % N) if per else x
        idxs.append(src)
        if not per:
            bad = ~inner
            shape = [1, 1, 1]
            shape[axis - 1] = -1
            zero |= bad.reshape(shape)
    i1, i2, i3 = idxs
    Q = P[:, i3][:, :, i2][:, :, :, i1]
    Q[:, zero] = 0.
    return Q


def b2_and_pressure(cfg, P, geo):
    """b^2 and gas pressure of the fluid element (physics.cpp:53-116)."""
    idx = C.var_index(cfg)
    G = cfg["adiabaticIndex"]
    gcov, gcon, alpha = geo["gCov"], geo["gCon"], geo["alpha"]
    rho = np.maximum(P[idx["RHO"]], cfg["rhoFloorInFluidElement"])
    u = np.maximum(P[idx["U"]], cfg["uFloorInFluidElement"])
    v = [P[idx["U1"]], P[idx["U2"]], P[idx["U3"]]]
    B = [P[idx["B1"]], P[idx["B2"]], P[idx["B3"]]]
    gam = np.sqrt(1 + gcov[1][1] * v[0] * v[0] + gcov[2][2] * v[1] * v[1] + gcov[3][3] * v[2] * v[2]
                  + 2 * (gcov[1][2] * v[0] * v[1] + gcov[1][3] * v[0] * v[2] + gcov[2][3] * v[1] * v[2]))
    ucon = [gam / alpha] + [v[m] - gam * gcon[0][m + 1] * alpha for m in range(3)]
    ucov = [sum(gcov[mu][n] * ucon[n] for n in range(4)) for mu in range(4)]
    bcon0 = B[0] * ucov[1] + B[1] * ucov[2] + B[2] * ucov[3]
    bcon = [bcon0] + [(B[m] + bcon0 * ucon[m + 1]) / ucon[0] for m in range(3)]
    bcov = [sum(gcov[mu][n] * bcon[n] for n in range(4)) for mu in range(4)]
    bsq = sum(bcon[m] * bcov[m] for m in range(4)) + cfg["bSqrFloorInFluidElement"]
    return bsq, (G - 1.) * u
