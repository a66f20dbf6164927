"""Run-time configuration of the implicit timestep.

The reference configures its timestep through compile-time globals
(``params::`` and ``vars::`` in src/params.hpp:8-210, filled per problem in
src/problem/<name>/params.cpp).  Here the same fields travel in one POD
struct, ``grim_config`` (include/grim_b200.h), with the reference's field
names.  This module holds the field list, the enum values and the defaults
(the values of src/problem/linear_modes/params.cpp:4-81).
"""
import ctypes
import math

# enums, src/params.hpp:32-94 (MP5 and the closures are additions)
PERIODIC, OUTFLOW, MIRROR, DIRICHLET, EXCHANGE = 0, 1, 2, 3, 4
MINKOWSKI, MODIFIED_KERR_SCHILD = 0, 1
MINMOD, WENO5, PPM, MP5 = 0, 1, 2, 3
HLL, LOCAL_LAX_FRIEDRICH = 0, 1
CENTER, LEFT, RIGHT, TOP, BOTTOM = 0, 1, 2, 3, 4
HALF_STEP, FULL_STEP = 0, 1

# setFluidElementParameters variants (problem hook)
CLOSURE_CONST_TAU = 0      # linear_modes/problem.cpp:3-8  (tau = closureTau0)
CLOSURE_TORUS = 1          # torus/problem.cpp:7-55
CLOSURE_TAU_PROFILE = 2    # tau linear in the physical X2 coordinate

# problem hooks (BCs, flux filter, diagnostics)
PROBLEM_NONE = 0
PROBLEM_TORUS = 1

# Newton variants
NEWTON_PARITY_FD64 = 0     # the reference's method (solve.cpp:3-230)
NEWTON_TANGENT64 = 1       # exact forward-tangent Jacobian, FP64 solve
NEWTON_MIXED32 = 2         # FP32 tangent Jacobian + FP32 solve, FP64 residual
NEWTON_FD64_FAST = 3       # the reference's FD Newton in the fast path's arithmetic and kernels

INT_FIELDS = [
    "N1", "N2", "N3", "dim", "numGhost",
    "boundaryLeft", "boundaryRight", "boundaryTop", "boundaryBottom",
    "boundaryFront", "boundaryBack",
    "metric",
    "DerefineThetaHorizon", "DoCylindrify",
    "conduction", "viscosity",
    "highOrderTermsConduction", "highOrderTermsViscosity",
    "reconstruction", "riemannSolver",
    "maxNonLinearIter", "maxLineSearchIters",
    "closure", "problem", "elemOldFromFullStep",
    "newtonMode", "perZoneConvergence", "N3Global",
]
N_RESERVED_INT = 4

DOUBLE_FIELDS = [
    "blackHoleSpin", "hSlope",
    "X1Start", "X1End", "X2Start", "X2End", "X3Start", "X3End",
    "time", "dt",
    "X1cyl", "X2cyl",
    "rhoFloorInFluidElement", "uFloorInFluidElement",
    "bSqrFloorInFluidElement", "temperatureFloorInFluidElement",
    "adiabaticIndex", "ConductionAlpha", "ViscosityAlpha",
    "ConductionClosureFactor", "ViscosityClosureFactor",
    "slopeLimTheta",
    "nonlinearsolve_atol", "nonlinearsolve_rtol",
    "JacobianAssembleEpsilon", "linesearchfloor",
    "CourantFactor", "maxDtIncrement",
    "closureTau0", "closureTau1",
    "MaxLorentzFactor", "RhoFloorAmpl", "UFloorAmpl", "RhoFloorSlope",
    "UFloorSlope", "BsqrOverRhoMax", "BsqrOverUMax",
    "ObserveEveryDt",
    "nonlinearsolve_ulps",
]
N_RESERVED_DOUBLE = 4


def _struct_fields():
    f = [(n, ctypes.c_int) for n in INT_FIELDS]
    f.append(("reserved_i", ctypes.c_int * N_RESERVED_INT))
    f += [(n, ctypes.c_double) for n in DOUBLE_FIELDS]
    f.append(("reserved_d", ctypes.c_double * N_RESERVED_DOUBLE))
    return f


class GrimConfig(ctypes.Structure):
    """ctypes mirror of ``grim_config`` in include/grim_b200.h."""
    _fields_ = _struct_fields()


def defaults():
    """Defaults = src/problem/linear_modes/params.cpp:4-81, ideal MHD."""
    return dict(
        N1=128, N2=128, N3=1, dim=2, numGhost=3,
        boundaryLeft=PERIODIC, boundaryRight=PERIODIC,
        boundaryTop=PERIODIC, boundaryBottom=PERIODIC,
        boundaryFront=PERIODIC, boundaryBack=PERIODIC,
        metric=MINKOWSKI,
        DerefineThetaHorizon=1, DoCylindrify=1,
        conduction=0, viscosity=0,
        highOrderTermsConduction=1, highOrderTermsViscosity=1,
        reconstruction=MINMOD, riemannSolver=HLL,
        maxNonLinearIter=3, maxLineSearchIters=3,
        closure=CLOSURE_CONST_TAU, problem=PROBLEM_NONE, elemOldFromFullStep=1,
        newtonMode=NEWTON_PARITY_FD64, perZoneConvergence=0, N3Global=0,
        blackHoleSpin=0.9375, hSlope=0.3,
        X1Start=0., X1End=1., X2Start=0., X2End=1., X3Start=0., X3End=1.,
        time=0., dt=0.5 / 128,
        X1cyl=0., X2cyl=1. / 128,
        rhoFloorInFluidElement=1e-20, uFloorInFluidElement=1e-20,
        bSqrFloorInFluidElement=1e-20, temperatureFloorInFluidElement=1e-20,
        adiabaticIndex=4. / 3, ConductionAlpha=1., ViscosityAlpha=1.,
        ConductionClosureFactor=1., ViscosityClosureFactor=1.,
        slopeLimTheta=2.,
        nonlinearsolve_atol=1e-20, nonlinearsolve_rtol=0.,
        JacobianAssembleEpsilon=4e-8, linesearchfloor=1e-24,
        CourantFactor=0.9, maxDtIncrement=1.3,
        closureTau0=1., closureTau1=1.,
        MaxLorentzFactor=10., RhoFloorAmpl=1e-3, UFloorAmpl=1e-5,
        RhoFloorSlope=-2.5, UFloorSlope=-2.5,
        BsqrOverRhoMax=10., BsqrOverUMax=500.,
        ObserveEveryDt=0., nonlinearsolve_ulps=0.,
    )


def make_config(**overrides):
    """Defaults updated with ``overrides``; unknown keys raise KeyError."""
    cfg = defaults()
    for k, v in overrides.items():
        if k not in cfg:
            raise KeyError("unknown grim_config field: %s" % k)
        cfg[k] = v
    if cfg["dim"] < 3:
        cfg["N3"] = 1
    if cfg["dim"] < 2:
        cfg["N2"] = 1
    return cfg


def to_struct(cfg, cls=GrimConfig):
    s = cls()
    for n in INT_FIELDS:
        setattr(s, n, int(cfg[n]))
    for n in DOUBLE_FIELDS:
        setattr(s, n, float(cfg[n]))
    return s


def var_counts(cfg):
    """(dof, numFluidVars), linear_modes/params.cpp:83-93."""
    nf = 5 + int(cfg["conduction"]) + int(cfg["viscosity"])
    return nf + 3, nf


def var_index(cfg):
    """Variable indices (vars:: namespace)."""
    dof, nf = var_counts(cfg)
    idx = dict(RHO=0, U=1, U1=2, U2=3, U3=4, B1=nf, B2=nf + 1, B3=nf + 2)
    if cfg["conduction"]:
        idx["Q"] = 5
    if cfg["viscosity"]:
        idx["DP"] = 5 + int(cfg["conduction"])
    return idx


def total_dims(cfg):
    """(N1Total, N2Total, N3Total) with numGhost ghosts per active dimension."""
    g = int(cfg["numGhost"])
    d = int(cfg["dim"])
    n1 = int(cfg["N1"]) + 2 * g
    n2 = int(cfg["N2"]) + (2 * g if d >= 2 else 0)
    n3 = int(cfg["N3"]) + (2 * g if d >= 3 else 0)
    return n1, n2, n3


def cell_centers(cfg):
    """X coordinates of zone centres incl. ghosts, grid.cpp:168-249 (CENTER)."""
    import numpy as np
    g = int(cfg["numGhost"])
    d = int(cfg["dim"])
    n1, n2, n3 = total_dims(cfg)
    dX1 = (cfg["X1End"] - cfg["X1Start"]) / cfg["N1"]
    dX2 = (cfg["X2End"] - cfg["X2Start"]) / cfg["N2"]
    dX3 = (cfg["X3End"] - cfg["X3Start"]) / cfg["N3"]
    i = np.arange(n1) - g
    j = np.arange(n2) - (g if d >= 2 else 0)
    k = np.arange(n3) - (g if d >= 3 else 0)
    X1 = cfg["X1Start"] + (i + 0.5) * dX1
    X2 = cfg["X2Start"] + (j + 0.5) * dX2
    X3 = cfg["X3Start"] + (k + 0.5) * dX3
    K, J, I = np.meshgrid(X3, X2, X1, indexing="ij")
    return I, J, K


def interior_slices(cfg):
    g = int(cfg["numGhost"])
    d = int(cfg["dim"])
    s1 = slice(g, g + int(cfg["N1"]))
    s2 = slice(g, g + int(cfg["N2"])) if d >= 2 else slice(None)
    s3 = slice(g, g + int(cfg["N3"])) if d >= 3 else slice(None)
    return (s3, s2, s1)


__all__ = [n for n in dir() if not n.startswith("_")] + ["math"]
