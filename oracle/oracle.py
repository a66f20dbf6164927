"""ctypes wrapper of the CPU oracle (liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, by bench.py's cpu_baseline /
reference leg and by __graft_entry__.smoke() as the checker.  The oracle is
a C++ restatement of the reference's timestep (see grim_oracle.cpp); the
product never calls it.

Configs are plain dicts with the grim_config field names (the product's
grim_b200.config.make_config builds them); this module declares its own copy
of the struct so it depends on nothing in the product package.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

INT_FIELDS = [
    "N1", "N2", "N3", "dim", "numGhost",
    "boundaryLeft", "boundaryRight", "boundaryTop", "boundaryBottom",
    "boundaryFront", "boundaryBack", "metric",
    "DerefineThetaHorizon", "DoCylindrify", "conduction", "viscosity",
    "highOrderTermsConduction", "highOrderTermsViscosity",
    "reconstruction", "riemannSolver", "maxNonLinearIter", "maxLineSearchIters",
    "closure", "problem", "elemOldFromFullStep", "newtonMode", "perZoneConvergence", "N3Global",
]
DOUBLE_FIELDS = [
    "blackHoleSpin", "hSlope", "X1Start", "X1End", "X2Start", "X2End",
    "X3Start", "X3End", "time", "dt", "X1cyl", "X2cyl",
    "rhoFloorInFluidElement", "uFloorInFluidElement",
    "bSqrFloorInFluidElement", "temperatureFloorInFluidElement",
    "adiabaticIndex", "ConductionAlpha", "ViscosityAlpha",
    "ConductionClosureFactor", "ViscosityClosureFactor", "slopeLimTheta",
    "nonlinearsolve_atol", "nonlinearsolve_rtol", "JacobianAssembleEpsilon",
    "linesearchfloor", "CourantFactor", "maxDtIncrement",
    "closureTau0", "closureTau1", "MaxLorentzFactor", "RhoFloorAmpl",
    "UFloorAmpl", "RhoFloorSlope", "UFloorSlope", "BsqrOverRhoMax", "BsqrOverUMax", "ObserveEveryDt",
    "nonlinearsolve_ulps",
]


class OrcConfig(ctypes.Structure):
    _fields_ = ([(n, ctypes.c_int) for n in INT_FIELDS] + [("reserved_i", ctypes.c_int * 4)]
                + [(n, ctypes.c_double) for n in DOUBLE_FIELDS]
                + [("reserved_d", ctypes.c_double * 4)])


PRIM_OLD, PRIM, PRIM_HALF = 0, 1, 2


def build():
    """Compile liboracle.so in place (make)."""
    subprocess.check_call(["make", "-s", "-C", _HERE, "liboracle.so"])


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        P = ctypes.POINTER
        d = ctypes.c_double
        i = ctypes.c_int
        vp = ctypes.c_void_p
        L.orc_create.argtypes = [P(OrcConfig), P(vp)]
        L.orc_destroy.argtypes = [vp]
        L.orc_destroy.restype = None
        L.orc_num_vars.argtypes = [vp, P(i), P(i)]
        L.orc_dims.argtypes = [vp, P(i), P(i), P(i)]
        L.orc_set_prims.argtypes = [vp, i, P(d)]
        L.orc_get_prims.argtypes = [vp, i, P(d)]
        L.orc_time_step.argtypes = [vp, i]
        L.orc_get_time.argtypes = [vp, P(d), P(d)]
        L.orc_set_time.argtypes = [vp, d, d]
        L.orc_compute_dt.argtypes = [vp]
        L.orc_apply_boundaries.argtypes = [vp, P(d), i]
        L.orc_geometry.argtypes = [vp, i, P(d), P(d), P(d)]
        L.orc_div_fluxes.argtypes = [vp, P(d), P(d), P(d), P(d)]
        L.orc_reconstruct.argtypes = [vp, P(d), i, P(d), P(d)]
        L.orc_conserved.argtypes = [vp, P(d), P(d)]
        L.orc_element_fluxes.argtypes = [vp, P(d), ctypes.c_int, P(d)]
        L.orc_get_stage_grid.argtypes = [vp, ctypes.c_int, P(d)]
        L.orc_compute_divb.argtypes = [vp, P(d), P(d)]
        L.orc_torus_observers.argtypes = [vp, P(d)]
        L.orc_char_speeds.argtypes = [vp, P(d), i, P(d), P(d)]
        L.orc_stage_setup.argtypes = [vp, i]
        L.orc_residual.argtypes = [vp, P(d), P(d)]
        L.orc_jacobian_fd.argtypes = [vp, P(d), P(d)]
        L.orc_newton.argtypes = [vp, P(i)]
        L.orc_batch_solve.argtypes = [i, i, P(d), P(d), P(d)]
        L.orc_last_newton_stats.argtypes = [vp, P(i), P(i)]
        L.orc_set_threads.argtypes = [i]
        L.orc_problem_init.argtypes = [vp]
        _LIB = L
    return _LIB


def _ptr(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def set_threads(n):
    lib().orc_set_threads(int(n))


def batch_solve(A, b):
    """x with A[z] x[z] = b[z] by the oracle's pivoted elimination."""
    A = np.ascontiguousarray(A, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    n = A.shape[-1]
    batch = A.shape[0]
    x = np.zeros((batch, n))
    rc = lib().orc_batch_solve(n, batch, _ptr(A), _ptr(b), _ptr(x))
    assert rc == 0
    return x


class Oracle:
    """One oracle timeStepper (the reference's timeStepper, on the CPU)."""

    def __init__(self, cfg):
        s = OrcConfig()
        for n in INT_FIELDS:
            setattr(s, n, int(cfg[n]))
        for n in DOUBLE_FIELDS:
            setattr(s, n, float(cfg[n]))
        self.cfg = dict(cfg)
        self._h = ctypes.c_void_p()
        rc = lib().orc_create(ctypes.byref(s), ctypes.byref(self._h))
        if rc != 0:
            raise RuntimeError("orc_create failed: %d" % rc)
        dof, nf = ctypes.c_int(), ctypes.c_int()
        lib().orc_num_vars(self._h, ctypes.byref(dof), ctypes.byref(nf))
        self.dof, self.nf = dof.value, nf.value
        a, b, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        lib().orc_dims(self._h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c))
        self.N1T, self.N2T, self.N3T = a.value, b.value, c.value
        self.shape = (self.dof, self.N3T, self.N2T, self.N1T)
        self.zshape = (self.N3T, self.N2T, self.N1T)

    def close(self):
        if self._h:
            lib().orc_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _arr(self, nv=None):
        nv = self.dof if nv is None else nv
        return np.zeros((nv,) + self.zshape)

    def set_prims(self, prim, which=PRIM_OLD):
        p = np.ascontiguousarray(prim, dtype=np.float64).reshape(self.shape)
        assert lib().orc_set_prims(self._h, which, _ptr(p)) == 0

    def get_prims(self, which=PRIM_OLD):
        out = self._arr()
        assert lib().orc_get_prims(self._h, which, _ptr(out)) == 0
        return out

    def time_step(self, n=1):
        assert lib().orc_time_step(self._h, int(n)) == 0

    @property
    def time(self):
        t, dt = ctypes.c_double(), ctypes.c_double()
        lib().orc_get_time(self._h, ctypes.byref(t), ctypes.byref(dt))
        return t.value

    @property
    def dt(self):
        t, dt = ctypes.c_double(), ctypes.c_double()
        lib().orc_get_time(self._h, ctypes.byref(t), ctypes.byref(dt))
        return dt.value

    def set_time(self, t, dt):
        lib().orc_set_time(self._h, float(t), float(dt))

    def compute_dt(self):
        lib().orc_compute_dt(self._h)
        return self.dt

    def apply_boundaries(self, prim):
        p = np.array(prim, dtype=np.float64, order="C")
        nv = p.shape[0]
        lib().orc_apply_boundaries(self._h, _ptr(p), nv)
        return p

    def geometry(self, location):
        Z = self.N1T * self.N2T * self.N3T
        out = np.zeros((34,) + self.zshape)
        gam = np.zeros((64,) + self.zshape)
        xc = np.zeros((5,) + self.zshape)
        lib().orc_geometry(self._h, int(location), _ptr(out), _ptr(gam), _ptr(xc))
        return dict(gCov=out[:16].reshape((4, 4) + self.zshape),
                    gCon=out[16:32].reshape((4, 4) + self.zshape),
                    g=out[32], alpha=out[33],
                    gamma=gam.reshape((4, 4, 4) + self.zshape), x=xc)

    def div_fluxes(self, prim):
        p = np.ascontiguousarray(prim, dtype=np.float64)
        divF = self._arr()
        fl = np.zeros((3, self.dof) + self.zshape)
        emf = np.zeros((3,) + self.zshape)
        lib().orc_div_fluxes(self._h, _ptr(p), _ptr(divF), _ptr(fl), _ptr(emf))
        return divF, fl, emf

    def reconstruct(self, prim, direction):
        p = np.ascontiguousarray(prim, dtype=np.float64)
        pl, pr = self._arr(), self._arr()
        lib().orc_reconstruct(self._h, _ptr(p), int(direction), _ptr(pl), _ptr(pr))
        return pl, pr

    def conserved(self, prim):
        p = np.ascontiguousarray(prim, dtype=np.float64)
        c = self._arr()
        lib().orc_conserved(self._h, _ptr(p), _ptr(c))
        return c

    def element_fluxes(self, prim, direction):
        """fluidElement::computeFluxes(direction) at the zone centres
        (physics.cpp:185-217); direction 0 gives the conserved variables."""
        p = np.ascontiguousarray(prim, dtype=np.float64)
        out = self._arr()
        assert lib().orc_element_fluxes(self._h, _ptr(p), int(direction), _ptr(out)) == 0
        return out

    def stage_grid(self, which):
        """consOld (0, dof rows), divFluxes (1) or sourcesExplicit (2, the
        fluid rows) as the last stage_setup left them."""
        out = self._arr(self.dof if which == 0 else self.nf)
        assert lib().orc_get_stage_grid(self._h, int(which), _ptr(out)) == 0
        return out

    def compute_divb(self, prim):
        p = np.ascontiguousarray(prim, dtype=np.float64)
        out = np.zeros(self.zshape)
        lib().orc_compute_divb(self._h, _ptr(p), _ptr(out))
        return out

    OBSERVERS = ("BaryonMass", "EMag", "ETh", "rhoMax", "betaMin", "MdotIn", "MdotOut",
                 "UnboundMdotOut", "RelativisticUnboundMdotOut")

    def torus_observers(self):
        """ObserversTorus.hpp on primOld: {name: value}."""
        out = np.zeros(9)
        lib().orc_torus_observers(self._h, _ptr(out))
        return dict(zip(self.OBSERVERS, out.tolist()))

    def char_speeds(self, prim, direction):
        p = np.ascontiguousarray(prim, dtype=np.float64)
        mn = np.zeros(self.zshape)
        mx = np.zeros(self.zshape)
        lib().orc_char_speeds(self._h, _ptr(p), int(direction), _ptr(mn), _ptr(mx))
        return mn, mx

    def stage_setup(self, stage):
        lib().orc_stage_setup(self._h, int(stage))

    def residual(self, prim_guess):
        p = np.ascontiguousarray(prim_guess, dtype=np.float64)
        r = self._arr(self.nf)
        lib().orc_residual(self._h, _ptr(p), _ptr(r))
        return r

    def jacobian_fd(self, prim_guess):
        p = np.ascontiguousarray(prim_guess, dtype=np.float64)
        Z = self.N1T * self.N2T * self.N3T
        J = np.zeros((Z, self.nf, self.nf))
        lib().orc_jacobian_fd(self._h, _ptr(p), _ptr(J))
        return J.reshape(self.zshape + (self.nf, self.nf))

    def problem_init(self):
        lib().orc_problem_init(self._h)

    def newton(self):
        it = ctypes.c_int()
        lib().orc_newton(self._h, ctypes.byref(it))
        return it.value

    def last_newton_iters(self):
        a, b = ctypes.c_int(), ctypes.c_int()
        lib().orc_last_newton_stats(self._h, ctypes.byref(a), ctypes.byref(b))
        return a.value, b.value
