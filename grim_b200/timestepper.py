"""Python mirror of the reference's timeStepperPy / gridPy interface
(src/timestepper/timeStepperPy.pyx:20-212, src/grid/gridPy.pyx:185-221),
implemented over the C ABI of libgrim_b200.so.

    ts = timeStepper(cfg)              # or timeStepper.fromArgs(N1, N2, ...)
    ts.primOld.setVars(P)              # numpy [var, k, j, i], ghosts included
    ts.timeStep()                      # -> (numReads, numWrites)
    P = ts.primOld.getVars()

Grids live on the GPU; getVars/setVars copy through host memory exactly as
gridPy does (device -> host in getVars).  Device pointers (e.g. from torch)
can be passed with ``setVarsDevice`` / ``getVarsDevice``.
"""
import ctypes

import numpy as np

from . import _lib
from . import config as C


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data)


class Grid:
    """One state grid of the stepper (gridPy)."""

    def __init__(self, ts, which):
        self._ts = ts
        self._which = which

    @property
    def shape(self):
        return [self._ts.dof, self._ts.N3Total, self._ts.N2Total, self._ts.N1Total]

    numVars = property(lambda self: self._ts.dof)
    N1Total = property(lambda self: self._ts.N1Total)
    N2Total = property(lambda self: self._ts.N2Total)
    N3Total = property(lambda self: self._ts.N3Total)
    numGhost = property(lambda self: self._ts.cfg["numGhost"])
    dim = property(lambda self: self._ts.cfg["dim"])

    def getVars(self):
        out = np.empty(self.shape, dtype=np.float64)
        _lib.check(_lib.lib().grim_get_prims(self._ts._h, self._which, _ptr(out), _lib.HOST), "getVars")
        return out

    def setVars(self, vars_):
        a = np.ascontiguousarray(vars_, dtype=np.float64)
        if list(a.shape) != self.shape:
            raise ValueError("setVars: shape %s, expected %s" % (a.shape, self.shape))
        _lib.check(_lib.lib().grim_set_prims(self._ts._h, self._which, _ptr(a), _lib.HOST), "setVars")

    def communicate(self):
        """grid::communicate + boundaries: periodic wrap, then the physical
        boundary fill."""
        _lib.check(_lib.lib().grim_apply_boundaries(self._ts._h, self._which), "communicate")

    def setVarsDevice(self, dev_ptr):
        _lib.check(_lib.lib().grim_set_prims(self._ts._h, self._which, ctypes.c_void_p(int(dev_ptr)),
                                             _lib.DEVICE), "setVarsDevice")

    def getVarsDevice(self, dev_ptr):
        _lib.check(_lib.lib().grim_get_prims(self._ts._h, self._which, ctypes.c_void_p(int(dev_ptr)),
                                             _lib.DEVICE), "getVarsDevice")


class timeStepper:
    """The reference's timeStepper (timestepper.hpp:19-132) on one B200."""

    HALF_STEP, FULL_STEP = C.HALF_STEP, C.FULL_STEP

    def __init__(self, cfg, device=0, _handle=None):
        self.cfg = dict(cfg)
        L = _lib.lib()
        if _handle is None:
            s = C.to_struct(self.cfg)
            self._h = ctypes.c_void_p()
            _lib.check(L.grim_create(ctypes.byref(s), int(device), ctypes.byref(self._h)), "grim_create")
            self._owned = True
        else:  # a problem of a Batch: the batch owns the handle
            self._h = ctypes.c_void_p(_handle)
            self._owned = False
        a, b, c, dof, nf = (ctypes.c_int() for _ in range(5))
        L.grim_dims(self._h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c), ctypes.byref(dof),
                    ctypes.byref(nf))
        self.N1Total, self.N2Total, self.N3Total = a.value, b.value, c.value
        self.dof, self.numFluidVars = dof.value, nf.value
        self.zshape = (self.N3Total, self.N2Total, self.N1Total)
        self.prim = Grid(self, _lib.PRIM)
        self.primOld = Grid(self, _lib.PRIM_OLD)
        self.primHalfStep = Grid(self, _lib.PRIM_HALF)

    @classmethod
    def fromArgs(cls, N1, N2, N3, dim, numVars, numGhost, time, dt, boundaryLeft, boundaryRight,
                 boundaryTop, boundaryBottom, boundaryFront, boundaryBack, metric, blackHoleSpin, hSlope,
                 X1Start, X1End, X2Start, X2End, X3Start, X3End, **params):
        """The reference constructor's argument list (timeStepperPy.pyx:22-50);
        the remaining params:: values come as keywords."""
        cfg = C.make_config(N1=N1, N2=N2, N3=N3, dim=dim, numGhost=numGhost, time=time, dt=dt,
                            boundaryLeft=boundaryLeft, boundaryRight=boundaryRight,
                            boundaryTop=boundaryTop, boundaryBottom=boundaryBottom,
                            boundaryFront=boundaryFront, boundaryBack=boundaryBack, metric=metric,
                            blackHoleSpin=blackHoleSpin, hSlope=hSlope, X1Start=X1Start, X1End=X1End,
                            X2Start=X2Start, X2End=X2End, X3Start=X3Start, X3End=X3End, **params)
        if C.var_counts(cfg)[0] != numVars:
            raise ValueError("numVars %d does not match the EMHD switches" % numVars)
        return cls(cfg)

    def close(self):
        if getattr(self, "_h", None) and self._h.value and getattr(self, "_owned", True):
            _lib.lib().grim_destroy(self._h)
        self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def problemInit(self):
        """The problem's tail of initialConditions (torus: floors + the first
        fullStepDiagnostics); call after primOld.setVars."""
        _lib.check(_lib.lib().grim_problem_init(self._h), "problem_init")

    # ---- stepping ----------------------------------------------------------
    def timeStep(self):
        r, w = ctypes.c_int(), ctypes.c_int()
        _lib.check(_lib.lib().grim_time_step(self._h, ctypes.byref(r), ctypes.byref(w)), "timeStep")
        return r.value, w.value

    def timeSteps(self, n):
        _lib.check(_lib.lib().grim_time_steps(self._h, int(n)), "timeSteps")

    def timeStepsHost(self, inputs, outputs, interior=False):
        """grim_time_steps_host: per step, primOld from inputs[k] (a host
        address, or None to continue from the current state), one
        timeStep, primOld to outputs[k] (a host address or None); the
        copies overlap the other steps' work when the buffers are pinned.
        Addresses are ints (numpy ``a.ctypes.data``, torch
        ``t.data_ptr()``) of float64 [var][k][j][i] arrays with ghosts, or
        of the interior zones only with ``interior``."""
        n = len(inputs)
        if len(outputs) != n:
            raise ValueError("inputs and outputs differ in length")
        ins = (ctypes.c_void_p * n)(*[None if a is None else int(a) for a in inputs])
        outs = (ctypes.c_void_p * n)(*[None if a is None else int(a) for a in outputs])
        layout = _lib.LAYOUT_INTERIOR if interior else _lib.LAYOUT_GHOSTED
        _lib.check(_lib.lib().grim_time_steps_host(self._h, n, ins, outs, layout), "timeStepsHost")

    @property
    def time(self):
        t, dt = ctypes.c_double(), ctypes.c_double()
        _lib.check(_lib.lib().grim_get_time(self._h, ctypes.byref(t), ctypes.byref(dt)), "get_time")
        return t.value

    @property
    def dt(self):
        t, dt = ctypes.c_double(), ctypes.c_double()
        _lib.check(_lib.lib().grim_get_time(self._h, ctypes.byref(t), ctypes.byref(dt)), "get_time")
        return dt.value

    def setTime(self, time, dt):
        _lib.check(_lib.lib().grim_set_time(self._h, float(time), float(dt)), "set_time")

    def computeDt(self):
        _lib.check(_lib.lib().grim_compute_dt(self._h), "computeDt")
        return self.dt

    def synchronize(self):
        _lib.check(_lib.lib().grim_synchronize(self._h), "synchronize")

    def enableGraph(self, on=True):
        _lib.check(_lib.lib().grim_enable_graph(self._h, int(bool(on))), "enable_graph")

    def setNewtonMode(self, mode, perZone=1, rtol=0.0):
        _lib.check(_lib.lib().grim_set_newton_mode(self._h, int(mode), int(perZone), float(rtol)),
                   "set_newton_mode")
        self.cfg["newtonMode"] = int(mode)
        self.cfg["nonlinearsolve_rtol"] = float(rtol)

    def stats(self):
        s = _lib.GrimStats()
        _lib.check(_lib.lib().grim_get_stats(self._h, ctypes.byref(s)), "get_stats")
        return dict(newtonIters=list(s.newtonIters), unconverged=list(s.unconverged),
                    nonFinite=s.nonFinite, msStep=s.msStep, msStencil=s.msStencil,
                    msNewton=s.msNewton, msOther=s.msOther, kernelLaunches=s.kernelLaunches,
                    waitTimeouts=s.waitTimeouts, drainTimeouts=s.drainTimeouts)

    def setDebug(self, setting, value):
        """Test hook (grim_set_debug), e.g. _lib.DEBUG_SKIP_BULK_COPIES."""
        _lib.check(_lib.lib().grim_set_debug(self._h, int(setting), int(value)), "set_debug")

    def newtonHistogram(self):
        """[stage][iterations] -> zones, for the last step (tangent / mixed)."""
        out = (ctypes.c_longlong * 32)()
        _lib.check(_lib.lib().grim_get_newton_histogram(self._h, out), "newton_histogram")
        return [list(out[0:16]), list(out[16:32])]

    def stream(self):
        return _lib.lib().grim_stream(self._h)

    PROF_GROUPS = ("boundary", "faces_x1", "faces_x2", "faces_x3", "epilogue", "newton", "dt",
                   "diagnostics", "finish", "emhd_prepass")

    def profileSteps(self, nsteps=1):
        """Advance nsteps without the graph, timing every kernel group with
        CUDA events on the stepper's stream: {group: (ms, launch runs)}."""
        n = len(self.PROF_GROUPS)
        ms = (ctypes.c_double * n)()
        cnt = (ctypes.c_longlong * n)()
        _lib.check(_lib.lib().grim_profile_steps(self._h, int(nsteps), ms, cnt, n), "profile_steps")
        return {g: (ms[k], cnt[k]) for k, g in enumerate(self.PROF_GROUPS)}

    def autotune(self):
        """Pick the fastest launch shape of each direction's face kernel on
        the current state (for the current Newton mode): {dir: (variant, ms)}."""
        v = (ctypes.c_int * 3)()
        ms = (ctypes.c_double * 3)()
        _lib.check(_lib.lib().grim_autotune(self._h, v, ms), "autotune")
        return {d: (v[d], ms[d]) for d in range(self.cfg["dim"])}

    def setFaceVariant(self, dir, variant):
        _lib.check(_lib.lib().grim_set_face_variant(self._h, int(dir), int(variant)), "set_face_variant")

    def setFixedDt(self, fixed=True):
        """Hold dt at its current value instead of computeDt."""
        _lib.check(_lib.lib().grim_set_dt_mode(self._h, int(bool(fixed))), "set_dt_mode")

    def adjointForward(self, nsteps, every=10):
        """Advance nsteps with dt fixed, checkpointing primOld every `every`
        steps, for a following adjointBackward."""
        _lib.check(_lib.lib().grim_adjoint_forward(self._h, int(nsteps), int(every)), "adjoint_forward")

    def adjointBackward(self, lam):
        """dL/d(initial primOld) from lam = dL/d(final primOld), both
        [var][k][j][i] with ghosts (interior entries used / returned)."""
        lam = np.ascontiguousarray(lam, dtype=np.float64)
        grad = self._zeros(self.dof)
        _lib.check(_lib.lib().grim_adjoint_backward(self._h, _ptr(lam), _ptr(grad), _lib.HOST),
                   "adjoint_backward")
        return grad

    def adjointStencil(self, prim, gbar):
        """(d divF / d prim)^T gbar on the interior (test entry point)."""
        p = np.ascontiguousarray(prim, dtype=np.float64)
        g = np.ascontiguousarray(gbar, dtype=np.float64)
        out = self._zeros(self.dof)
        _lib.check(_lib.lib().grim_adjoint_stencil(self._h, _ptr(p), _ptr(g), _ptr(out), _lib.HOST),
                   "adjoint_stencil")
        return out

    def countFlops(self):
        """Algorithmic flops of one zone: residual (FP64), tangent pass
        (FP32 and FP64), pivoted solve (FP32 and FP64)."""
        out = (ctypes.c_double * 11)()
        _lib.check(_lib.lib().grim_count_flops(self._h, out), "count_flops")
        keys = ("residual64", "tangent32", "tangent64", "solve32", "solve64", "residual_div", "residual_sqrt_exp",
                "dual_tangent32", "recon_zone_dir", "riemann_face", "epilogue_zone")
        return {k: out[i] for i, k in enumerate(keys)}

    # ---- stage pieces --------------------------------------------------------
    def _zeros(self, nv):
        return np.zeros((nv,) + self.zshape)

    def applyBoundaryConditions(self, which=_lib.PRIM_OLD):
        _lib.check(_lib.lib().grim_apply_boundaries(self._h, int(which)), "apply_boundaries")

    def computeDivOfFluxes(self, prim):
        """divFluxes (dof x Z) and the face fluxes (3 x dof x Z, before CT)."""
        p = np.ascontiguousarray(prim, dtype=np.float64)
        divF = self._zeros(self.dof)
        fl = np.zeros((3, self.dof) + self.zshape)
        _lib.check(_lib.lib().grim_compute_div_fluxes(self._h, _ptr(p), _ptr(divF), _ptr(fl), None,
                                                      _lib.HOST), "computeDivOfFluxes")
        return divF, fl

    def computeEMF(self, prim):
        """timeStepperPy.computeEMF on a prim array: [emfX1, emfX2, emfX3]
        (3 x Z) from the Riemann fluxes of prim."""
        p = np.ascontiguousarray(prim, dtype=np.float64)
        out = np.zeros((3,) + self.zshape)
        _lib.check(_lib.lib().grim_compute_emf(self._h, _ptr(p), _ptr(out), _lib.HOST), "computeEMF")
        return out

    def fluxCT(self, prim):
        """timeStepperPy.fluxCT (constrainedtransport.cpp:3-51) on a prim
        array: the face fluxes (3 x dof x Z) with the field rows replaced by
        the constrained-transport values formed from the edge EMFs on the
        GPU (grim_flux_ct), neighbours by circular shift as in the
        reference: F1_B2 = (E3 + E3[j+1]) / 2, F2_B1 = -(E3 + E3[i+1]) / 2
        and, in 3D, F1_B3 = -(E2 + E2[k+1]) / 2, F3_B1 = (E2 + E2[i+1]) / 2,
        F2_B3 = (E1 + E1[k+1]) / 2, F3_B2 = -(E1 + E1[j+1]) / 2; a
        direction's own field row is zero.  In 1D the Riemann fluxes."""
        p = np.ascontiguousarray(prim, dtype=np.float64)
        fl = np.zeros((3, self.dof) + self.zshape)
        _lib.check(_lib.lib().grim_flux_ct(self._h, _ptr(p), _ptr(fl), _lib.HOST), "fluxCT")
        return fl

    def computeDivB(self, prim):
        """timeStepperPy.computeDivB: corner divergence of sqrt(-g) B (2D)."""
        p = np.ascontiguousarray(prim, dtype=np.float64)
        out = np.zeros(self.zshape)
        _lib.check(_lib.lib().grim_compute_divb(self._h, _ptr(p), _ptr(out), _lib.HOST), "computeDivB")
        return out

    OBSERVERS = ("BaryonMass", "EMag", "ETh", "rhoMax", "betaMin", "MdotIn", "MdotOut",
                 "UnboundMdotOut", "RelativisticUnboundMdotOut")

    def torusObservers(self):
        """The torus observers (ComputeMinMaxVariables, ComputeEnergyIntegrals,
        ComputeBoundaryFluxes of ObserversTorus.hpp) on primOld: {name: value}."""
        out = (ctypes.c_double * 9)()
        _lib.check(_lib.lib().grim_torus_observers(self._h, out), "torus_observers")
        return dict(zip(self.OBSERVERS, list(out)))

    def observations(self, maxRecords=4096):
        """Records written by the steps when ObserveEveryDt > 0, oldest
        first: [{"time": t, name: value, ...}]."""
        buf = (ctypes.c_double * (10 * maxRecords))()
        n = ctypes.c_int(0)
        _lib.check(_lib.lib().grim_get_observations(self._h, buf, int(maxRecords), ctypes.byref(n)),
                   "get_observations")
        recs = []
        for r in range(n.value):
            row = buf[10 * r:10 * r + 10]
            recs.append(dict(time=row[0], **dict(zip(self.OBSERVERS, row[1:]))))
        return recs

    # ---- checkpoint files (grid::dump / grid::load, restart flow) --------
    def dump(self, fileName, which=None):
        """grid::dump of a state (default primOld) as a PETSc binary Vec."""
        w = _lib.PRIM_OLD if which is None else which
        _lib.check(_lib.lib().grim_dump(self._h, int(w), str(fileName).encode()), "dump")

    def load(self, fileName, which=None):
        """grid::load: interior from the file, ghosts as communicate sets them."""
        w = _lib.PRIM_OLD if which is None else which
        _lib.check(_lib.lib().grim_load(self._h, int(w), str(fileName).encode()), "load")

    def writeRestart(self, restartFileName="restartFileName.txt", restartFileTime="restartFileTime.txt"):
        """CheckWallClockTermination's write; returns the data file's name."""
        buf = ctypes.create_string_buffer(256)
        _lib.check(_lib.lib().grim_write_restart(self._h, str(restartFileName).encode(),
                                                 str(restartFileTime).encode(), buf, 256), "write_restart")
        return buf.value.decode()

    def restart(self, restartFileName="restartFileName.txt", restartFileTime="restartFileTime.txt",
                restartFile=None):
        """The constructor's restart branch (timestepper.cpp:386-445)."""
        _lib.check(_lib.lib().grim_restart(self._h, str(restartFileName).encode(), str(restartFileTime).encode(),
                                           None if restartFile is None else str(restartFile).encode()),
                   "restart")

    def reconstruct(self, prim, direction):
        p = np.ascontiguousarray(prim, dtype=np.float64)
        pl, pr = self._zeros(self.dof), self._zeros(self.dof)
        _lib.check(_lib.lib().grim_reconstruct(self._h, _ptr(p), int(direction), _ptr(pl), _ptr(pr),
                                               _lib.HOST), "reconstruct")
        return pl, pr

    def conserved(self, prim):
        p = np.ascontiguousarray(prim, dtype=np.float64)
        out = self._zeros(self.dof)
        _lib.check(_lib.lib().grim_conserved(self._h, _ptr(p), _ptr(out), _lib.HOST), "conserved")
        return out

    def elementFluxes(self, prim, direction):
        """fluidElement::computeFluxes(direction) at the zone centres
        (physics.cpp:185-217): dof x Z; direction 0 gives the conserved
        variables."""
        p = np.ascontiguousarray(prim, dtype=np.float64)
        out = self._zeros(self.dof)
        _lib.check(_lib.lib().grim_element_fluxes(self._h, _ptr(p), int(direction), _ptr(out), _lib.HOST),
                   "elementFluxes")
        return out

    def charSpeeds(self, prim, direction):
        p = np.ascontiguousarray(prim, dtype=np.float64)
        mn, mx = np.zeros(self.zshape), np.zeros(self.zshape)
        _lib.check(_lib.lib().grim_char_speeds(self._h, _ptr(p), int(direction), _ptr(mn), _ptr(mx),
                                               _lib.HOST), "charSpeeds")
        return mn, mx

    def stageGrid(self, which):
        """consOld (STAGE_CONS_OLD, dof rows), divFluxes or sourcesExplicit
        (nf fluid rows) as the last stage left them; interior zones."""
        rows = self.dof if which == _lib.STAGE_CONS_OLD else self.numFluidVars
        out = self._zeros(rows)
        _lib.check(_lib.lib().grim_get_stage_grid(self._h, int(which), _ptr(out), _lib.HOST), "stageGrid")
        return out

    def stageSetup(self, stage):
        _lib.check(_lib.lib().grim_stage_setup(self._h, int(stage)), "stage_setup")

    def computeResidual(self, primGuess):
        p = np.ascontiguousarray(primGuess, dtype=np.float64)
        out = self._zeros(self.numFluidVars)
        _lib.check(_lib.lib().grim_residual(self._h, _ptr(p), _ptr(out), _lib.HOST), "residual")
        return out

    def jacobianFD(self, primGuess):
        p = np.ascontiguousarray(primGuess, dtype=np.float64)
        nf = self.numFluidVars
        J = np.zeros(self.zshape + (nf, nf))
        _lib.check(_lib.lib().grim_jacobian_fd(self._h, _ptr(p), _ptr(J), _lib.HOST), "jacobian_fd")
        return J

    def jacobianTangent(self, primGuess):
        p = np.ascontiguousarray(primGuess, dtype=np.float64)
        nf = self.numFluidVars
        J = np.zeros(self.zshape + (nf, nf))
        _lib.check(_lib.lib().grim_jacobian_tangent(self._h, _ptr(p), _ptr(J), _lib.HOST), "jacobian_tangent")
        return J

    JAC_FD64, JAC_FAST64, JAC_DUAL64, JAC_FAST32 = 0, 1, 2, 3

    def jacobianForm(self, primGuess, form):
        """The Jacobian in one of the JAC_* forms (grim_jacobian_form)."""
        p = np.ascontiguousarray(primGuess, dtype=np.float64)
        nf = self.numFluidVars
        J = np.zeros(self.zshape + (nf, nf))
        _lib.check(_lib.lib().grim_jacobian_form(self._h, _ptr(p), _ptr(J), int(form), _lib.HOST), "jacobian_form")
        return J

    def solve(self):
        it = ctypes.c_int()
        _lib.check(_lib.lib().grim_newton_solve(self._h, ctypes.byref(it)), "newton_solve")
        return it.value

    def getGeometry(self, location):
        out = np.zeros((34,) + self.zshape)
        gam = np.zeros((64,) + self.zshape)
        xc = np.zeros((5,) + self.zshape)
        _lib.check(_lib.lib().grim_get_geometry(self._h, int(location), _ptr(out), _ptr(gam), _ptr(xc),
                                                _lib.HOST), "get_geometry")
        return dict(gCov=out[:16].reshape((4, 4) + self.zshape), gCon=out[16:32].reshape((4, 4) + self.zshape),
                    g=out[32], alpha=out[33], gamma=gam.reshape((4, 4, 4) + self.zshape), x=xc)

    def setGeometry(self, location, gCov, gCon, g, alpha, x=None, gamma=None):
        out = np.concatenate([np.reshape(gCov, (16,) + self.zshape), np.reshape(gCon, (16,) + self.zshape),
                              np.reshape(g, (1,) + self.zshape), np.reshape(alpha, (1,) + self.zshape)])
        out = np.ascontiguousarray(out, dtype=np.float64)
        xc = None if x is None else np.ascontiguousarray(np.reshape(x, (-1,) + self.zshape)[:5])
        gm = None if gamma is None else np.ascontiguousarray(np.reshape(gamma, (64,) + self.zshape))
        _lib.check(_lib.lib().grim_set_geometry(self._h, int(location), _ptr(out),
                                                None if gm is None else _ptr(gm),
                                                None if xc is None else _ptr(xc), _lib.HOST), "set_geometry")


class Batch:
    """Independent problems stepped together (grim_batch_*): per problem the
    stencil launches, per stage one compacted Newton launch per iteration
    over all problems' unconverged zones.  problems[p] is a timeStepper view
    of problem p (state, time, statistics); the batch owns it."""

    def __init__(self, cfgs, device=0):
        L = _lib.lib()
        n = len(cfgs)
        arr = (type(C.to_struct(cfgs[0])) * n)(*[C.to_struct(dict(c)) for c in cfgs])
        self._b = ctypes.c_void_p()
        _lib.check(L.grim_batch_create(ctypes.cast(arr, ctypes.c_void_p), n, int(device), ctypes.byref(self._b)),
                   "grim_batch_create")
        self.problems = []
        for p, cfg in enumerate(cfgs):
            h = ctypes.c_void_p()
            _lib.check(L.grim_batch_problem(self._b, p, ctypes.byref(h)), "grim_batch_problem")
            ts = timeStepper(cfg, _handle=h.value)
            ts.cfg["newtonMode"] = C.NEWTON_MIXED32
            self.problems.append(ts)

    def setNewtonMode(self, mode, rtol=0.0):
        _lib.check(_lib.lib().grim_batch_set_newton_mode(self._b, int(mode), float(rtol)), "batch_newton_mode")
        for ts in self.problems:
            ts.cfg["newtonMode"] = int(mode)

    def enableGraph(self, on=True):
        _lib.check(_lib.lib().grim_batch_enable_graph(self._b, int(bool(on))), "batch_enable_graph")

    def timeSteps(self, n):
        _lib.check(_lib.lib().grim_batch_time_steps(self._b, int(n)), "batch_time_steps")

    def synchronize(self):
        _lib.check(_lib.lib().grim_batch_synchronize(self._b), "batch_synchronize")

    def stream(self):
        return self.problems[0].stream()

    def close(self):
        if getattr(self, "_b", None) and self._b.value:
            for ts in self.problems:
                ts._h = ctypes.c_void_p()
            _lib.lib().grim_batch_destroy(self._b)
            self._b = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def measurePeaks(device=0):
    """(fp64 TFLOP/s, fp32 TFLOP/s, HBM GB/s) measured on ``device``."""
    a, b, c = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
    _lib.check(_lib.lib().grim_measure_peaks(int(device), ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)),
               "measure_peaks")
    return a.value, b.value, c.value


def batchSolve(A, b):
    """The batched pivoted solve of the Newton kernels on a host batch."""
    A = np.ascontiguousarray(A, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    n, batch = A.shape[-1], A.shape[0]
    x = np.zeros((batch, n))
    _lib.check(_lib.lib().grim_batch_solve(n, batch, _ptr(A), _ptr(b), _ptr(x), _lib.HOST), "batch_solve")
    return x
