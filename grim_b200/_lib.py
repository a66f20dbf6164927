"""ctypes binding of libgrim_b200.so (include/grim_b200.h).

The library is built in place by grim_b200/build.py (``__graft_entry__.build``)
and loaded from this package directory.  A missing library is an error:
there is no CPU fallback for the timestep.
"""
import ctypes
import os
import re

from .config import GrimConfig

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libgrim_b200.so")
HEADER = os.path.join(_HERE, "..", "include", "grim_b200.h")
_LIB = None

GRIM_OK = 0
GRIM_ETIMEOUT = -6
DEBUG_SKIP_BULK_COPIES = 1
LAYOUT_GHOSTED, LAYOUT_INTERIOR = 0, 1
HOST, DEVICE = 0, 1
PRIM_OLD, PRIM, PRIM_HALF = 0, 1, 2
STAGE_CONS_OLD, STAGE_DIV_FLUXES, STAGE_SOURCES_EXPLICIT = 0, 1, 2


class GrimStats(ctypes.Structure):
    _fields_ = [
        ("newtonIters", ctypes.c_int * 2),
        ("unconverged", ctypes.c_longlong * 2),
        ("nonFinite", ctypes.c_longlong),
        ("msStep", ctypes.c_double),
        ("msStencil", ctypes.c_double),
        ("msNewton", ctypes.c_double),
        ("msOther", ctypes.c_double),
        ("kernelLaunches", ctypes.c_longlong),
        ("waitTimeouts", ctypes.c_longlong),
        ("drainTimeouts", ctypes.c_longlong),
        ("reserved", ctypes.c_double * 6),
    ]


class GrimError(RuntimeError):
    def __init__(self, msg, status=None):
        super().__init__(msg)
        self.status = status


def declared_symbols():
    """Function names declared in include/grim_b200.h."""
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(grim_[a-z_0-9]+)\s*\(", txt)))


def lib():
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise GrimError("libgrim_b200.so not built (run __graft_entry__.build()); "
                        "there is no CPU fallback")
    L = ctypes.CDLL(LIB_PATH)
    P = ctypes.POINTER
    vp, i, d = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
    dp = P(ctypes.c_double)
    sig = {
        "grim_create": [P(GrimConfig), i, P(vp)],
        "grim_destroy": [vp],
        "grim_dims": [vp, P(i), P(i), P(i), P(i), P(i)],
        "grim_set_prims": [vp, i, vp, i],
        "grim_get_prims": [vp, i, vp, i],
        "grim_time_step": [vp, P(i), P(i)],
        "grim_time_steps": [vp, i],
        "grim_time_steps_host": [vp, i, vp, vp, i],
        "grim_get_time": [vp, P(d), P(d)],
        "grim_set_time": [vp, d, d],
        "grim_compute_dt": [vp],
        "grim_apply_boundaries": [vp, i],
        "grim_communicate": [vp, i],
        "grim_compute_div_fluxes": [vp, vp, vp, vp, vp, i],
        "grim_compute_emf": [vp, vp, vp, i],
        "grim_flux_ct": [vp, vp, vp, i],
        "grim_capture_graph": [vp, i],
        "grim_reconstruct": [vp, vp, i, vp, vp, i],
        "grim_compute_divb": [vp, vp, vp, i],
        "grim_torus_observers": [vp, P(d)],
        "grim_step_segment": [vp, i],
        "grim_halo_x3": [vp, i, i, i, vp],
        "grim_scalar_get": [vp, i, vp],
        "grim_scalar_set": [vp, i, vp],
        "grim_dump": [vp, i, ctypes.c_char_p],
        "grim_load": [vp, i, ctypes.c_char_p],
        "grim_write_restart": [vp, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, i],
        "grim_restart": [vp, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p],
        "grim_petsc_vec_write": [ctypes.c_char_p, vp, ctypes.c_longlong],
        "grim_petsc_vec_read": [ctypes.c_char_p, vp, ctypes.c_longlong],
        "grim_natural_from_prims": [P(GrimConfig), vp, vp],
        "grim_prims_from_natural": [P(GrimConfig), vp, vp],
        "grim_get_observations": [vp, P(d), i, P(i)],
        "grim_conserved": [vp, vp, vp, i],
        "grim_element_fluxes": [vp, vp, i, vp, i],
        "grim_char_speeds": [vp, vp, i, vp, vp, i],
        "grim_stage_setup": [vp, i],
        "grim_get_stage_grid": [vp, i, vp, i],
        "grim_residual": [vp, vp, vp, i],
        "grim_jacobian_fd": [vp, vp, vp, i],
        "grim_jacobian_tangent": [vp, vp, vp, i],
        "grim_jacobian_form": [vp, vp, vp, i, i],
        "grim_newton_solve": [vp, P(i)],
        "grim_batch_solve": [i, i, vp, vp, vp, i],
        "grim_get_geometry": [vp, i, vp, vp, vp, i],
        "grim_set_geometry": [vp, i, vp, vp, vp, i],
        "grim_set_newton_mode": [vp, i, i, d],
        "grim_get_stats": [vp, P(GrimStats)],
        "grim_enable_graph": [vp, i],
        "grim_synchronize": [vp],
        "grim_problem_init": [vp],
        "grim_get_newton_histogram": [vp, P(ctypes.c_longlong)],
        "grim_measure_peaks": [i, P(d), P(d), P(d)],
        "grim_profile_steps": [vp, i, P(d), P(ctypes.c_longlong), i],
        "grim_count_flops": [vp, P(d)],
        "grim_autotune": [vp, P(i), P(d)],
        "grim_set_face_variant": [vp, i, i],
        "grim_set_dt_mode": [vp, i],
        "grim_set_debug": [vp, i, i],
        "grim_adjoint_forward": [vp, i, i],
        "grim_adjoint_backward": [vp, vp, vp, i],
        "grim_adjoint_stencil": [vp, vp, vp, vp, i],
        "grim_batch_create": [vp, i, i, P(vp)],
        "grim_batch_destroy": [vp],
        "grim_batch_problem": [vp, i, P(vp)],
        "grim_batch_set_newton_mode": [vp, i, d],
        "grim_batch_enable_graph": [vp, i],
        "grim_batch_time_steps": [vp, i],
        "grim_batch_synchronize": [vp],
        "grim_batch_size": [vp],
    }
    for name, args in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = ctypes.c_int
    L.grim_version.restype = ctypes.c_char_p
    L.grim_last_error.restype = ctypes.c_char_p
    L.grim_stream.argtypes = [vp]
    L.grim_stream.restype = vp
    _LIB = L
    return L


def check(rc, what=""):
    if rc != GRIM_OK:
        msg = lib().grim_last_error().decode(errors="replace")
        raise GrimError("%s failed (status %d): %s" % (what, rc, msg), rc)
