"""Bad arguments on a live handle are refused and change nothing.

Each call below passes one invalid argument (a state selector, memory
kind, layout, direction, variant, mode, location, segment, setting or count
outside its range, or a NULL buffer) and must return GRIM_EINVAL with
grim_last_error() saying why, before any work is enqueued.  After all of
them the handle steps to the same bits as a handle that never saw them.
"""
import ctypes

import numpy as np
import pytest

from grim_b200 import _lib
from grim_b200 import config as C
from grim_b200 import problems as PR

pytestmark = pytest.mark.gpu

EINVAL = -1


def _stepper(cfg, P):
    from grim_b200.timestepper import timeStepper
    ts = timeStepper(cfg)
    ts.setFixedDt(True)
    ts.primOld.setVars(P)
    return ts


def _refused(rc, words):
    assert rc == EINVAL, rc
    msg = _lib.lib().grim_last_error().decode()
    assert words in msg, msg


def test_bad_arguments_are_refused_and_leave_the_handle_as_it_was():
    cfg = PR.fast_mode_config(N=32)
    P = PR.fast_mode_prims(cfg)
    ts, ref = _stepper(cfg, P), _stepper(cfg, P)
    L, h = _lib.lib(), ts._h
    host = np.zeros(ts.prim.getVars().shape)
    hp = ctypes.c_void_p(host.ctypes.data)

    _refused(L.grim_set_prims(h, 9, hp, _lib.HOST), "state selector")
    _refused(L.grim_set_prims(h, _lib.PRIM_OLD, hp, 7), "memKind")
    _refused(L.grim_set_prims(h, _lib.PRIM_OLD, None, _lib.HOST), "null")
    _refused(L.grim_get_prims(h, -1, hp, _lib.HOST), "state selector")
    _refused(L.grim_get_prims(h, _lib.PRIM_OLD, hp, -3), "memKind")
    _refused(L.grim_time_steps(h, -1), "nsteps")
    _refused(L.grim_time_steps_host(h, 1, None, None, 5), "grim_time_steps_host")
    _refused(L.grim_apply_boundaries(h, 9), "state selector")
    _refused(L.grim_communicate(h, 9), "state selector")
    _refused(L.grim_set_face_variant(h, 2, 0), "direction")  # a 2D grid has no X3 faces
    _refused(L.grim_set_face_variant(h, 0, 999), "variant")
    _refused(L.grim_set_newton_mode(h, 7, 1, 1e-10), "mode")
    _refused(L.grim_get_geometry(h, 9, None, None, None, _lib.HOST), "location")
    _refused(L.grim_step_segment(h, 9), "segment")
    _refused(L.grim_halo_x3(h, _lib.PRIM_OLD, 0, 0, hp), "3D grid")
    _refused(L.grim_set_debug(h, 99, 1), "setting")
    _refused(L.grim_adjoint_forward(h, 0, 1), "grim_adjoint_forward")
    ms = (ctypes.c_double * 8)()
    _refused(L.grim_profile_steps(h, 1, ms, None, 0), "grim_profile_steps")
    nrec = ctypes.c_int()
    _refused(L.grim_get_observations(h, None, 4, ctypes.byref(nrec)), "grim_get_observations")
    _refused(L.grim_residual(h, hp, hp, 2), "memKind")

    for s in (ts, ref):
        for _ in range(3):
            s.timeStep()
    np.testing.assert_array_equal(ts.primOld.getVars(), ref.primOld.getVars())
    assert (ts.time, ts.dt) == (ref.time, ref.dt)


ESTATE = -4


def test_calls_out_of_order_are_refused_with_estate():
    """The Newton pieces read the stage grim_stage_setup formed: before it,
    and after a step has replaced its constants, they return GRIM_ESTATE;
    the adjoint's backward sweep needs a forward run first."""
    cfg = PR.fast_mode_config(N=16)
    P = PR.fast_mode_prims(cfg)
    ts = _stepper(cfg, P)
    L, h = _lib.lib(), ts._h
    host = np.zeros(ts.prim.getVars().shape)
    hp = ctypes.c_void_p(host.ctypes.data)
    it = ctypes.c_int()

    def refused(rc):
        assert rc == ESTATE, rc
        assert "grim_stage_setup" in L.grim_last_error().decode()

    refused(L.grim_residual(h, hp, hp, _lib.HOST))
    refused(L.grim_jacobian_fd(h, hp, hp, _lib.HOST))
    refused(L.grim_newton_solve(h, ctypes.byref(it)))
    ts.stageSetup(C.HALF_STEP)
    r = ts.computeResidual(P)
    assert np.isfinite(r).all()
    ts.timeStep()
    refused(L.grim_jacobian_tangent(h, hp, hp, _lib.HOST))
    ts.stageSetup(C.HALF_STEP)
    assert np.isfinite(ts.computeResidual(ts.primOld.getVars())).all()

    rc = L.grim_adjoint_backward(h, hp, hp, _lib.HOST)
    assert rc == ESTATE and "grim_adjoint_forward" in L.grim_last_error().decode()
