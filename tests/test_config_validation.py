"""grim_create's configuration checks (include/grim_b200.h, grim_create),
and the NULL-handle refusal of every entry point that takes a handle.

The checks run before any CUDA call, so these run on the CPU: each invalid
configuration is refused with GRIM_EINVAL and grim_last_error() naming
what is wrong, and no handle is returned.  The reference's timeStepper
constructor (timestepper.cpp:4-446) takes its parameters as given; the C
ABI refuses what its kernels cannot run instead of running something else.
"""
import ctypes
import math

import pytest

from grim_b200 import _lib
from grim_b200 import config as C

EINVAL = -1


def _create(cfg):
    s = C.to_struct(cfg)
    h = ctypes.c_void_p(12345)
    rc = _lib.lib().grim_create(ctypes.byref(s), 0, ctypes.byref(h))
    return rc, h.value, _lib.lib().grim_last_error().decode()


def _base(**kw):
    return C.make_config(dim=2, N1=16, N2=16, **kw)


CASES = [
    ("dim 0", dict(dim=0), "dim"),
    ("dim 4", dict(dim=4), "dim"),
    ("numGhost 2", dict(numGhost=2), "numGhost"),
    ("N1 below 4", dict(N1=3), "at least 4 zones"),
    ("N2 below 4 in 2D", dict(N2=2), "at least 4 zones"),
    ("reconstruction 4", dict(reconstruction=4), "reconstruction"),
    ("reconstruction -1", dict(reconstruction=-1), "reconstruction"),
    ("maxNonLinearIter 0", dict(maxNonLinearIter=0), "maxNonLinearIter"),
    ("maxNonLinearIter 16", dict(maxNonLinearIter=16), "maxNonLinearIter"),
    ("maxLineSearchIters 0", dict(maxLineSearchIters=0), "maxLineSearchIters"),
    ("maxLineSearchIters 33", dict(maxLineSearchIters=33), "maxLineSearchIters"),
    ("metric 2", dict(metric=2), "metric"),
    ("riemannSolver 2", dict(riemannSolver=2), "riemannSolver"),
    ("closure 3", dict(closure=3), "closure"),
    ("problem 2", dict(problem=2), "problem"),
    ("newtonMode 4", dict(newtonMode=4), "newtonMode"),
    ("newtonMode -1", dict(newtonMode=-1), "newtonMode"),
    ("perZoneConvergence 4", dict(perZoneConvergence=4), "perZoneConvergence"),
    ("X1End == X1Start", dict(X1End=0.), "XEnd > XStart"),
    ("X2End < X2Start", dict(X2Start=1., X2End=0.), "XEnd > XStart"),
    ("X1End NaN", dict(X1End=math.nan), "XEnd > XStart"),
    ("boundary 5", dict(boundaryLeft=5), "boundary"),
    ("boundary -1", dict(boundaryTop=-1), "boundary"),
    ("N3Global in 2D", dict(N3Global=8), "N3Global"),
    ("N3Global negative", dict(N3Global=-1), "N3Global"),
    ("ulps negative", dict(nonlinearsolve_ulps=-1.), "nonlinearsolve_ulps"),
    ("ulps NaN", dict(nonlinearsolve_ulps=math.nan), "nonlinearsolve_ulps"),
    ("torus problem, Minkowski", dict(problem=C.PROBLEM_TORUS), "MKS"),
    ("torus closure, Minkowski", dict(closure=C.CLOSURE_TORUS), "MKS"),
]


@pytest.mark.parametrize("name,overrides,words", CASES, ids=[c[0] for c in CASES])
def test_invalid_configuration_is_refused(name, overrides, words):
    cfg = _base()
    cfg.update(overrides)
    rc, h, msg = _create(cfg)
    assert rc == EINVAL, (name, rc, msg)
    assert h is None, "no handle on a refused configuration"
    assert words in msg, (name, msg)


def test_dirichlet_sides_are_not_supported():
    """boundary.cpp:5-241 leaves DIRICHLET sides to the problem's hook; no
    supported problem has one, so such a side is refused, not filled."""
    cfg = _base(boundaryRight=C.DIRICHLET)
    rc, h, msg = _create(cfg)
    assert rc == -5 and h is None and "GRIM_DIRICHLET" in msg


def test_slab_count_below_the_slab_is_refused():
    cfg = C.make_config(dim=3, N1=8, N2=8, N3=8, N3Global=4)
    rc, h, msg = _create(cfg)
    assert rc == EINVAL and h is None and "N3Global" in msg


def test_grid_beyond_32_bit_zone_indices_is_refused():
    # 1300^3 interior zones: 1306^3 > 2^31 with ghosts
    cfg = C.make_config(dim=3, N1=1300, N2=1300, N3=1300)
    rc, h, msg = _create(cfg)
    assert rc == EINVAL and h is None and "2^31" in msg


def test_null_arguments_are_refused():
    L = _lib.lib()
    h = ctypes.c_void_p()
    assert L.grim_create(None, 0, ctypes.byref(h)) == EINVAL
    s = C.to_struct(_base())
    assert L.grim_create(ctypes.byref(s), 0, None) == EINVAL


# entry points whose first argument is a handle; grim_destroy and
# grim_batch_destroy accept NULL as a no-op and grim_batch_size(NULL) is 0
_NO_OP_ON_NULL = {"grim_destroy": 0, "grim_batch_destroy": 0, "grim_batch_size": 0}


def _handle_entry_points():
    import re
    import inspect
    src = inspect.getsource(_lib.lib)
    return re.findall(r'"(grim_[a-z0-9_]+)": \[vp', src)


def test_every_handle_entry_point_refuses_a_null_handle():
    """Each call taking a grim_handle / grim_batch first returns GRIM_EINVAL
    (nothing runs, no CUDA call) when that handle is NULL, with every other
    pointer NULL and every number zero."""
    L = _lib.lib()
    names = _handle_entry_points()
    assert len(names) > 50
    for n in names:
        f = getattr(L, n)
        args = [None]
        for t in f.argtypes[1:]:
            if t in (ctypes.c_int, ctypes.c_longlong):
                args.append(0)
            elif t is ctypes.c_double:
                args.append(0.)
            else:
                args.append(None)
        want = _NO_OP_ON_NULL.get(n, EINVAL)
        assert f(*args) == want, n
