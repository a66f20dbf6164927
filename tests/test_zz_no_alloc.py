"""grim_div_fluxes_noalloc: the flux divergence for callers that cannot call
cudaMalloc (their device memory belongs to their own pool allocator, or they
call in the middle of asynchronous work).  It takes device pointers for the
primitives and the result and keeps all of its scratch in one static 64 MiB
device array, so it must give the same divergence as the allocating entry
point grim_compute_div_fluxes.

Calls in a row with different workloads (ideal MHD in 2D, EMHD, whose
scratch layout differs, Orszag-Tang with WENO5/HLL, and a 3D grid with its
three corner EMFs) are each compared with grim_compute_div_fluxes at the
tolerance of the other divergence tests (1e-13 of each variable's scale).
A grid whose scratch fits just under the limit is computed; the next size
up is refused.  This file is collected last so a failure here leaves the
rest of the suite already run.
"""
import ctypes

import numpy as np
import pytest

from grim_b200 import _lib
from grim_b200 import config as C
from grim_b200 import problems as PR
from tests.helpers import interior, scaled_err

pytestmark = pytest.mark.gpu


def _noalloc(cfg, prim_dev, out_dev, stream):
    L = _lib.lib()
    f = L.grim_div_fluxes_noalloc
    f.argtypes = [ctypes.POINTER(C.GrimConfig), ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    f.restype = ctypes.c_int
    s = C.to_struct(cfg)
    return f(ctypes.byref(s), ctypes.c_void_p(prim_dev), ctypes.c_void_p(out_dev), ctypes.c_void_p(stream))


def test_noalloc_divergence_matches_allocating_entry_point():
    cases = [
        (PR.fast_mode_config(N=48), PR.fast_mode_prims),
        (PR.linear_modes_config(N=40), lambda c: PR.linear_modes_prims(c, amplitude=1e-3)),
        (PR.orszag_tang_config(N=64), PR.orszag_tang_prims),
        (PR.fast_mode_config(N=24, dim=3, N3=24), PR.fast_mode_prims),
        (PR.fast_mode_config(N=48), PR.fast_mode_prims),  # the first workload again, after the others
    ]
    _compare_cases(cases)


def _compare_cases(cases):
    import torch
    from grim_b200.timestepper import timeStepper
    stream = torch.cuda.current_stream().cuda_stream
    for cfg, mk in cases:
        P = np.ascontiguousarray(mk(cfg))
        ref, _ = timeStepper(cfg).computeDivOfFluxes(P)
        prim_dev = torch.from_numpy(P).cuda()
        out_dev = torch.zeros_like(prim_dev)
        torch.cuda.synchronize()
        rc = _noalloc(cfg, prim_dev.data_ptr(), out_dev.data_ptr(), stream)
        torch.cuda.synchronize()
        assert rc == 0, _lib.lib().grim_last_error()
        got = out_dev.cpu().numpy()
        assert scaled_err(interior(cfg, got), interior(cfg, ref)) <= 1e-13


SCRATCH_WORDS = 8 * 1024 * 1024  # the documented limit: 64 MiB of doubles


def _scratch_words(cfg):
    """Scratch the call needs for a 2D/3D ideal-MHD grid: face fluxes per
    direction, the stage's conserved variables and guess (dof rows each),
    the explicit sources (nf rows), plus at most 1024 words of device
    scalars."""
    dof, nf = C.var_counts(cfg)
    n1, n2, n3 = C.total_dims(cfg)
    Z = n1 * n2 * n3
    return cfg["dim"] * dof * Z + 2 * dof * Z + nf * Z


def test_noalloc_at_the_scratch_limit():
    """The largest 2D ideal-MHD grid whose scratch fits (470^2 + ghosts) is
    computed like the allocating entry point; 471^2 is refused."""
    fits, over = PR.fast_mode_config(N=470), PR.fast_mode_config(N=471)
    assert _scratch_words(fits) + 1024 <= SCRATCH_WORDS < _scratch_words(over)
    _compare_cases([(fits, PR.fast_mode_prims)])
    _expect_refused(over)


def _expect_refused(cfg):
    import torch
    dof, _ = C.var_counts(cfg)
    n1, n2, n3 = C.total_dims(cfg)
    prim_dev = torch.zeros((dof, n3, n2, n1), dtype=torch.float64, device="cuda")
    out_dev = torch.zeros_like(prim_dev)
    rc = _noalloc(cfg, prim_dev.data_ptr(), out_dev.data_ptr(), torch.cuda.current_stream().cuda_stream)
    assert rc == -1
    assert b"maximum" in _lib.lib().grim_last_error()


def test_noalloc_rejects_grids_beyond_the_scratch_limit():
    _expect_refused(PR.fast_mode_config(N=1024))
