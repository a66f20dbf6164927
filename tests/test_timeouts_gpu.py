"""Bounded device waits are reported, and the handle stays usable.

The TMA-staged face kernels wait at most 1 s on each copy they issue.  The
debug setting GRIM_DEBUG_SKIP_BULK_COPIES makes them issue none, so every
wait runs out (no copy is ever in flight, nothing faults): the step's X1
fluxes are not computed, the give-up is counted in grim_stats.waitTimeouts
and the next synchronising call returns GRIM_ETIMEOUT once.  After the
setting is cleared and the primitives are set again, the handle steps to
the same bits as a handle that never saw the setting.
"""
import numpy as np
import pytest

from grim_b200 import _lib
from grim_b200 import problems as PR

pytestmark = pytest.mark.gpu

X1_TMA_VARIANT = 2  # k_face_flux_x1_tma, 3 blocks per SM (ideal MHD face kernels)


def _stepper(cfg, P):
    from grim_b200.timestepper import timeStepper
    ts = timeStepper(cfg)
    ts.setFaceVariant(0, X1_TMA_VARIANT)
    ts.setFixedDt(True)
    ts.primOld.setVars(P)
    return ts


def test_copy_wait_that_runs_out_is_reported_and_the_handle_recovers():
    cfg = PR.fast_mode_config(N=64)
    P = PR.fast_mode_prims(cfg)
    ts, ref = _stepper(cfg, P), _stepper(cfg, P)
    t0, dt0 = ts.time, ts.dt

    ts.setDebug(_lib.DEBUG_SKIP_BULK_COPIES, 1)
    ts.timeStep()  # enqueued; the waits run out on the device
    with pytest.raises(_lib.GrimError) as err:
        ts.synchronize()
    assert err.value.status == _lib.GRIM_ETIMEOUT
    st = ts.stats()
    assert st["waitTimeouts"] > 0
    assert st["drainTimeouts"] == 0  # no copy was in flight when the warps stopped
    ts.synchronize()  # reported once
    # a stepping call refuses while the error word is raised (the stats
    # getter waits for the stream but leaves the word for the next call)
    ts.timeStep()
    ts.stats()
    with pytest.raises(_lib.GrimError) as err:
        ts.timeStep()
    assert err.value.status == _lib.GRIM_ETIMEOUT
    ts.synchronize()

    ts.setDebug(_lib.DEBUG_SKIP_BULK_COPIES, 0)
    seen = ts.stats()["waitTimeouts"]
    for h in (ts, ref):
        h.primOld.setVars(P)
        h.setTime(t0, dt0)
        for _ in range(3):
            h.timeStep()
        h.synchronize()
    assert ts.stats()["waitTimeouts"] == seen
    a, b = ts.primOld.getVars(), ref.primOld.getVars()
    assert np.array_equal(a, b)
    assert np.all(np.isfinite(a))
