"""grim_time_steps_host: steps fed from and read back to host buffers with
the copies overlapped against the steps, bit for bit the same as the same
sequence of grim_set_prims / grim_time_step / grim_get_prims calls.

Each case runs one handle through the pipelined call and a second, equal
handle through the sequential calls, with states loaded before some steps
(None elsewhere: the step continues from the last one) and read after some
steps, in pinned (torch pin_memory) and pageable (numpy) host memory, with
the step as a CUDA graph and as plain launches.
"""
import numpy as np
import pytest

from grim_b200 import config as C
from grim_b200 import problems as PR

pytestmark = pytest.mark.gpu

# which steps load a state (index into the inputs) and which are read back
LOADS = [0, None, 1, None, None, 2, None]
READS = [True, False, True, True, False, True, True]


def _pair(cfg, P, graph):
    from grim_b200.timestepper import timeStepper
    out = []
    for _ in range(2):
        ts = timeStepper(cfg)
        ts.setNewtonMode(C.NEWTON_MIXED32, 1, cfg["nonlinearsolve_rtol"])
        ts.primOld.setVars(P)
        ts.enableGraph(graph)
        out.append(ts)
    return out


def _states(cfg, P, count, seed=3):
    rng = np.random.default_rng(seed)
    return [np.ascontiguousarray(P * (1 + 1e-3 * rng.standard_normal(P.shape))) for _ in range(count)]


def _host(shape, pinned):
    if pinned:
        import torch
        t = torch.zeros(shape, dtype=torch.float64).pin_memory()
        return t, t.data_ptr(), lambda: t.numpy().copy()
    a = np.zeros(shape)
    return a, a.ctypes.data, lambda: a.copy()


@pytest.mark.parametrize("graph", [True, False])
@pytest.mark.parametrize("pinned", [True, False])
def test_pipelined_steps_match_the_sequential_calls(graph, pinned):
    cfg = PR.orszag_tang_config(N=128, maxNonLinearIter=4, nonlinearsolve_rtol=1e-10, nonlinearsolve_ulps=8.)
    P = PR.orszag_tang_prims(cfg)
    piped, seq = _pair(cfg, P, graph)
    inputs = _states(cfg, P, 3)
    held = []
    in_ptrs = []
    for a in inputs:
        if pinned:
            import torch
            t = torch.from_numpy(a).pin_memory()
            held.append(t)
            in_ptrs.append(t.data_ptr())
        else:
            in_ptrs.append(a.ctypes.data)
    outs = [_host(P.shape, pinned) if r else None for r in READS]

    piped.timeStepsHost([None if k is None else in_ptrs[k] for k in LOADS],
                        [None if o is None else o[1] for o in outs])

    expect = []
    for k, r in zip(LOADS, READS):
        if k is not None:
            seq.primOld.setVars(inputs[k])
        seq.timeStep()
        expect.append(seq.primOld.getVars() if r else None)

    for step, (o, e) in enumerate(zip(outs, expect)):
        if o is None:
            continue
        got = o[2]()
        assert np.array_equal(got, e), "step %d differs by %g" % (step, np.max(np.abs(got - e)))
    assert piped.time == seq.time and piped.dt == seq.dt
    assert np.array_equal(piped.primOld.getVars(), seq.primOld.getVars())


def test_no_host_buffers_is_plain_stepping():
    """NULL input and output lists step like grim_time_steps; the
    handle's later sequential calls see the state the pipelined call left."""
    cfg = PR.orszag_tang_config(N=64)
    P = PR.orszag_tang_prims(cfg)
    piped, seq = _pair(cfg, P, True)
    piped.timeStepsHost([None] * 4, [None] * 4)
    seq.timeSteps(4)
    assert np.array_equal(piped.primOld.getVars(), seq.primOld.getVars())
    piped.timeStep()
    seq.timeStep()
    assert np.array_equal(piped.primOld.getVars(), seq.primOld.getVars())


@pytest.mark.parametrize("problem", ["orszag_tang", "torus"])
def test_interior_layout_matches_the_ghosted_calls(problem):
    """GRIM_LAYOUT_INTERIOR: host arrays of the interior zones only; the
    library forms the periodic ghosts as grid::communicate does and the
    step's boundary pass the others, so the results equal the sequential
    calls given whole arrays whose ghosts were communicated (here the
    input's interior with garbage ghosts, then grim_communicate), bit for
    bit."""
    import torch
    if problem == "torus":
        from grim_b200.problems import torus as T
        from grim_b200.timestepper import timeStepper
        cfg = dict(T.torus_config(N1=64, N2=32, N3=8), nonlinearsolve_atol=1e-24, nonlinearsolve_rtol=1e-10,
                   nonlinearsolve_ulps=8.)
        P, _ = T.torus_prims(cfg, timeStepper(cfg).getGeometry(C.CENTER))
    else:
        cfg = PR.orszag_tang_config(N=128, maxNonLinearIter=4, nonlinearsolve_rtol=1e-10,
                                    nonlinearsolve_ulps=8.)
        P = PR.orszag_tang_prims(cfg)
    piped, seq = _pair(cfg, P, True)
    if problem == "torus":
        for ts in (piped, seq):
            ts.problemInit()
    sl = (slice(None),) + tuple(C.interior_slices(cfg))
    inputs = _states(cfg, P, 2)
    inner = [torch.from_numpy(np.ascontiguousarray(a[sl])).pin_memory() for a in inputs]
    outs = [torch.zeros(inner[0].shape, dtype=torch.float64).pin_memory() for _ in range(4)]
    loads = [0, None, 1, None]
    piped.timeStepsHost([None if k is None else inner[k].data_ptr() for k in loads],
                        [o.data_ptr() for o in outs], interior=True)
    rng = np.random.default_rng(11)
    for step, k in enumerate(loads):
        if k is not None:
            full = rng.standard_normal(P.shape)
            full[sl] = inputs[k][sl]
            seq.primOld.setVars(full)
            seq.primOld.communicate()
        seq.timeStep()
        e = seq.primOld.getVars()[sl]
        assert np.array_equal(outs[step].numpy(), e), step
    assert piped.time == seq.time and piped.dt == seq.dt


def test_timeout_inside_the_pipeline_is_reported():
    """A bounded device wait that runs out during the pipelined steps (the
    debug setting that makes the TMA-staged face kernels issue no copies)
    ends the call with GRIM_ETIMEOUT after every issued copy has finished;
    with the setting cleared and the state set again the handle steps as a
    fresh one does."""
    import torch
    from grim_b200 import _lib
    from grim_b200.timestepper import timeStepper
    cfg = PR.fast_mode_config(N=64)
    P = PR.fast_mode_prims(cfg)
    ts, ref = timeStepper(cfg), timeStepper(cfg)
    for h in (ts, ref):
        h.setFaceVariant(0, 2)  # the TMA-staged X1 kernel
        h.setFixedDt(True)
        h.primOld.setVars(P)
    t0, dt0 = ts.time, ts.dt
    inp = torch.from_numpy(np.ascontiguousarray(P)).pin_memory()
    out = torch.zeros_like(inp).pin_memory()
    ts.setDebug(_lib.DEBUG_SKIP_BULK_COPIES, 1)
    with pytest.raises(_lib.GrimError) as err:
        ts.timeStepsHost([inp.data_ptr()] * 3, [out.data_ptr()] * 3)
    assert err.value.status == _lib.GRIM_ETIMEOUT
    ts.setDebug(_lib.DEBUG_SKIP_BULK_COPIES, 0)
    ts.synchronize()
    for h in (ts, ref):
        h.primOld.setVars(P)
        h.setTime(t0, dt0)
    ts.timeStepsHost([inp.data_ptr(), None], [None, out.data_ptr()])
    ref.timeSteps(2)
    assert np.array_equal(out.numpy(), ref.primOld.getVars())
