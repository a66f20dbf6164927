"""Benchmark of the implicit GRMHD timestep: zone-cycles/s.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
                    [--workload torus|orszag_tang|fast_mode|emhd_stratified|batch]

One JSON line on rank 0.  ``value`` is the zone-cycles/s of the product's
fast Newton form (forward-tangent Jacobian, FP32 Jacobian/solve refined by
the FP64 residual, per-zone convergence) with inputs resident in HBM;
``fd64`` is the same workload through the plain FP64 finite-difference
path (the reference's method) at the same Newton tolerance; ``e2e`` adds
the host<->device copies of the primitives every step through the C ABI
(grim_time_steps_host on arrays of the interior zones: each step's copies
overlap the neighbouring steps; the same call on whole arrays with ghosts
and the same steps as separate grim_set_prims / grim_time_step /
grim_get_prims calls are reported beside it as ``ghosted`` and
``sequential``).
Each timed step is bracketed by CUDA events on the stepper's stream; the
L2 is flushed between timed steps (a 256 MB write) and the flush is not
timed.  With --impl reference the CPU oracle (a C++ restatement of the
reference's algorithm) is timed on the host cores instead.
Multi-GPU: one independent replica per rank ("replicas only"), max over
ranks of the device time.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

from grim_b200 import config as C  # noqa: E402
from grim_b200 import problems as PR  # noqa: E402

METRIC = "zone-cycles/s per implicit step: plain FP64 FD-Jac vs tangent/mixed form, same tol"
RTOL = 1e-10
# absolute floor of the squared zone residual: |R| <= 1e-12, above the roundoff
# of the residual for these workloads (|U|/dt' ~ 1e3, eps ~ 1e-16)
ATOL = 1e-24
# rounding floor of the zone test, in ulps of the residual's largest term
# (|U|/dt' at the solution: max over the conserved rows of
# |divF + S - U_old/dt'|): relative 1e-10
# of the first residual lies below the rounding of an FP64 residual in about
# 0.1% of the torus zones (their first residual is 1e-6..1e-9 of |U|/dt'),
# which then never test converged in any Newton form
ULPS = 8.


def workload(name, grid=None):
    """(config, prims, description) of a named workload; grid "N1xN2xN3"
    (torus) or "N" (2D workloads) overrides the size, for small profiler
    captures of the same set-up"""
    dims = [int(x) for x in grid.split("x")] if grid else None
    if dims and name != "torus":
        n = dims[0]
        if name == "orszag_tang":
            cfg = PR.orszag_tang_config(N=n, nonlinearsolve_atol=ATOL, nonlinearsolve_rtol=RTOL, nonlinearsolve_ulps=ULPS, maxNonLinearIter=4)
            return cfg, PR.orszag_tang_prims(cfg), "2D Orszag-Tang %dx%d" % (n, n)
        if name == "fast_mode":
            cfg = PR.fast_mode_config(N=n, nonlinearsolve_atol=ATOL, nonlinearsolve_rtol=RTOL, nonlinearsolve_ulps=ULPS, maxNonLinearIter=4)
            return cfg, PR.fast_mode_prims(cfg), "2D fast mode %dx%d" % (n, n)
        if name == "emhd_stratified":
            cfg = PR.emhd_stratified_config(N=n, nonlinearsolve_atol=ATOL, nonlinearsolve_rtol=RTOL, nonlinearsolve_ulps=ULPS,
                                            maxNonLinearIter=4)
            return cfg, PR.emhd_stratified_prims(cfg), "2D EMHD %dx%d" % (n, n)
    if name == "orszag_tang":
        cfg = PR.orszag_tang_config(N=512, nonlinearsolve_atol=ATOL, nonlinearsolve_rtol=RTOL, nonlinearsolve_ulps=ULPS,
                                    maxNonLinearIter=4)
        return cfg, PR.orszag_tang_prims(cfg), "2D Orszag-Tang 512x512, Minkowski, WENO5, HLL, flux-CT, ideal MHD (dof 8)"
    if name == "fast_mode":
        cfg = PR.fast_mode_config(N=128, nonlinearsolve_atol=ATOL, nonlinearsolve_rtol=RTOL, nonlinearsolve_ulps=ULPS, maxNonLinearIter=4)
        return cfg, PR.fast_mode_prims(cfg), "2D fast mode 128x128, Minkowski, minmod, LLF, flux-CT"
    if name == "emhd_stratified":
        cfg = PR.emhd_stratified_config(N=256, nonlinearsolve_atol=ATOL, nonlinearsolve_rtol=RTOL, nonlinearsolve_ulps=ULPS,
                                        maxNonLinearIter=4)
        return cfg, PR.emhd_stratified_prims(cfg), "2D EMHD 256x256 (dof 10), MP5, HLL, tau(y) closure"
    if name == "torus":
        from grim_b200.problems import torus as T
        n1, n2, n3 = dims if dims else (256, 128, 64)
        cfg = T.torus_config(N1=n1, N2=n2, N3=n3, nonlinearsolve_atol=ATOL, nonlinearsolve_rtol=RTOL, nonlinearsolve_ulps=ULPS)
        return cfg, None, ("3D Fishbone-Moncrief torus in MKS, a=0.9375, r_in=6, r_max=12, %dx%dx%d, "
                           "PPM, LLF, flux-CT, floors, ideal MHD (dof 8)" % (n1, n2, n3))
    raise SystemExit("unknown workload %s" % name)


def torus_state(cfg, ts):
    """Initial conditions of the torus from the stepper's own geometry."""
    from grim_b200.problems import torus as T
    geo = ts.getGeometry(C.CENTER)
    P, _ = T.torus_prims(cfg, geo)
    return P


def cpu_sample_config(name, cfg):
    """The workload of the one-core CPU figure: the full grid, except the
    torus, whose one-core run is bounded to a 64x32x16 sample of the same
    set-up (a full 256x128x64 step takes minutes on one core)."""
    if name == "torus":
        from grim_b200.problems import torus as T
        return T.torus_config(N1=64, N2=32, N3=16, nonlinearsolve_atol=ATOL, nonlinearsolve_rtol=RTOL, nonlinearsolve_ulps=ULPS)
    return cfg


def workload_config(name, desc, cfg):
    """The `config` of a bench line: what the workload is, the same for the
    GPU arm and the CPU reference arm (how each arm computes it goes under
    `method`)."""
    return {"workload": name, "description": desc, "zones": cfg["N1"] * cfg["N2"] * cfg["N3"],
            "rel_residual_tol": RTOL, "abs_residual_floor": ATOL, "maxNonLinearIter": cfg["maxNonLinearIter"],
            "l2": "working set above the L2 size in both arms; the GPU arm also flushes L2 between timed steps "
                  "(256 MB write, untimed)"}


class Clocks:
    """nvidia-smi clock/throttle sampling during the timed region."""

    def __init__(self, index):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._p = None

    def start(self):
        q = "clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown," \
            "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown," \
            "clocks_event_reasons.sw_power_cap"
        try:
            self._p = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + q,
                                        "--format=csv,noheader,nounits", "-lms", "100"],
                                       stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self._p = None
            return

        def rd():
            for line in self._p.stdout:
                self.samples.append([x.strip() for x in line.split(",")])
        self._t = threading.Thread(target=rd, daemon=True)
        self._t.start()
        # the sampler's first line comes before the timed region: wait for it
        # (nvidia-smi takes a while to start) and leave it out
        t0 = time.time()
        while not self.samples and time.time() - t0 < 5.0 and self._p.poll() is None:
            time.sleep(0.01)
        self._n0 = len(self.samples)

    def stop(self):
        n0 = getattr(self, "_n0", 0)
        if self._p:
            # a timed region shorter than the sampling period: take the line
            # that follows it
            t0 = time.time()
            while len(self.samples) <= n0 and time.time() - t0 < 1.0 and self._p.poll() is None:
                time.sleep(0.005)
            self._p.terminate()
            try:
                self._p.wait(timeout=5)
            except Exception:
                self._p.kill()
        got = self.samples[n0:]
        sm = [float(s[0]) for s in got if len(s) >= 7 and s[0].replace('.', '').isdigit()]
        mx = [float(s[1]) for s in got if len(s) >= 7 and s[1].replace('.', '').isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for s in got:
            if len(s) >= 7:
                for n, v in zip(names, s[3:7]):
                    if v.lower().startswith("active"):
                        reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_reference(cfg, P, seconds=15.0, threads=None):
    """Time the CPU oracle on the workload's grid: set-up and one warm-up
    step untimed, then whole steps until `seconds` have passed (at least
    one, at most 50).  Returns (zone-cycles/s, threads, sample text)."""
    from oracle import oracle as O
    n = threads or os.cpu_count()
    O.set_threads(n)
    t_setup = time.perf_counter()
    o = O.Oracle(cfg)
    if P is None:  # torus: initial conditions from the oracle's geometry
        from grim_b200.problems import torus as T
        P, _ = T.torus_prims(cfg, o.geometry(C.CENTER))
        o.set_prims(P)
        o.problem_init()
    else:
        o.set_prims(P)
    o.time_step(1)  # warm-up (page faults, first dt)
    t_setup = time.perf_counter() - t_setup
    steps, t0 = 0, time.perf_counter()
    while True:
        o.time_step(1)
        steps += 1
        el = time.perf_counter() - t0
        if el >= seconds or steps >= 50:
            break
    zones = cfg["N1"] * cfg["N2"] * cfg["N3"]
    return zones * steps / el, n, ("%d timed step(s) of the full %dx%dx%d grid, %.1f s, after %.1f s of set-up "
                                   "and 1 warm-up step (untimed)" % (steps, cfg["N1"], cfg["N2"], cfg["N3"], el, t_setup))


def profile_path(ts, steps, flush):
    """Per kernel group device time (CUDA events on the stepper's stream
    around each launch, graph off, L2 flushed between steps), the Newton
    iteration histogram of every profiled step and the algorithmic flop
    counts of one zone."""
    import torch
    stream = torch.cuda.ExternalStream(ts.stream())
    tot = {}
    hist = [[0] * 16, [0] * 16]
    for _ in range(steps):
        with torch.cuda.stream(stream):
            flush.fill_(2.0)
        p = ts.profileSteps(1)
        for g, (ms, n) in p.items():
            a = tot.setdefault(g, [0.0, 0])
            a[0] += ms
            a[1] += n
        h = ts.newtonHistogram()
        for st in range(2):
            for k in range(16):
                hist[st][k] += h[st][k]
    return {"steps": steps, "groups": tot, "hist": hist, "flops": ts.countFlops(), "nf": ts.numFluidVars, "dof": ts.dof,
            "maxIter": ts.cfg["maxNonLinearIter"], "mode": ts.cfg["newtonMode"]}


def stencil_bytes_per_zone(cfg, dof, nf):
    """Algorithmic HBM bytes of one zone's stencil (all face kernels + the
    epilogue of one stage): the primitives in, the stage constants and the
    new B out, and the geometry words the reconstruction/Riemann/source
    terms need (22 per face location x 3, 40 Christoffels).  The geometry
    is stored once per (i, j) plane, so its words are shared by the N3 + 2
    ghost zones along X3; none for Minkowski, whose metric is a
    compile-time constant."""
    G = 0. if cfg["metric"] == C.MINKOWSKI else (3 * 22 + 40) / float(cfg["N3"] + 2 * cfg["numGhost"] * (cfg["dim"] > 2))
    return 8 * (dof + nf + 3 + G)


def newton_flops(prof):
    """(fp64, fp32) algorithmic flops of the profiled steps' Newton kernels.
    Fast form, per zone: one residual at entry, then per iteration one
    tangent pass and pivoted solve (FP32 in the mixed form) and one
    line-search residual, which is also the next convergence test.  FD form
    (reference method), per zone and iteration: residual + nf FD columns
    (nf + 1 residuals), an FP64 solve and one line-search residual."""
    f, nf = prof["flops"], prof["nf"]
    zone_its = sum(k * n for st in prof["hist"] for k, n in enumerate(st))
    zones = sum(n for st in prof["hist"] for n in st)
    if prof["mode"] == C.NEWTON_PARITY_FD64:
        return None
    if prof["mode"] == C.NEWTON_MIXED32:
        f64 = zones * f["residual64"] + zone_its * f["residual64"]
        f32 = zone_its * (f["tangent32"] + f["solve32"])
    else:
        f64 = zones * f["residual64"] + zone_its * (f["residual64"] + f["tangent64"] + f["solve64"])
        f32 = 0.0
    return f64, f32


def rooflines(cfg, prof, prof_fd, device):
    """The roofline object of the dominant kernel group and the same figures
    for the other groups."""
    from grim_b200.timestepper import measurePeaks
    fp64_peak, fp32_peak, hbm_local = measurePeaks(device)
    with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
        hbm_peak = float(json.load(fh)["hbm_gbs"])
    zones = cfg["N1"] * cfg["N2"] * cfg["N3"]
    steps = prof["steps"]
    g = prof["groups"]
    stencil_ms = sum(g[k][0] for k in ("faces_x1", "faces_x2", "faces_x3", "epilogue", "emhd_prepass"))
    stencil_launches = g["epilogue"][1]  # one epilogue per stage
    B = stencil_bytes_per_zone(cfg, prof["dof"], prof["nf"])
    fz = prof["flops"]
    # counted FP64 flops of one zone's stencil stage: per direction one
    # reconstruction and (about) one face, plus the epilogue's centre work
    F = cfg["dim"] * (fz["recon_zone_dir"] + fz["riemann_face"]) + fz["epilogue_zone"]
    t_st = stencil_ms * 1e-3 / stencil_launches  # s per stage
    st_gbs = B * zones / t_st / 1e9
    st_tf = F * zones / t_st / 1e12
    t_hbm, t_fp = B * zones / (hbm_peak * 1e9), F * zones / (fp64_peak * 1e12)
    f64, f32 = newton_flops(prof)
    newton_ms, newton_launches = g["newton"]
    n64 = f64 / (newton_ms * 1e-3) / 1e12
    n32 = f32 / (newton_ms * 1e-3) / 1e12
    pipe_frac = (n64 / fp64_peak) + (n32 / fp32_peak)
    traffic, traffic_src = _ncu_traffic(cfg)
    newton = {"bound": "fp64", "achieved": n64, "peak": fp64_peak, "unit": "TFLOP/s", "frac": n64 / fp64_peak,
              "fp32_achieved": n32, "fp32_peak": fp32_peak, "fp32_frac": n32 / fp32_peak,
              "pipe_time_frac": pipe_frac,
              "traffic": traffic.get("newton"), "traffic_source": traffic_src,
              "kernel": "newton (one launch per stage)", "ms_per_launch": newton_ms / newton_launches,
              "flops_per_zone": prof["flops"],
              "peak_source": "measured: FMA-chain self-test of this GPU (grim_measure_peaks)"}
    common = {"traffic": traffic.get("stencil"), "traffic_source": traffic_src,
              "kernel": "stencil (face fluxes x%d + epilogue, per stage)" % cfg["dim"],
              "ms_per_launch": t_st * 1e3, "bytes_per_zone": B, "flops_per_zone": F,
              "hbm_achieved_gbs": st_gbs, "hbm_peak_gbs": hbm_peak, "hbm_frac": st_gbs / hbm_peak,
              "fp64_achieved_tflops": st_tf, "fp64_peak_tflops": fp64_peak, "fp64_frac": st_tf / fp64_peak,
              "peak_source": "HBM of measured (MEASURED_PEAKS.json hbm_gbs); FP64 measured (grim_measure_peaks)",
              "hbm_selftest_gbs": hbm_local}
    if t_fp >= t_hbm:
        stencil = dict({"bound": "fp64", "achieved": st_tf, "peak": fp64_peak, "unit": "TFLOP/s",
                        "frac": st_tf / fp64_peak}, **common)
    else:
        stencil = dict({"bound": "hbm", "achieved": st_gbs, "peak": hbm_peak, "unit": "GB/s",
                        "frac": st_gbs / hbm_peak}, **common)
    # whole step against sum over the stencil and Newton kernels of
    # max(bytes / BW, flops / peak) (the other kernels are not in the bound)
    t_newton_bound = f64 / (fp64_peak * 1e12) + f32 / (fp32_peak * 1e12)  # all profiled steps
    t_bound = steps * 2 * max(t_hbm, t_fp) + t_newton_bound
    step_bound = {"zone_cycles_per_s": zones * steps / t_bound,
                  "achieved_profiled": zones * steps / (sum(v[0] for v in g.values()) * 1e-3)}
    step_bound["frac"] = step_bound["achieved_profiled"] / step_bound["zone_cycles_per_s"]
    total = sum(v[0] for v in g.values())
    shares = {k: round(v[0] / total, 4) for k, v in g.items() if v[0] > 0}
    dominant = newton if g["newton"][0] >= stencil_ms else stencil
    out = {"roofline": dict(dominant), "roofline_other": stencil if dominant is newton else newton,
           "step_roofline": step_bound, "kernel_shares": shares, "profiled_ms_per_step": total / steps}
    if prof_fd is not None:
        gf = prof_fd["groups"]
        tf = sum(v[0] for v in gf.values())
        out["fd64_kernel_shares"] = {k: round(v[0] / tf, 4) for k, v in gf.items() if v[0] > 0}
    return out


# the sources that define the step's kernels: a DRAM capture describes the
# kernels these files built
KERNEL_SOURCES = ("kernels.cuh", "physics.cuh", "recon.cuh", "stage.cuh", "common.cuh", "torus.cuh",
                  "launch.h", "kernels_fast.cu", "faces_fast.cu")


def kernel_sources_sha16():
    """Fingerprint of the kernel sources' code: comments and blank space
    removed, so that only a change of code makes a capture stale."""
    import hashlib
    import re
    h = hashlib.sha256()
    for n in KERNEL_SOURCES:
        with open(os.path.join(ROOT, "grim_b200", "csrc", n)) as fh:
            t = fh.read()
        t = re.sub(r"/\*.*?\*/", " ", t, flags=re.S)
        t = re.sub(r"//[^\n]*", " ", t)
        t = " ".join(t.split())
        h.update(n.encode() + b"\0" + t.encode())
    return h.hexdigest()[:16]


def _ncu_traffic(cfg):
    """DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum)
    of the workload's kernel groups from the committed ncu summary, when
    one exists for this grid and was taken on the current kernel sources
    (else {} and the line's traffic is null), and what was found."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(path) as fh:
            table = json.load(fh)
    except (OSError, ValueError):
        return {}, "no profiles/traffic.json"
    key = "%dx%dx%d" % (cfg["N1"], cfg["N2"], cfg["N3"])
    entry = table.get(key)
    if entry is None:
        return {}, "no capture of the %s grid" % key
    if entry.get("sources_sha16") != kernel_sources_sha16():
        return {}, "stale: the kernel sources changed since the capture of the %s grid" % key
    return entry, "profiles/traffic.json, %s grid, captured on these kernel sources (%s)" % (
        key, entry["sources_sha16"])


def batch_problems(seed=5, count=16):
    """The ragged batch of the adjoint / batching workload at the bench's
    Newton tolerances (grim_b200.problems.ragged_batch)."""
    return PR.ragged_batch(seed=seed, count=count, nonlinearsolve_atol=ATOL, nonlinearsolve_rtol=RTOL,
                           nonlinearsolve_ulps=ULPS, maxNonLinearIter=4)


def run_batch(args, local_rank):
    """The ragged-batch workload: value = all problems' zone-cycles/s stepped
    as one batch (one graph per step, one compacted Newton launch per
    iteration for all problems); beside it the same problems as separate
    steppers (fast form and FD64 form) and the adjoint of the largest."""
    import torch
    from grim_b200.timestepper import Batch, timeStepper
    torch.cuda.set_device(local_rank)
    probs = batch_problems()
    zones = sum(cfg["N1"] * cfg["N2"] for cfg, _ in probs)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def timed(run, sync, stream_ptr, steps):
        stream = torch.cuda.ExternalStream(stream_ptr)
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        torch.cuda.synchronize()
        for a, b in evs:
            with torch.cuda.stream(stream):
                flush.fill_(1.0)
                a.record(stream)
            run()
            b.record(stream)
        sync()
        torch.cuda.synchronize()
        return sum(a.elapsed_time(b) for a, b in evs)

    clocks = Clocks(local_rank)
    B = Batch([cfg for cfg, _ in probs])
    B.setNewtonMode(C.NEWTON_MIXED32, RTOL)
    for (cfg, P), ts in zip(probs, B.problems):
        ts.primOld.setVars(P)
    B.enableGraph(True)
    B.timeSteps(args.warmup)
    B.synchronize()
    clocks.start()
    ms_b = timed(lambda: B.timeSteps(1), B.synchronize, B.stream(), args.steps)
    clocks_info = clocks.stop()
    unconv = sum(sum(ts.stats()["unconverged"]) for ts in B.problems)

    def separate(mode):
        sts = []
        for cfg, P in probs:
            ts = timeStepper(cfg)
            ts.setNewtonMode(mode, 2, RTOL)
            ts.primOld.setVars(P)
            ts.enableGraph(True)
            for _ in range(args.warmup):
                ts.timeStep()
            sts.append(ts)
        for ts in sts:
            ts.synchronize()
        # steps issued problem after problem; each stepper has its own stream
        ms = 0.0
        for ts in sts:
            ms += timed(ts.timeStep, ts.synchronize, ts.stream(), max(2, args.steps // 2)) / max(2, args.steps // 2)
        return ms, sts

    ms_sep, _ = separate(C.NEWTON_MIXED32)
    ms_fd, _ = separate(C.NEWTON_PARITY_FD64)
    # adjoint of the largest problem: 20 steps, checkpoints every 10
    cfg, P = max(probs, key=lambda p: p[0]["N1"])
    ts = timeStepper(cfg)
    ts.setNewtonMode(C.NEWTON_TANGENT64, 1, 0.0)
    ts.primOld.setVars(P)
    ts.primOld.communicate()
    ts.setFixedDt(True)
    # one untimed forward / backward pair of the same shape first: the
    # adjoint's checkpoint and segment buffers are allocated and its kernels
    # loaded on the first call
    time0, dt0 = ts.time, ts.dt
    ts.adjointForward(20, 10)
    ts.adjointBackward(ts.primOld.getVars())
    ts.setTime(time0, dt0)
    ts.primOld.setVars(P)
    ts.primOld.communicate()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ts.adjointForward(20, 10)
    lam = ts.primOld.getVars() - np.array([1.0, 2.0, 0, 0, 0, 0.1, 0.3, 0])[:, None, None, None]
    t1 = time.perf_counter()
    ts.adjointBackward(lam)
    t2 = time.perf_counter()
    value = zones * args.steps / (ms_b / 1e3)
    return {
        "metric": METRIC, "value": value, "unit": "zone-cycles/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_b / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64 residual / f32 Jacobian+solve",
        "data": "synthetic (seeded linear modes)",
        "config": {"workload": "batch", "description": "16 independent 2D ideal linear-mode problems, N = 64..512, "
                   "minmod/LLF/flux-CT, one batch", "zones": zones,
                   "sizes": [cfg["N1"] for cfg, _ in probs], "rel_residual_tol": RTOL,
                   "l2": "flushed between timed steps (256 MB write, untimed)", "cuda_graph": True},
        "unconverged": unconv,
        "separate_fast": {"value": zones / (ms_sep / 1e3), "ms_per_step": ms_sep},
        "fd64": {"value": zones / (ms_fd / 1e3), "ms_per_step": ms_fd},
        "speedup_vs_fd64": value / (zones / (ms_fd / 1e3)),
        "batch_vs_separate": value / (zones / (ms_sep / 1e3)),
        "adjoint": {"problem": "%dx%d" % (cfg["N1"], cfg["N2"]), "steps": 20, "checkpoint_every": 10,
                    "forward_s": t1 - t0, "backward_s": t2 - t1,
                    "backward_zone_steps_per_s": cfg["N1"] * cfg["N2"] * 20 / (t2 - t1)},
        "clocks": clocks_info,
    }


def _free_port():
    import socket
    sk = socket.socket()
    sk.bind(("127.0.0.1", 0))
    port = sk.getsockname()[1]
    sk.close()
    return port


def run_decomposed(args, rank, world, local_rank):
    """The workload's grid split into X3 slabs over the ranks (one GPU
    each; NCCL halos and reductions between the library's step segments):
    total work fixed as N grows.  Fast Newton form."""
    import torch
    torch.cuda.set_device(local_rank)
    from grim_b200.slab import SlabTimeStepper
    from grim_b200.timestepper import timeStepper
    cfg, P, desc = workload(args.workload, args.grid)
    cfg = dict(cfg, newtonMode=C.NEWTON_MIXED32, perZoneConvergence=args.per_zone, nonlinearsolve_rtol=RTOL, nonlinearsolve_ulps=ULPS)
    if P is None:
        P = torus_state(cfg, timeStepper(cfg, device=local_rank))
    zones = cfg["N1"] * cfg["N2"] * cfg["N3"]
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    sl = SlabTimeStepper(cfg, device=local_rank)
    sl.setGlobalPrims(P)
    sl.ts.problemInit()
    tuned = {str(d): v for d, (v, _) in sl.ts.autotune().items()}
    stream = sl.stream
    for _ in range(args.warmup):
        sl.timeStep()
    sl.synchronize()
    torch.distributed.barrier()
    clocks = Clocks(local_rank)
    clocks.start()
    ms = 0.
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            flush.fill_(1.0)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
        sl.timeStep()
        b.record(stream)
        torch.cuda.synchronize()
        ms += a.elapsed_time(b)
    clocks_info = clocks.stop()
    torch.distributed.barrier()
    # e2e: this rank's slab in from pinned host memory, the step, the slab back
    import ctypes
    from grim_b200 import _lib
    host_in = torch.from_numpy(np.ascontiguousarray(sl.ts.primOld.getVars())).pin_memory()
    host_out = torch.empty_like(host_in).pin_memory()
    L = _lib.lib()
    e2e_steps = max(3, args.steps // 2)
    torch.distributed.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        _lib.check(L.grim_set_prims(sl.ts._h, _lib.PRIM_OLD, ctypes.c_void_p(host_in.data_ptr()), _lib.HOST))
        sl.timeStep()
        _lib.check(L.grim_get_prims(sl.ts._h, _lib.PRIM_OLD, ctypes.c_void_p(host_out.data_ptr()), _lib.HOST))
    e2e_s = time.perf_counter() - t0
    t = torch.tensor([ms, e2e_s], dtype=torch.float64, device="cuda")
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    ms, e2e_s = [float(x) for x in t.tolist()]
    return {
        "metric": METRIC, "value": zones * args.steps / (ms / 1e3), "unit": "zone-cycles/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "f64 residual / f32 Jacobian+solve",
        "data": "synthetic (seeded initial conditions of the named workload)",
        "config": workload_config(args.workload, desc, cfg),
        "method": {"parallelism": "X3 slabs of %d planes on %d GPUs (NCCL halos)" % (cfg["N3"] // world, world),
                   "face_kernel_variants": tuned},
        "e2e": {"value": zones * e2e_steps / e2e_s, "unit": "zone-cycles/s",
                "h2d_bytes_per_step": host_in.numel() * 8 * world, "d2h_bytes_per_step": host_in.numel() * 8 * world},
        "gpu_launches": None, "clocks": clocks_info, "roofline": None, "cpu_baseline": None,
    }


def run_gpu(args, rank, world, local_rank):
    import torch
    torch.cuda.set_device(local_rank)
    from grim_b200.timestepper import timeStepper
    cfg, P, desc = workload(args.workload, args.grid)
    zones = cfg["N1"] * cfg["N2"] * cfg["N3"]
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    state = {"P": P}

    def time_path(mode, graph):
        ts = timeStepper(cfg, device=local_rank)
        ts.setNewtonMode(mode, args.per_zone, RTOL)
        if state["P"] is None:
            state["P"] = torus_state(cfg, ts)
        ts.primOld.setVars(state["P"])
        ts.problemInit()
        if args.variants:
            for d, v in enumerate(int(x) for x in args.variants.split(",")):
                ts.setFaceVariant(d, v)
            state.setdefault("tuned", {})[mode] = "forced " + args.variants
        else:
            state.setdefault("tuned", {})[mode] = {str(d): v for d, (v, _) in ts.autotune().items()}
        if graph:
            ts.enableGraph(True)
        stream = torch.cuda.ExternalStream(ts.stream())
        for _ in range(args.warmup):
            ts.timeStep()
        ts.synchronize()
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(args.steps)]
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        for a, b in evs:
            with torch.cuda.stream(stream):
                flush.fill_(1.0)
                a.record(stream)
            ts.timeStep()
            b.record(stream)
        torch.cuda.synchronize()
        ms = sum(a.elapsed_time(b) for a, b in evs)
        st = ts.stats()
        return ts, ms, st

    clocks = Clocks(local_rank)
    clocks.start()
    ts_fast, ms_fast, st_fast = time_path(C.NEWTON_MIXED32, True)
    clocks_info = clocks.stop()
    prof_fast = profile_path(ts_fast, args.steps, flush)
    if args.no_fd:
        ms_fd, st_fd, prof_fd = float("nan"), {"newtonIters": None, "unconverged": None}, None
        ms_fdf, st_fdf = float("nan"), {"newtonIters": None, "unconverged": None}
    else:
        ts_fd, ms_fd, st_fd = time_path(C.NEWTON_PARITY_FD64, True)
        prof_fd = profile_path(ts_fd, max(3, args.steps // 4), flush)
        del ts_fd
        # the same FD Newton built like the fast form (FMA arithmetic, the
        # fast stencil, finish and guess kernels): the like-for-like baseline
        ts_fdf, ms_fdf, st_fdf = time_path(C.NEWTON_FD64_FAST, True)
        del ts_fdf

    # e2e: the C-ABI call with host buffers, copies inside the timed region
    import ctypes
    from grim_b200 import _lib
    dof = ts_fast.dof
    host_in = torch.from_numpy(np.ascontiguousarray(state["P"])).pin_memory()
    host_out = torch.empty_like(host_in).pin_memory()
    L = _lib.lib()
    e2e_steps = max(3, args.steps)
    ts_fast.synchronize()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        _lib.check(L.grim_set_prims(ts_fast._h, _lib.PRIM_OLD, ctypes.c_void_p(host_in.data_ptr()), _lib.HOST))
        _lib.check(L.grim_time_step(ts_fast._h, None, None))
        _lib.check(L.grim_get_prims(ts_fast._h, _lib.PRIM_OLD, ctypes.c_void_p(host_out.data_ptr()), _lib.HOST))
    e2e_seq_s = time.perf_counter() - t0
    # the same steps through grim_time_steps_host: every step's state in
    # from pinned host memory and its result back, the copies of one step
    # overlapped with the neighbouring steps (one untimed call first
    # allocates the staging buffers); whole arrays with ghosts, then the
    # interior zones only (the step's boundary pass refills the ghosts)
    host_outs = [host_out, torch.empty_like(host_in).pin_memory()]
    ins = [host_in.data_ptr()] * e2e_steps
    outs = [host_outs[k & 1].data_ptr() for k in range(e2e_steps)]
    ts_fast.timeStepsHost(ins[:2], outs[:2])
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ts_fast.timeStepsHost(ins, outs)
    e2e_ghosted_s = time.perf_counter() - t0
    sl = (slice(None),) + tuple(C.interior_slices(cfg))
    inner_in = torch.from_numpy(np.ascontiguousarray(state["P"][sl])).pin_memory()
    inner_outs = [torch.empty_like(inner_in).pin_memory() for _ in range(2)]
    ins = [inner_in.data_ptr()] * e2e_steps
    outs = [inner_outs[k & 1].data_ptr() for k in range(e2e_steps)]
    ts_fast.timeStepsHost(ins[:2], outs[:2], interior=True)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ts_fast.timeStepsHost(ins, outs, interior=True)
    e2e_s = time.perf_counter() - t0
    e2e_bytes = inner_in.numel() * 8
    e2e_ghosted_bytes = host_in.numel() * 8
    side = torus_side_costs(ts_fast, cfg) if args.workload == "torus" else None

    # max over ranks of the device time
    t = torch.tensor([ms_fast, ms_fd, ms_fdf, e2e_s, e2e_seq_s, e2e_ghosted_s], dtype=torch.float64, device="cuda")
    if world > 1:
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    ms_fast, ms_fd, ms_fdf, e2e_s, e2e_seq_s, e2e_ghosted_s = [float(x) for x in t.tolist()]
    value = world * zones * args.steps / (ms_fast / 1e3)
    fd = world * zones * args.steps / (ms_fd / 1e3) if ms_fd == ms_fd else None
    fdf = world * zones * args.steps / (ms_fdf / 1e3) if ms_fdf == ms_fdf else None
    out = {
        "metric": METRIC,
        "value": value,
        "unit": "zone-cycles/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_fast / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64 residual / f32 Jacobian+solve",
        "data": "synthetic (seeded initial conditions of the named workload)",
        "config": workload_config(args.workload, desc, cfg),
        "method": {"newton": "tangent Jacobian, FP32 solve, FP64 residual, per-zone convergence",
                   "rounding_floor_ulps": ULPS,
                   "parallelism": "replicas" if world > 1 else "single GPU", "cuda_graph": True,
                   "face_kernel_variants": state.get("tuned", {})},
        "fd64": {"value": fd, "ms_per_step": ms_fd / args.steps, "newton_iters": st_fd["newtonIters"],
                 "unconverged": st_fd["unconverged"],
                 "form": "parity path: FD Jacobian Newton, global break, every kernel without FMA contraction"},
        "speedup_vs_fd64": value / fd if fd else None,
        "fd64_fast": {"value": fdf, "ms_per_step": ms_fdf / args.steps, "newton_iters": st_fdf["newtonIters"],
                      "unconverged": st_fdf["unconverged"],
                      "form": "FD Jacobian Newton, global break, in the fast form's arithmetic and kernels"},
        "speedup_vs_fd64_fast": value / fdf if fdf else None,
        "newton_iters": st_fast["newtonIters"],
        "unconverged": st_fast["unconverged"],
        # zones per Newton iteration count (index = updates taken), summed
        # over the profiled steps, per stage
        "newton_iteration_histogram": {
            "fast": {"half": prof_fast["hist"][0][:cfg["maxNonLinearIter"] + 1],
                     "full": prof_fast["hist"][1][:cfg["maxNonLinearIter"] + 1]},
            "fd64": None if prof_fd is None else {"half": prof_fd["hist"][0][:cfg["maxNonLinearIter"] + 1],
                                                  "full": prof_fd["hist"][1][:cfg["maxNonLinearIter"] + 1]}},
        "e2e": {"value": world * zones * e2e_steps / e2e_s, "unit": "zone-cycles/s",
                "h2d_bytes_per_step": e2e_bytes, "d2h_bytes_per_step": e2e_bytes,
                "call": "grim_time_steps_host, interior zones (pinned buffers; copies overlapped with the steps)",
                "ghosted": {"value": world * zones * e2e_steps / e2e_ghosted_s,
                            "h2d_bytes_per_step": e2e_ghosted_bytes, "d2h_bytes_per_step": e2e_ghosted_bytes,
                            "call": "grim_time_steps_host, whole arrays with ghosts"},
                "sequential": {"value": world * zones * e2e_steps / e2e_seq_s,
                               "h2d_bytes_per_step": e2e_ghosted_bytes, "d2h_bytes_per_step": e2e_ghosted_bytes,
                               "call": "grim_set_prims, grim_time_step, grim_get_prims per step"}},
        "gpu_launches": int(st_fast["kernelLaunches"]) * args.steps,
        "clocks": clocks_info,
    }
    if side is not None:
        out["torus_side"] = side
    out.update(rooflines(cfg, prof_fast, prof_fd, local_rank))
    return out, cfg, state["P"]


def torus_side_costs(ts, cfg):
    """Beside the step: one record of the torus observers (the element and
    the integrands per interior zone, fixed-order partials; two launches and
    a 9-value read-back per call, timed by the wall clock around the
    synchronous call), and a checkpoint round trip of primOld (grid::dump
    then grid::load as a PETSc binary Vec: device copy, natural-order
    reshuffle, big-endian file I/O)."""
    import tempfile
    zones = cfg["N1"] * cfg["N2"] * cfg["N3"]
    for _ in range(3):
        ts.torusObservers()
    n = 20
    t0 = time.perf_counter()
    for _ in range(n):
        ts.torusObservers()
    obs_s = (time.perf_counter() - t0) / n
    obs_bytes = zones * ts.dof * 8  # the primitives each record reads
    with tempfile.TemporaryDirectory() as d:
        f = os.path.join(d, "primOld.bin")
        t0 = time.perf_counter()
        ts.dump(f)
        t1 = time.perf_counter()
        ts.load(f)
        t2 = time.perf_counter()
        size = os.path.getsize(f)
    return {"observers": {"ms_per_record": obs_s * 1e3, "primitive_bytes": obs_bytes,
                          "gbs": obs_bytes / obs_s / 1e9},
            "checkpoint": {"file_bytes": size, "dump_s": t1 - t0, "load_s": t2 - t1}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="grim_b200")
    ap.add_argument("--workload", default="torus")
    ap.add_argument("--grid", default=None, help="override the workload size: N1xN2xN3 (torus) or N")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-fd", action="store_true", help="skip the FD64 comparison path (profiler captures)")
    ap.add_argument("--variants", default=None,
                    help="face-kernel launch variants per direction, e.g. 1,5,5, instead of autotuning")
    ap.add_argument("--decomp", default=None, choices=[None, "x3"],
                    help="x3: split the grid into X3 slabs over the GPUs (strong scaling) instead of replicas")
    ap.add_argument("--per-zone", type=int, default=1,
                    help="fast Newton: 1 = per-zone loop in one kernel, 2 = compacted worklists")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return
        cfg, P, desc = workload(args.workload, args.grid)
        # the whole workload grid, whole steps for about 20 s after an
        # untimed set-up and warm-up step
        v, n, sample = cpu_reference(cfg, P, seconds=20.0)
        print(json.dumps({
            "impl": "reference", "metric": METRIC, "value": v, "unit": "zone-cycles/s", "n_gpus": 0,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded initial conditions of the named workload)",
            "config": workload_config(args.workload, desc, cfg),
            "method": {"newton": "FD Jacobian (reference method), FP64, global break",
                       "runs_on": "host cores: the CPU restatement of the reference's step (oracle/grim_oracle.cpp), "
                                  "OpenMP over zones"},
            "cpu_baseline": {"value": v, "unit": "zone-cycles/s", "cores": n, "kind": "port", "sample": sample},
            "e2e": {"value": v, "unit": "zone-cycles/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }))
        return

    if world > 1:
        import torch
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    if args.workload == "batch":
        out = run_batch(args, local_rank)
        if rank == 0 and world == 1 and not args.no_cpu:
            cfg, P = batch_problems()[0]
            v, n, sample = cpu_reference(cfg, P, seconds=10.0)
            out["cpu_baseline"] = {"value": v, "unit": "zone-cycles/s", "cores": n, "kind": "port",
                                   "sample": sample}
        if rank == 0:
            print(json.dumps(out))
        return
    if args.decomp == "x3":
        if world == 1:
            import torch
            import datetime
            torch.distributed.init_process_group("nccl", init_method="tcp://127.0.0.1:%d" % _free_port(),
                                                 rank=0, world_size=1, timeout=datetime.timedelta(seconds=120))
        out = run_decomposed(args, rank, world, local_rank)
        import torch
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
        if rank == 0:
            print(json.dumps(out))
        return
    out, cfg, P = run_gpu(args, rank, world, local_rank)
    if rank == 0 and world == 1 and not args.no_cpu:
        v, n, sample = cpu_reference(cfg, P, seconds=20.0)
        out["cpu_baseline"] = {"value": v, "unit": "zone-cycles/s", "cores": n, "kind": "port",
                               "sample": sample, "host_nproc": os.cpu_count()}
        # one core (the oracle's OpenMP loops on one thread), on a smaller
        # sample of the torus set-up
        ccfg = cpu_sample_config(args.workload, cfg)
        v1, n1, sample1 = cpu_reference(ccfg, P if ccfg is cfg else None, seconds=10.0, threads=1)
        out["cpu_baseline_1core"] = {"value": v1, "unit": "zone-cycles/s", "cores": n1, "kind": "port",
                                     "sample": sample1}
    elif world > 1:
        # timed at N=1 only: the other ranks would wait for it in the barrier
        out["cpu_baseline"] = None
    if world > 1:
        import torch
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if rank == 0:
        print(json.dumps(out))


if __name__ == "__main__":
    main()
