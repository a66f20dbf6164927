"""Shared helpers of the parity tests: run the CUDA product and the CPU
oracle (the checker) on the same seeded inputs and compare."""
import numpy as np

from grim_b200 import config as C
from grim_b200 import problems as PR


def interior(cfg, a):
    s3, s2, s1 = C.interior_slices(cfg)
    return a[..., s3, s2, s1]


def rel_err(a, b, floor=1e-300):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    scale = np.maximum(np.abs(b), floor)
    return float(np.max(np.abs(a - b) / scale)) if a.size else 0.0


def scaled_err(a, b):
    """max |a-b| / max |b| per leading index (variable), then max."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    out = 0.0
    for v in range(a.shape[0]):
        s = float(np.max(np.abs(b[v]))) or 1.0
        out = max(out, float(np.max(np.abs(a[v] - b[v]))) / s)
    return out


def pair(cfg):
    """(product stepper, oracle) with the same config."""
    from grim_b200.timestepper import timeStepper
    from oracle.oracle import Oracle
    return timeStepper(cfg), Oracle(cfg)
