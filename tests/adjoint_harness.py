"""Test harness around the adjoint entry points (grim_adjoint_forward /
grim_adjoint_backward, through the ctypes binding): a torch.autograd.Function
over whole checkpointed timesteps, and the central-difference check of a
gradient that the adjoint tests share.

This module is test infrastructure: the library exposes the adjoint through
its C ABI only; the autograd wrapper lives here, beside the tests that use
it.
"""
import math

import numpy as np
import torch

from tests.helpers import interior


def prepare(ts, cfg, P, t0=0.0):
    """Load P as primOld with its ghosts the periodic images of the
    interior, time t0 and the config's dt held fixed."""
    ts.primOld.setVars(P)
    ts.primOld.communicate()
    ts.setTime(t0, cfg["dt"])
    ts.setFixedDt(True)


def fold_ghosts(cfg, a):
    """a (2D periodic, [var][1][j][i] with ghosts) with every ghost entry
    added to the interior zone it is the periodic image of, ghosts zeroed"""
    g, N1, N2 = cfg["numGhost"], cfg["N1"], cfg["N2"]
    out = np.zeros_like(a)
    jj = (np.arange(a.shape[2]) - g) % N2 + g
    ii = (np.arange(a.shape[3]) - g) % N1 + g
    J, I = np.meshgrid(jj, ii, indexing="ij")
    for v in range(a.shape[0]):
        np.add.at(out[v, 0], (J, I), a[v, 0])
    return out


def interior_mask(cfg, shape):
    g = cfg["numGhost"]
    m = np.zeros(shape, bool)
    m[:, :, g:g + cfg["N2"], g:g + cfg["N1"]] = True
    return m


class TimeSteps(torch.autograd.Function):
    """P_final = S^n(P_initial) for a stepper ``ts`` of a 2D periodic ideal
    MHD problem: forward = grim_adjoint_forward (checkpoints every
    ``every`` steps, dt fixed), backward = grim_adjoint_backward (the
    vector-Jacobian product of the whole run, checkpoints recomputed).
    Tensors are float64 [var][k][j][i] with ghosts on the CPU; the ghosts of
    the input are replaced by periodic images, so their gradient is zero;
    the ghosts of the output are periodic images of its interior, so the
    incoming gradient's ghost entries are added to the interior zones they
    copy.  The stepper keeps
    the checkpoints of its last forward run only: a backward whose forward
    is no longer the stepper's last runs it again first."""

    @staticmethod
    def forward(ctx, p0, ts, cfg, nsteps, every):
        ctx.p0 = np.ascontiguousarray(p0.detach().numpy()).copy()
        ctx.ts, ctx.cfg, ctx.nsteps, ctx.every = ts, cfg, int(nsteps), int(every)
        prepare(ts, cfg, ctx.p0)
        ts.adjointForward(ctx.nsteps, ctx.every)
        ts._adjoint_run = ctx
        return torch.from_numpy(ts.primOld.getVars())

    @staticmethod
    def backward(ctx, gout):
        ts = ctx.ts
        if getattr(ts, "_adjoint_run", None) is not ctx:
            prepare(ts, ctx.cfg, ctx.p0)
            ts.adjointForward(ctx.nsteps, ctx.every)
            ts._adjoint_run = ctx
        lam = fold_ghosts(ctx.cfg, np.ascontiguousarray(gout.detach().numpy(), dtype=np.float64))
        grad = ts.adjointBackward(lam)
        return torch.from_numpy(grad), None, None, None, None


def fd_check(loss_of, L0, adjoint, picks, scale, rtol=1e-6):
    """Central differences of the scalar map ``loss_of(*pick, h)`` (the
    loss after shifting the interior entry ``pick``, e.g. (v, j, i), by h)
    against ``adjoint[pick]`` at the picked entries.  The forward map is
    piecewise smooth (limiter branches, the Riemann solvers' min / max of
    speeds): an entry counts only where the differences at h = 1e-6 and
    1e-7 agree and the second differences show no slope jump at the point;
    there the adjoint must match one of the two differences to ``rtol``
    of max(|adjoint|, 1e-3 scale).  The screens allow for the rounding of
    the loss itself, two ulps of L0 per evaluation (the loss is an exactly
    rounded sum; the forward map's last bits add about as much), divided
    by the step.  Returns (entries checked, failures)."""
    smooth, bad = 0, []
    noise = 2 * math.ulp(abs(L0))  # rounding of one loss evaluation
    for pick in picks:
        ad = adjoint[tuple(pick)]
        tol = max(abs(ad), 1e-3 * scale)
        p6, m6 = loss_of(*pick, 1e-6), loss_of(*pick, -1e-6)
        p7, m7 = loss_of(*pick, 1e-7), loss_of(*pick, -1e-7)
        f6, f7 = (p6 - m6) / 2e-6, (p7 - m7) / 2e-7
        if abs(f6 - f7) > 3e-6 * tol + 2 * noise / 2e-7:
            continue  # a branch switch inside the bracket
        s6, s7 = (p6 - 2 * L0 + m6) / 1e-6, (p7 - 2 * L0 + m7) / 1e-7
        if abs(s7 - s6 / 10.) > 1e-6 * tol + 4 * noise / 1e-7:
            continue  # a slope jump at the point
        smooth += 1
        # the two differences carry different errors (truncation at 1e-6,
        # rounding at 1e-7); the adjoint must match one of them
        if min(abs(f6 - ad), abs(f7 - ad)) > rtol * tol:
            bad.append(tuple(pick) + (f6, f7, ad))
    return smooth, bad


def energy(cfg, Pf, background):
    """L = 1/2 sum over the interior of (P_final - background)^2, the sum
    exactly rounded"""
    d = (interior(cfg, Pf) - np.asarray(background)[:, None, None, None]).ravel()
    return 0.5 * math.fsum((d * d).tolist())


def energy_lambda(cfg, Pf, background):
    """dL / dP_final of ``energy`` (zero on the ghosts)"""
    lam = Pf - np.asarray(background)[:, None, None, None]
    lam[~interior_mask(cfg, lam.shape)] = 0.0
    return lam


def fd_check_richardson(loss_of, L0, adjoint, picks, scale, rtol=1e-6, h=1e-6):
    """As fd_check, for maps whose third derivatives make the 1e-6 central
    difference's truncation error larger than 1e-6 (the EMHD runs): the
    central differences D(h) at h, 2h and 4h, Richardson-extrapolated to
    R(h) = (4 D(h) - D(2h)) / 3 and R(2h) likewise (truncation O(h^4)).  An
    entry counts where R(h) and R(2h) agree to 1e-5 of max(|adjoint|, 1e-3
    scale) (no branch switch within 4h; the loss's rounding allowed for),
    and there the adjoint must match one of them to ``rtol`` of that, or to twice
    the two extrapolations' own scatter where it is larger: the EMHD runs'
    differences scatter by 1e-7..6e-6 of their value (measured, the
    forward's Newton converging to its own floor), and no gradient can be
    checked more tightly than the differences repeat.  Returns (entries
    checked, failures)."""
    smooth, bad = 0, []
    noise = 2 * math.ulp(abs(L0))
    for pick in picks:
        ad = adjoint[tuple(pick)]
        tol = max(abs(ad), 1e-3 * scale)
        D = {}
        for k in (1, 2, 4):
            D[k] = (loss_of(*pick, k * h) - loss_of(*pick, -k * h)) / (2 * k * h)
        if not all(math.isfinite(d) for d in D.values()):
            continue  # a perturbed run left the map (a non-finite loss)
        r1 = (4 * D[1] - D[2]) / 3
        r2 = (4 * D[2] - D[4]) / 3
        spread = abs(r1 - r2)
        if spread > 1e-5 * tol + 4 * noise / h:
            continue  # a branch switch within 4h of the point
        smooth += 1
        if min(abs(r1 - ad), abs(r2 - ad)) > max(rtol * tol, 2 * spread):
            bad.append(tuple(pick) + (r1, r2, ad))
    return smooth, bad
