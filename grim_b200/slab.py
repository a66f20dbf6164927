"""Slab decomposition of a 3D grid along X3 over ranks: one process and one
handle per GPU, the X3 halos and the two global scalars moved by
torch.distributed (NCCL between GPUs; gloo through host memory).

The reference decomposes with a PETSc DMDA and MPI (grid.cpp:306-360 for
the halo, timestep.cpp:336-400 for the dt reduction); here each rank's
handle holds N3 / world planes of the global grid (``N3Global``), its X3
ghost sides are ``GRIM_EXCHANGE`` wherever a neighbour exists (both sides
when X3 is periodic, the ring closing on rank 0), and a step runs the
library's four segments with, between them,

    before PRE   maxInvDt <- max over ranks   (the next computeDt)
    after HALF   X3 halo of primHalfStep      (the stage-end communicate)
    after FULL   nanFlag  <- sum over ranks   (fullStepDiagnostics)
    after POST   X3 halo of primOld

Every zone's arithmetic is the single-GPU step's, so a decomposed run gives
the same primitives bit for bit.  The torus observers are each slab's own
sums and extrema; ``torusObservers`` and ``observations`` combine them over
the ranks as ObserversTorus.hpp does over MPI ranks.
"""
import ctypes

import numpy as np
import torch
import torch.distributed as dist

from . import _lib
from . import config as C
from .timestepper import timeStepper

SEG_PRE, SEG_HALF, SEG_FULL, SEG_POST = 0, 1, 2, 3
SCALAR_MAXINVDT, SCALAR_NANFLAG = 0, 1

# How each torus observer (timeStepper.OBSERVERS order) combines over slabs,
# as ObserversTorus.hpp:6-253 combines it over MPI ranks: the integrals and
# boundary fluxes are summed (rank 0's value, then rank 1's, ...), rhoMax is
# a maximum, betaMin a minimum.
OBS_COMBINE = ("sum", "sum", "sum", "max", "min", "sum", "sum", "sum", "sum")


def combine_observer_rows(rows):
    """The global observers from each rank's values, ``rows`` in rank order
    (a sequence of equal-shape arrays whose last axis is the 9 observers)."""
    rows = [np.asarray(r, dtype=np.float64) for r in rows]
    out = rows[0].copy()
    for r in rows[1:]:
        for k, how in enumerate(OBS_COMBINE):
            if how == "sum":
                out[..., k] = out[..., k] + r[..., k]
            elif how == "max":
                out[..., k] = np.maximum(out[..., k], r[..., k])
            else:
                out[..., k] = np.minimum(out[..., k], r[..., k])
    return out


def slab_config(cfg, rank, world):
    """The configuration of rank's slab: N3 / world planes of the global
    grid, X3 ghost sides exchanged where a neighbour exists."""
    if cfg["dim"] != 3:
        raise ValueError("the slab decomposition splits X3 of a 3D grid")
    N3 = cfg["N3"]
    if N3 % world:
        raise ValueError("N3 = %d is not a multiple of %d ranks" % (N3, world))
    n3 = N3 // world
    if n3 < 4:
        raise ValueError("each slab needs at least 4 planes (it has %d)" % n3)
    local = dict(cfg)
    local["N3"] = n3
    local["N3Global"] = N3
    periodic = cfg["boundaryBack"] == C.PERIODIC or cfg["boundaryFront"] == C.PERIODIC
    if periodic or rank > 0:
        local["boundaryBack"] = C.EXCHANGE
    if periodic or rank < world - 1:
        local["boundaryFront"] = C.EXCHANGE
    return local


def all_gather_rows(a, world, group=None, device=None):
    """Every rank's float64 array ``a`` (same shape on all ranks), in rank
    order; through ``device`` memory for NCCL, host memory when None."""
    loc = torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64))
    if world == 1:
        return [loc.numpy()]
    t = loc if device is None else loc.to(device)
    parts = [torch.empty_like(t) for _ in range(world)]
    dist.all_gather(parts, t, group=group)
    return [p.cpu().numpy() for p in parts]


def neighbours(rank, world, periodic):
    """(lower, upper) ranks along X3; None at a physical end."""
    lower = (rank - 1) % world if (periodic or rank > 0) else None
    upper = (rank + 1) % world if (periodic or rank < world - 1) else None
    return lower, upper


def exchange_planes(send_lo, send_hi, recv_lo, recv_hi, lower, upper, rank, group=None):
    """The X3 halo swap between neighbours: recv_lo <- lower's send_hi,
    recv_hi <- upper's send_lo.  A rank that is its own neighbour (one rank,
    periodic) copies.  Tensors live where the backend wants them (CUDA for
    NCCL, CPU for gloo)."""
    ops = []
    if lower == rank and upper == rank:
        recv_lo.copy_(send_hi)
        recv_hi.copy_(send_lo)
        return
    # one send and one receive per side, posted in the same order on every
    # rank so that two messages to the same peer (two ranks, periodic) pair
    # up in order
    if lower is not None:
        ops.append(dist.P2POp(dist.isend, send_lo, lower, group))
    if upper is not None:
        ops.append(dist.P2POp(dist.irecv, recv_hi, upper, group))
    if upper is not None:
        ops.append(dist.P2POp(dist.isend, send_hi, upper, group))
    if lower is not None:
        ops.append(dist.P2POp(dist.irecv, recv_lo, lower, group))
    if ops:
        for r in dist.batch_isend_irecv(ops):
            r.wait()


class SlabTimeStepper:
    """timeStepper over one slab of a decomposed grid (rank of the default
    process group, or of ``group``)."""

    def __init__(self, cfg, group=None, device=None):
        self.group = group
        self.rank = dist.get_rank(group) if dist.is_initialized() else 0
        self.world = dist.get_world_size(group) if dist.is_initialized() else 1
        self.cfg = dict(cfg)
        self.local = slab_config(cfg, self.rank, self.world)
        self.periodic = cfg["boundaryBack"] == C.PERIODIC or cfg["boundaryFront"] == C.PERIODIC
        self.lower, self.upper = neighbours(self.rank, self.world, self.periodic)
        dev = torch.device("cuda", torch.cuda.current_device() if device is None else device)
        self.ts = timeStepper(self.local, device=dev.index)
        self.device = dev
        self.stream = torch.cuda.ExternalStream(self.ts.stream(), device=dev)
        self.host = (not dist.is_initialized()) or dist.get_backend(group) == "gloo"
        n1t, n2t = self.ts.zshape[2], self.ts.zshape[1]
        self.haloShape = (self.ts.dof, 3, n2t, n1t)
        with torch.cuda.stream(self.stream):
            mk = lambda: torch.zeros(self.haloShape, dtype=torch.float64, device=dev)
            self.sendLo, self.sendHi, self.recvLo, self.recvHi = mk(), mk(), mk(), mk()
            self.scalarD = torch.zeros(1, dtype=torch.float64, device=dev)
            self.scalarI = torch.zeros(1, dtype=torch.int64, device=dev)
        self.k0 = self.rank * self.local["N3"]

    # ---- state ---------------------------------------------------------
    def setGlobalPrims(self, P):
        """Set primOld from the global [var][k][j][i] array (ghosts included):
        this slab's planes and the 3 on each side of them."""
        n3 = self.local["N3"]
        self.ts.primOld.setVars(np.ascontiguousarray(P[:, self.k0:self.k0 + n3 + 6]))

    def localInterior(self, which=None):
        """This slab's interior of a state, [var][k][j][i]."""
        w = self.ts.primOld if which is None else which
        s3, s2, s1 = C.interior_slices(self.local)
        return w.getVars()[:, s3, s2, s1]

    def _all_gather_rows(self, a):
        return all_gather_rows(a, self.world, self.group, None if self.host else self.device)

    def torusObservers(self):
        """The torus observers of the whole decomposed grid on primOld
        (every rank gets them): each slab's, combined as OBS_COMBINE says."""
        names = timeStepper.OBSERVERS
        loc = self.ts.torusObservers()
        rows = self._all_gather_rows(np.array([loc[n] for n in names]))
        return dict(zip(names, combine_observer_rows(rows).tolist()))

    def observations(self, maxRecords=4096):
        """The records the steps wrote (ObserveEveryDt > 0), combined over
        the slabs; every rank records at the same global times."""
        names = timeStepper.OBSERVERS
        recs = self.ts.observations(maxRecords)
        n = np.array([len(recs)], dtype=np.float64)
        counts = self._all_gather_rows(n)
        if any(int(c[0]) != len(recs) for c in counts):
            raise RuntimeError("slabs hold different numbers of observer records: %s"
                               % [int(c[0]) for c in counts])
        tab = np.array([[r["time"]] + [r[k] for k in names] for r in recs]).reshape(len(recs), 1 + len(names))
        parts = self._all_gather_rows(tab)
        for p in parts[1:]:
            if not np.array_equal(p[:, 0], parts[0][:, 0]):
                raise RuntimeError("slabs recorded their observers at different times")
        vals = combine_observer_rows([p[:, 1:] for p in parts])
        return [dict(time=float(parts[0][i, 0]), **dict(zip(names, vals[i].tolist()))) for i in range(len(recs))]

    def gatherInterior(self):
        """The global interior of primOld on every rank (all-gather)."""
        loc = torch.from_numpy(np.ascontiguousarray(self.localInterior()))
        if self.world == 1:
            return loc.numpy()
        t = loc.to(self.device) if not self.host else loc
        parts = [torch.empty_like(t) for _ in range(self.world)]
        dist.all_gather(parts, t, group=self.group)
        return torch.cat([p.cpu() for p in parts], dim=1).numpy()

    # ---- the decomposed step ------------------------------------------
    def _segment(self, seg):
        _lib.check(_lib.lib().grim_step_segment(self.ts._h, int(seg)), "step_segment")

    def _ptr(self, t):
        return ctypes.c_void_p(t.data_ptr())

    def exchange(self, which):
        """The X3 halo of a state (GRIM_PRIM_OLD / GRIM_PRIM_HALF)."""
        L = _lib.lib()
        h = self.ts._h
        if self.lower is not None:
            _lib.check(L.grim_halo_x3(h, int(which), 0, 0, self._ptr(self.sendLo)), "halo pack")
        if self.upper is not None:
            _lib.check(L.grim_halo_x3(h, int(which), 1, 0, self._ptr(self.sendHi)), "halo pack")
        with torch.cuda.stream(self.stream):
            if self.host:
                bufs = [b.cpu() for b in (self.sendLo, self.sendHi, self.recvLo, self.recvHi)]
                exchange_planes(*bufs, self.lower, self.upper, self.rank, self.group)
                self.recvLo.copy_(bufs[2])
                self.recvHi.copy_(bufs[3])
            else:
                exchange_planes(self.sendLo, self.sendHi, self.recvLo, self.recvHi, self.lower, self.upper,
                                self.rank, self.group)
        if self.lower is not None:
            _lib.check(L.grim_halo_x3(h, int(which), 0, 1, self._ptr(self.recvLo)), "halo unpack")
        if self.upper is not None:
            _lib.check(L.grim_halo_x3(h, int(which), 1, 1, self._ptr(self.recvHi)), "halo unpack")

    def _reduce(self, which, op):
        if self.world == 1:
            return
        buf = self.scalarD if which == SCALAR_MAXINVDT else self.scalarI
        L = _lib.lib()
        _lib.check(L.grim_scalar_get(self.ts._h, int(which), self._ptr(buf)), "scalar_get")
        with torch.cuda.stream(self.stream):
            if self.host:
                cpu = buf.cpu()
                dist.all_reduce(cpu, op=op, group=self.group)
                buf.copy_(cpu)
            else:
                dist.all_reduce(buf, op=op, group=self.group)
        _lib.check(L.grim_scalar_set(self.ts._h, int(which), self._ptr(buf)), "scalar_set")

    def timeStep(self):
        self._reduce(SCALAR_MAXINVDT, dist.ReduceOp.MAX)
        self._segment(SEG_PRE)
        self._segment(SEG_HALF)
        self.exchange(_lib.PRIM_HALF)
        self._segment(SEG_FULL)
        self._reduce(SCALAR_NANFLAG, dist.ReduceOp.SUM)
        self._segment(SEG_POST)
        self.exchange(_lib.PRIM_OLD)

    def synchronize(self):
        self.ts.synchronize()

    @property
    def time(self):
        return self.ts.time

    @property
    def dt(self):
        return self.ts.dt
