"""boundaryPy (src/boundary/boundaryPy.pyx): applyBoundaryConditionsPy
fills a grid's ghost zones (boundary.cpp:5-241) with the library's ghost
fill kernel on the GPU."""
import ctypes

import numpy as np

from .. import _lib
from .. import config as C

# boundaries:: (src/params.hpp:50-53), the library's GRIM_PERIODIC ..
PERIODIC, OUTFLOW, MIRROR, DIRICHLET = C.PERIODIC, C.OUTFLOW, C.MIRROR, C.DIRICHLET

_handles = {}


def _handle(prim, bcs):
    """A library handle of prim's shape with these boundary kinds (cached);
    ideal MHD (8 variables per zone).  boundary.cpp:5-241 fills OUTFLOW and
    MIRROR sides only and leaves PERIODIC (grid::communicate's) and
    DIRICHLET (a problem hook's) sides as they are: those sides are
    GRIM_EXCHANGE here, the library's "keep these ghosts"."""
    key = (prim.N1, prim.N2, prim.N3, prim.dim, prim.numGhostX1, bcs)
    if key not in _handles:
        from ..timestepper import timeStepper
        left, right, top, bottom, front, back = (C.EXCHANGE if b in (PERIODIC, DIRICHLET) else b for b in bcs)
        cfg = C.make_config(N1=prim.N1, N2=prim.N2, N3=prim.N3, dim=prim.dim, numGhost=prim.numGhostX1,
                            boundaryLeft=left, boundaryRight=right, boundaryTop=top, boundaryBottom=bottom,
                            boundaryFront=front, boundaryBack=back)
        _handles[key] = timeStepper(cfg)
    return _handles[key]


def applyBoundaryConditionsPy(boundaryLeft, boundaryRight, boundaryTop, boundaryBottom, boundaryFront,
                              boundaryBack, prim):
    """The ghost fill of the OUTFLOW and MIRROR sides, in place on prim's
    variables (the other sides keep their ghosts): they pass through the
    library's state grid eight at a time."""
    bcs = tuple(int(b) for b in (boundaryLeft, boundaryRight, boundaryTop, boundaryBottom, boundaryFront,
                                 boundaryBack))
    ts = _handle(prim, bcs)
    v = prim.getVars()
    for v0 in range(0, prim.numVars, ts.dof):
        n = min(ts.dof, prim.numVars - v0)
        block = np.zeros([ts.dof] + prim.shape[1:])
        block[:n] = v[v0:v0 + n]
        ts.primOld.setVars(block)
        _lib.check(_lib.lib().grim_apply_boundaries(ts._h, _lib.PRIM_OLD), "apply_boundaries")
        v[v0:v0 + n] = ts.primOld.getVars()[:n]
    prim.setVars(v)
