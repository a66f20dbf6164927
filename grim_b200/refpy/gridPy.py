"""gridPy (src/grid/gridPy.pyx:36-300): a grid of numVars variables with
ghost zones, and the coordinates of its zones at a location."""
import numpy as np

from .. import config as C

# locations::CENTER ... BACK (src/params.hpp:34-37); the first five are the
# library's GRIM_CENTER .. GRIM_BOTTOM
CENTER, LEFT, RIGHT, TOP, BOTTOM, FRONT, BACK = range(7)
# directions:: (src/params.hpp:40-46)
X1, X2, X3 = 0, 1, 2


def _totals(N1, N2, N3, dim, numGhost):
    g1 = numGhost
    g2 = numGhost if dim >= 2 else 0
    g3 = numGhost if dim >= 3 else 0
    return (g1, g2, g3), (N1 + 2 * g1, N2 + 2 * g2, N3 + 2 * g3)


class gridPy:
    """grid (grid.cpp:3-120): numVars x N3Total x N2Total x N1Total doubles."""

    def __init__(self, N1, N2, N3, dim, numVars, numGhost, periodicBoundariesX1=False,
                 periodicBoundariesX2=False, periodicBoundariesX3=False):
        self._N = (int(N1), int(N2), int(N3))
        self._dim, self._numVars, self._numGhost = int(dim), int(numVars), int(numGhost)
        if (self._dim < 2 and self._N[1] != 1) or (self._dim < 3 and self._N[2] != 1):
            raise ValueError("the library holds one zone along each inactive direction (dim %d: N2, N3 = %d, %d)"
                             % (self._dim, self._N[1], self._N[2]))
        self.periodic = (bool(periodicBoundariesX1), bool(periodicBoundariesX2), bool(periodicBoundariesX3))
        self._ghost, self._total = _totals(*self._N, self._dim, self._numGhost)
        self._vars = np.zeros(self.shape)

    numVars = property(lambda self: self._numVars)
    N1 = property(lambda self: self._N[0])
    N2 = property(lambda self: self._N[1])
    N3 = property(lambda self: self._N[2])
    dim = property(lambda self: self._dim)
    # one rank: the local block is the whole grid
    iLocalStart = jLocalStart = kLocalStart = property(lambda self: 0)
    iLocalEnd = property(lambda self: self._N[0])
    jLocalEnd = property(lambda self: self._N[1])
    kLocalEnd = property(lambda self: self._N[2])
    N1Local = property(lambda self: self._N[0])
    N2Local = property(lambda self: self._N[1])
    N3Local = property(lambda self: self._N[2])
    N1Total = property(lambda self: self._total[0])
    N2Total = property(lambda self: self._total[1])
    N3Total = property(lambda self: self._total[2])
    numGhostX1 = property(lambda self: self._ghost[0])
    numGhostX2 = property(lambda self: self._ghost[1])
    numGhostX3 = property(lambda self: self._ghost[2])

    @property
    def shape(self):
        return [self._numVars, self._total[2], self._total[1], self._total[0]]

    def getVars(self):
        return self._vars.copy()

    def setVars(self, inputVars):
        a = np.ascontiguousarray(inputVars, dtype=np.float64)
        if list(a.shape) != self.shape:
            raise ValueError("setVars: shape %s, expected %s" % (list(a.shape), self.shape))
        self._vars = a.copy()

    def communicate(self):
        """grid::communicate (grid.cpp:306-360) by the library's kernel: the
        ghosts of the periodic directions become images of the interior,
        the other ghosts zero; the variables pass through a library state
        grid eight at a time."""
        from .. import _lib
        ts = self._handle()
        v = self._vars
        for v0 in range(0, self._numVars, ts.dof):
            n = min(ts.dof, self._numVars - v0)
            block = np.zeros([ts.dof] + self.shape[1:])
            block[:n] = v[v0:v0 + n]
            ts.primOld.setVars(block)
            _lib.check(_lib.lib().grim_communicate(ts._h, _lib.PRIM_OLD), "communicate")
            v[v0:v0 + n] = ts.primOld.getVars()[:n]

    def _handle(self):
        if getattr(self, "_ts", None) is None:
            from ..timestepper import timeStepper
            side = [C.PERIODIC if p else C.OUTFLOW for p in self.periodic]
            cfg = C.make_config(N1=self._N[0], N2=self._N[1], N3=self._N[2], dim=self._dim,
                                numGhost=self._numGhost, boundaryLeft=side[0], boundaryRight=side[0],
                                boundaryBottom=side[1], boundaryTop=side[1], boundaryBack=side[2],
                                boundaryFront=side[2])
            self._ts = timeStepper(cfg)
        return self._ts


class coordinatesGridPy:
    """coordinatesGrid (grid.cpp:122-249): X1, X2, X3 of every zone
    (ghosts included) at one location, set by getCoords."""

    def __init__(self, N1, N2, N3, dim, numGhost, X1Start, X1End, X2Start, X2End, X3Start, X3End):
        self._N = (int(N1), int(N2), int(N3))
        self.dim, self.numGhost = int(dim), int(numGhost)
        self.X1Start, self.X1End = float(X1Start), float(X1End)
        self.X2Start, self.X2End = float(X2Start), float(X2End)
        self.X3Start, self.X3End = float(X3Start), float(X3End)
        self._ghost, self._total = _totals(*self._N, self.dim, self.numGhost)
        self.location = CENTER

    N1 = property(lambda self: self._N[0])
    N2 = property(lambda self: self._N[1])
    N3 = property(lambda self: self._N[2])
    N1Total = property(lambda self: self._total[0])
    N2Total = property(lambda self: self._total[1])
    N3Total = property(lambda self: self._total[2])

    def config(self, **kw):
        """The library configuration of this grid (with ``kw`` on top)."""
        return C.make_config(N1=self._N[0], N2=self._N[1], N3=self._N[2], dim=self.dim, numGhost=self.numGhost,
                             X1Start=self.X1Start, X1End=self.X1End, X2Start=self.X2Start, X2End=self.X2End,
                             X3Start=self.X3Start, X3End=self.X3End, **kw)

    def getCoords(self, location):
        """setXCoords (grid.cpp:168-249): the zone index plus 0.5 along
        each direction, 0 on the face a location names and 1 on the far
        one; returns (X1, X2, X3) as [k][j][i] arrays."""
        off = {CENTER: (.5, .5, .5), LEFT: (0., .5, .5), RIGHT: (1., .5, .5), BOTTOM: (.5, 0., .5),
               TOP: (.5, 1., .5), BACK: (.5, .5, 0.), FRONT: (.5, .5, 1.)}[location]
        self.location = location
        d = [(self.X1End - self.X1Start) / self._N[0], (self.X2End - self.X2Start) / self._N[1],
             (self.X3End - self.X3Start) / self._N[2]]
        start = (self.X1Start, self.X2Start, self.X3Start)
        ax = [start[a] + (np.arange(self._total[a]) - self._ghost[a] + off[a]) * d[a] for a in range(3)]
        K, J, I = np.meshgrid(ax[2], ax[1], ax[0], indexing="ij")
        return I, J, K
