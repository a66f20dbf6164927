"""timeStepperPy (src/timestepper/timeStepperPy.pyx): the reference's
timeStepper as a Python object, over one library handle.

The constructor takes the reference's argument list; the state grids prim,
primOld and primHalfStep are the handle's own (getVars / setVars copy to
and from the GPU).  The diagnostic calls fill grids the object holds, as
the reference's do:
  computeDivOfFluxes(prim) -> fluxesX1..X3 (the Riemann fluxes with the
      field rows replaced by their constrained-transport values, as
      fvmfluxes.cpp:3-183 leaves them), emfX1..X3 (the edge EMFs they are
      formed from) and divFluxes (every row);
  computeEMF() / fluxCT() -> the same from the last prim computeDivOfFluxes
      was given (the reference recomputes them from its stored fluxes);
  computeDivB(prim) -> divB;
  timeStep() -> the state grids, and sourcesExplicit (the full stage's
      explicit sources, fluid rows).
The grids are gridPy objects ([var][k][j][i] with ghosts).  numVars selects
the physics as in the reference's build: 8 ideal MHD, 10 with conduction
and viscosity (other params:: values are keywords).
"""
from .. import _lib
from . import gridPy as _g
from .geometryPy import geometryPy
from .physicsPy import fluidElementPy


class timeStepperPy:
    def __init__(self, N1, N2, N3, dim, numVars, numGhost, time, dt, boundaryLeft, boundaryRight, boundaryTop,
                 boundaryBottom, boundaryFront, boundaryBack, metric, blackHoleSpin, hSlope, X1Start, X1End,
                 X2Start, X2End, X3Start, X3End, **params):
        from ..timestepper import timeStepper
        if "conduction" not in params and "viscosity" not in params:
            if numVars not in (8, 10):
                raise ValueError("numVars %d: give conduction and viscosity" % numVars)
            params["conduction"] = params["viscosity"] = 1 if numVars == 10 else 0
        self._ts = timeStepper.fromArgs(N1, N2, N3, dim, numVars, numGhost, time, dt, boundaryLeft,
                                        boundaryRight, boundaryTop, boundaryBottom, boundaryFront, boundaryBack,
                                        metric, blackHoleSpin, hSlope, X1Start, X1End, X2Start, X2End, X3Start,
                                        X3End, **params)
        cfg = self._ts.cfg  # N2, N3 are 1 along inactive directions
        self._args = (cfg["N1"], cfg["N2"], cfg["N3"], cfg["dim"], cfg["numGhost"])
        self.XCoords = self._coords()
        nv, nf = self._ts.dof, self._ts.numFluidVars
        self.fluxesX1, self.fluxesX2, self.fluxesX3 = (self._grid(nv) for _ in range(3))
        self.emfX1, self.emfX2, self.emfX3 = (self._grid(1) for _ in range(3))
        self.divFluxes = self._grid(nv)
        self.sourcesExplicit = self._grid(nf)
        self.divB = self._grid(1)
        self._geoms = {}
        self._lastFluxPrim = None

    def _grid(self, nv):
        N1, N2, N3, dim, ng = self._args
        return _g.gridPy(N1, N2, N3, dim, nv, ng)

    # the state grids (timestepper.hpp:60-62)
    prim = property(lambda self: self._ts.prim)
    primOld = property(lambda self: self._ts.primOld)
    primHalfStep = property(lambda self: self._ts.primHalfStep)

    def _coords(self):
        c = self._ts.cfg
        return _g.coordinatesGridPy(*self._args, c["X1Start"], c["X1End"], c["X2Start"], c["X2End"], c["X3Start"],
                                    c["X3End"])

    def _geom(self, location):
        if location not in self._geoms:
            cfg = self._ts.cfg
            X = self._coords()
            X.getCoords(location)
            self._geoms[location] = geometryPy(cfg["metric"], cfg["blackHoleSpin"], cfg["hSlope"], X,
                                               cfg["DerefineThetaHorizon"], cfg["DoCylindrify"])
        return self._geoms[location]

    geomCenter = property(lambda self: self._geom(_g.CENTER))
    geomLeft = property(lambda self: self._geom(_g.LEFT))
    geomRight = property(lambda self: self._geom(_g.RIGHT))
    geomBottom = property(lambda self: self._geom(_g.BOTTOM))
    geomTop = property(lambda self: self._geom(_g.TOP))

    @property
    def elem(self):
        """The fluid element of primOld at the zone centres."""
        p = self._grid(self._ts.dof)
        p.setVars(self._ts.primOld.getVars())
        return fluidElementPy(p, self.geomCenter, conduction=self._ts.cfg["conduction"],
                              viscosity=self._ts.cfg["viscosity"])

    @staticmethod
    def _vars(prim):
        return prim.getVars() if hasattr(prim, "getVars") else prim

    def timeStep(self):
        self._ts.timeStep()
        self.sourcesExplicit.setVars(self._ts.stageGrid(_lib.STAGE_SOURCES_EXPLICIT))

    def computeDivOfFluxes(self, prim):
        p = self._vars(prim)
        self._lastFluxPrim = p.copy()
        divF, _ = self._ts.computeDivOfFluxes(p)
        self.divFluxes.setVars(divF)
        self.fluxCT()

    def computeEMF(self):
        if self._lastFluxPrim is None:
            raise RuntimeError("computeEMF: no fluxes yet (call computeDivOfFluxes)")
        e = self._ts.computeEMF(self._lastFluxPrim)
        for g, a in zip((self.emfX1, self.emfX2, self.emfX3), e):
            g.setVars(a[None])

    def fluxCT(self):
        if self._lastFluxPrim is None:
            raise RuntimeError("fluxCT: no fluxes yet (call computeDivOfFluxes)")
        self.computeEMF()
        fl = self._ts.fluxCT(self._lastFluxPrim)
        for g, a in zip((self.fluxesX1, self.fluxesX2, self.fluxesX3), fl):
            g.setVars(a)

    def computeDivB(self, prim):
        self.divB.setVars(self._ts.computeDivB(self._vars(prim))[None])

