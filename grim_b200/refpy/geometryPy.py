"""geometryPy (src/geometry/geometryPy.pyx): the metric of a coordinates
grid, computed by the library's geometry kernel (geometry.cpp:4-680) on the
GPU."""
import numpy as np

from .. import config as C
from .gridPy import BACK, FRONT

# metrics:: (src/params.hpp:58-61)
MINKOWSKI, MODIFIED_KERR_SCHILD = C.MINKOWSKI, C.MODIFIED_KERR_SCHILD


class geometryPy:
    """geometry(metric, blackHoleSpin, hSlope, XCoordsGrid): gCov and gCon
    as [4][4][k][j][i], g and alpha as [k][j][i], xCoords as [3][k][j][i]
    at the location XCoordsGrid was last set to.  DerefineThetaHorizon and
    DoCylindrify are params:: globals in the reference (off in its
    geometry tests); they are keywords here."""

    def __init__(self, metric, blackHoleSpin, hSlope, XCoordsGrid, DerefineThetaHorizon=0, DoCylindrify=0):
        from ..timestepper import timeStepper
        if XCoordsGrid.location in (FRONT, BACK):
            raise ValueError("the X3 faces have the centre's metric (no metric here depends on X3); "
                             "set the coordinates to CENTER")
        self.metric, self.blackHoleSpin, self.hSlope = int(metric), float(blackHoleSpin), float(hSlope)
        self._X = XCoordsGrid
        cfg = XCoordsGrid.config(metric=self.metric, blackHoleSpin=self.blackHoleSpin, hSlope=self.hSlope,
                                 DerefineThetaHorizon=int(DerefineThetaHorizon), DoCylindrify=int(DoCylindrify))
        self._ts = timeStepper(cfg)
        G = self._ts.getGeometry(XCoordsGrid.location)
        self.gCov, self.gCon, self.g, self.alpha = G["gCov"], G["gCon"], G["g"], G["alpha"]
        # x^3 = X3 for both metrics (geometry.cpp:510-539); the library's
        # metric does not depend on it, so only x^1, x^2 are stored
        X3 = XCoordsGrid.getCoords(XCoordsGrid.location)[2]
        self.xCoords = np.stack([G["x"][0], G["x"][1], X3])
        self._centre = XCoordsGrid.location

    N1 = property(lambda self: self._X.N1)
    N2 = property(lambda self: self._X.N2)
    N3 = property(lambda self: self._X.N3)
    dim = property(lambda self: self._X.dim)
    numGhost = property(lambda self: self._X.numGhost)

    def computeConnectionCoeffs(self):
        """gammaUpDownDown[mu][nu][la] as [4][4][4][k][j][i] (central
        differences of the metric, eps = 1e-5, geometry.cpp:61-119); the
        library forms them at the zone centres."""
        from .gridPy import CENTER
        if self._centre != CENTER:
            raise ValueError("the connection is computed at the zone centres")
        self.gammaUpDownDown = self._ts.getGeometry(CENTER)["gamma"]
