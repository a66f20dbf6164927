"""physicsPy (src/physics/physicsPy.pyx): fluidElementPy, the fluid element
of a grid of primitives (fluidElement, physics.cpp:53-183) and its fluxes
(computeFluxes, physics.cpp:185-217), computed by the library's centre-
element kernel on the GPU (grim_element_fluxes)."""
from .gridPy import CENTER

_handles = {}


def _handle(cfg):
    """A library handle of this configuration (cached: an element holds
    only its primitives, the handle's grids are scratch)."""
    from ..timestepper import timeStepper
    key = tuple(sorted(cfg.items()))
    if key not in _handles:
        _handles[key] = timeStepper(cfg)
    return _handles[key]


class fluidElementPy:
    """fluidElement(prim, geom): the element is set from prim when it is
    made, as the reference's constructor sets it.  conduction and viscosity
    are params:: globals in the reference; they follow prim.numVars here (8:
    ideal MHD, 10: both) unless given.  The element uses the geometry at the
    zone centres (geom set to CENTER)."""

    def __init__(self, prim, geom, conduction=None, viscosity=None):
        if conduction is None and viscosity is None:
            if prim.numVars not in (8, 10):
                raise ValueError("numVars %d: give conduction and viscosity" % prim.numVars)
            conduction = viscosity = 1 if prim.numVars == 10 else 0
        if geom._centre != CENTER:
            raise ValueError("the element is set with the geometry at the zone centres")
        cfg = dict(geom._ts.cfg)
        cfg.update(conduction=int(bool(conduction)), viscosity=int(bool(viscosity)))
        self._ts = _handle(cfg)
        if self._ts.dof != prim.numVars:
            raise ValueError("numVars %d, but the element has %d variables" % (prim.numVars, self._ts.dof))
        self._prim = prim.getVars().copy()

    def computeFluxes(self, geom, direction, flux):
        """fluidElement::computeFluxes(direction) into the grid flux:
        direction indexes the four-vector (0 gives the conserved variables,
        1..3 the fluxes along X1..X3), as the reference's call does.  Returns
        (numReads, numWrites), which this library does not count: (0, 0)."""
        flux.setVars(self._ts.elementFluxes(self._prim, int(direction)))
        return 0, 0
