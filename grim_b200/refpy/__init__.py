"""The reference's Python modules for its grid, geometry, boundaries, fluid
element and timestepper (src/grid/gridPy.pyx, src/geometry/geometryPy.pyx,
src/boundary/boundaryPy.pyx, src/physics/physicsPy.pyx,
src/timestepper/timeStepperPy.pyx: Cython over ArrayFire) restated over
libgrim_b200.so, with the same names, constructor arguments, constants and
array shapes, so the reference's own tests of those pieces run against this
library: ``from grim_b200.refpy import gridPy, geometryPy, boundaryPy,
physicsPy, timeStepperPy``.

Grids live on the host here (numpy, [var][k][j][i] with ghosts, the layout
gridPy.getVars returns); the geometry and the boundary fill are computed by
the library's kernels on the GPU.  One process, one rank: the local extents
equal the global ones.
"""
