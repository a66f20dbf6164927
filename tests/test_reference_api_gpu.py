"""The reference's own tests of its grid boundaries, geometry and periodic
communication (src/boundary/test_boundary.py:56-243,
src/geometry/test_geometry.py:44-420, src/grid/test_mpi.py:1-200), run
against libgrim_b200.so through the reference-named modules gridPy,
geometryPy and boundaryPy (grim_b200/refpy).  Each test below restates one
of the reference's checks with its own tolerance; the grids are the
reference tests' set-up (unit cube, 3 ghost zones, outflow everywhere,
blackHoleSpin 0.5, hSlope 0.7, dim 3), at 16^3 zones instead of the
command-line default 64^3.

Two expectations of the reference's geometry test are restated as the
reference's code computes them rather than as that test writes them:
  * phi: the test expects 2 pi X3, but the coordinate map it tests
    (geometry.cpp:510-539) sets x^3 = X3 for both metrics;
  * the connection: the test's expected Christoffel symbols are a long
    closed form; here they are formed from the same analytic metric with
    complex-step derivatives (exact to rounding), for all 64 components.
"""
import numpy as np
import pytest

from grim_b200.refpy import boundaryPy, geometryPy, gridPy

pytestmark = pytest.mark.gpu

N1 = N2 = N3 = 16
DIM = 3
NUM_GHOST = 3
SPIN, H_SLOPE = 0.5, 0.7


# ---- boundaries (test_boundary.py) ------------------------------------------
@pytest.fixture(scope="module")
def prim():
    """gridPy of random values, like the module-level set-up of
    test_boundary.py:33-53 (numVars 1; 10 here, to also pass variables
    beyond one block of the library's eight)."""
    g = gridPy.gridPy(N1, N2, N3, DIM, 10, NUM_GHOST, False, False, False)
    g.setVars(np.random.default_rng(0).random(g.shape))
    return g


def _apply(prim, **sides):
    bc = dict(left=boundaryPy.OUTFLOW, right=boundaryPy.OUTFLOW, top=boundaryPy.OUTFLOW,
              bottom=boundaryPy.OUTFLOW, front=boundaryPy.OUTFLOW, back=boundaryPy.OUTFLOW)
    bc.update(sides)
    boundaryPy.applyBoundaryConditionsPy(bc["left"], bc["right"], bc["top"], bc["bottom"], bc["front"],
                                         bc["back"], prim)
    return prim.getVars()


def _plane(v, axis, index):
    """v[:, ..., index, ...] along zone axis 0 (X1), 1 (X2) or 2 (X3)"""
    sl = [slice(None)] * 4
    sl[3 - axis] = index
    return v[tuple(sl)]


# (side keyword, axis, lower side?) of the six sides; test_boundary.py:56-243
SIDES = [("left", 0, True), ("right", 0, False), ("bottom", 1, True), ("top", 1, False),
         ("back", 2, True), ("front", 2, False)]


@pytest.mark.parametrize("side,axis,lower", SIDES)
def test_outflow(prim, side, axis, lower):
    """OUTFLOW copies the last interior zone into every ghost zone of the
    side (test_boundary.py:56-87, 119-149, 181-211)."""
    v = _apply(prim, **{side: boundaryPy.OUTFLOW})
    n = (prim.N1Local, prim.N2Local, prim.N3Local)[axis]
    for q in range(NUM_GHOST):
        if lower:
            np.testing.assert_equal(_plane(v, axis, q), _plane(v, axis, NUM_GHOST))
        else:
            np.testing.assert_equal(_plane(v, axis, n + NUM_GHOST + q), _plane(v, axis, n + NUM_GHOST - 1))


@pytest.mark.parametrize("side,axis,lower", SIDES)
def test_mirror(prim, side, axis, lower):
    """MIRROR reflects the interior about the boundary face, without a sign
    change (test_boundary.py:88-118, 150-180, 212-243)."""
    v = _apply(prim, **{side: boundaryPy.MIRROR})
    n = (prim.N1Local, prim.N2Local, prim.N3Local)[axis]
    for q in range(NUM_GHOST):
        if lower:
            np.testing.assert_equal(_plane(v, axis, q), _plane(v, axis, 2 * NUM_GHOST - q - 1))
        else:
            np.testing.assert_equal(_plane(v, axis, n + NUM_GHOST + q), _plane(v, axis, n + NUM_GHOST - 1 - q))


def _reference_fill(v, bcs, n, g):
    """boundary.cpp:5-241 on a [var][k][j][i] array: the X1 sides over all
    j, k, then the X2 sides over all i, k, then the X3 sides over all i, j;
    only OUTFLOW and MIRROR sides are written."""
    v = v.copy()
    for axis in range(3):
        lo, hi = bcs[2 * axis], bcs[2 * axis + 1]
        N = n[axis]
        for q in range(g):
            dst_lo, dst_hi = q, N + g + q
            src = {boundaryPy.OUTFLOW: (g, N + g - 1), boundaryPy.MIRROR: (2 * g - 1 - q, N + g - 1 - q)}
            if lo in src:
                _plane(v, axis, dst_lo)[...] = _plane(v, axis, src[lo][0])
            if hi in src:
                _plane(v, axis, dst_hi)[...] = _plane(v, axis, src[hi][1])
    return v


MIXED = [
    # (left, right, bottom, top, back, front)
    (boundaryPy.OUTFLOW, boundaryPy.PERIODIC, boundaryPy.MIRROR, boundaryPy.DIRICHLET,
     boundaryPy.OUTFLOW, boundaryPy.PERIODIC),
    (boundaryPy.PERIODIC, boundaryPy.MIRROR, boundaryPy.DIRICHLET, boundaryPy.OUTFLOW,
     boundaryPy.MIRROR, boundaryPy.DIRICHLET),
    (boundaryPy.PERIODIC,) * 6,
]


@pytest.mark.parametrize("bcs", MIXED)
def test_mixed_sides_follow_the_reference_fill(bcs):
    """With PERIODIC and DIRICHLET sides among OUTFLOW and MIRROR ones the
    result is boundary.cpp's, corners included: the PERIODIC and DIRICHLET
    sides keep their ghosts (boundary.cpp has no case for them), and each
    later direction copies the earlier directions' ghost zones."""
    g0 = gridPy.gridPy(N1, N2, N3, DIM, 10, NUM_GHOST, False, False, False)
    g0.setVars(np.random.default_rng(3).random(g0.shape))
    before = g0.getVars()
    left, right, bottom, top, back, front = bcs
    boundaryPy.applyBoundaryConditionsPy(left, right, top, bottom, front, back, g0)
    want = _reference_fill(before, bcs, (g0.N1Local, g0.N2Local, g0.N3Local), NUM_GHOST)
    np.testing.assert_array_equal(g0.getVars(), want)


# ---- geometry (test_geometry.py) ---------------------------------------------
@pytest.fixture(scope="module")
def coords():
    X = gridPy.coordinatesGridPy(N1, N2, N3, DIM, NUM_GHOST, 0., 1., 0., 1., 0., 1.)
    return X, X.getCoords(gridPy.CENTER)


def _params(geom):
    assert (geom.N1, geom.N2, geom.N3, geom.dim, geom.numGhost) == (N1, N2, N3, DIM, NUM_GHOST)


def test_minkowski(coords):
    """test_geometry.py:44-91: parameters, gCov = gCon = diag(-1, 1, 1, 1),
    g = 1 and alpha = 1 everywhere."""
    X, _ = coords
    geom = geometryPy.geometryPy(geometryPy.MINKOWSKI, 0., 0., X)
    _params(geom)
    eta = np.diag([-1., 1., 1., 1.])
    for m in range(4):
        for n in range(4):
            np.testing.assert_allclose(geom.gCov[m][n], eta[m, n])
            np.testing.assert_allclose(geom.gCon[m][n], eta[m, n])
    np.testing.assert_allclose(geom.g, 1.)
    np.testing.assert_allclose(geom.alpha, 1.)


def _mks_gcov(X1, X2, a, h):
    """The modified Kerr-Schild metric of McKinney & Gammie (2004) in
    (t, X1, X2, phi), any (complex) dtype: r = exp(X1), theta = pi X2 +
    (1 - h)/2 sin(2 pi X2)."""
    r = np.exp(X1)
    th = np.pi * X2 + 0.5 * (1. - h) * np.sin(2. * np.pi * X2)
    s2 = np.sin(th) ** 2
    sigma = r * r + (a * np.cos(th)) ** 2
    dr = r
    dth = np.pi * (1. + (1. - h) * np.cos(2. * np.pi * X2))
    z = np.zeros_like(r)
    g = [[z] * 4 for _ in range(4)]
    g[0][0] = -(1. - 2. * r / sigma)
    g[0][1] = g[1][0] = 2. * r / sigma * dr
    g[0][3] = g[3][0] = -2. * a * r * s2 / sigma
    g[1][1] = (1. + 2. * r / sigma) * dr * dr
    g[1][3] = g[3][1] = -a * (1. + 2. * r / sigma) * s2 * dr
    g[2][2] = sigma * dth * dth
    g[3][3] = s2 * (sigma + a * a * (1. + 2. * r / sigma) * s2)
    return np.array([[np.asarray(g[m][n]) for n in range(4)] for m in range(4)])


def _connection(X1, X2, a, h):
    """Gamma^mu_{nu la} = 1/2 g^{mu eta} (d_la g_{eta nu} + d_nu g_{eta la}
    - d_eta g_{nu la}) of the analytic metric, the X1 and X2 derivatives by
    complex steps (exact to rounding; nothing depends on t or X3)."""
    step = 1e-30
    dg = np.zeros((4, 4, 4) + X1.shape)  # dg[d][m][n] = d g_mn / d X^d
    dg[1] = _mks_gcov(X1 + 1j * step, X2, a, h).imag / step
    dg[2] = _mks_gcov(X1, X2 + 1j * step, a, h).imag / step
    gcon = np.moveaxis(np.linalg.inv(np.moveaxis(_mks_gcov(X1, X2, a, h), (0, 1), (-2, -1))), (-2, -1), (0, 1))
    low = np.zeros_like(dg)  # Gamma_{eta nu la}
    for e in range(4):
        for n in range(4):
            for la in range(4):
                low[e, n, la] = 0.5 * (dg[la][e][n] + dg[n][e][la] - dg[e][n][la])
    return np.einsum("me...,enl...->mnl...", gcon, low)


@pytest.fixture(scope="module")
def mks(coords):
    X, (X1, X2, X3) = coords
    geom = geometryPy.geometryPy(geometryPy.MODIFIED_KERR_SCHILD, SPIN, H_SLOPE, X)
    return geom, X1, X2, X3


def test_modified_kerr_schild_params_and_coordinates(mks):
    """test_geometry.py:348-359: parameters; r = exp(X1), theta = pi X2 +
    (1 - hSlope)/2 sin(2 pi X2), phi = X3 (see the module docstring)."""
    geom, X1, X2, X3 = mks
    _params(geom)
    np.testing.assert_allclose(geom.xCoords[0], np.exp(X1))
    np.testing.assert_allclose(geom.xCoords[1], np.pi * X2 + 0.5 * (1. - H_SLOPE) * np.sin(2. * np.pi * X2))
    np.testing.assert_allclose(geom.xCoords[2], X3)


def test_modified_kerr_schild_metric(mks):
    """test_geometry.py:361-405: gCov against the analytic metric, gCon
    against its numerical inverse (1e-14 absolute where an entry vanishes),
    g = sqrt(-det gCov), alpha = 1/sqrt(-g^00), all at numpy's default
    relative tolerance of 1e-7, every zone including the ghosts."""
    geom, X1, X2, _ = mks
    g = _mks_gcov(X1, X2, SPIN, H_SLOPE)
    gm = np.moveaxis(g, (0, 1), (-2, -1))
    gcon = np.moveaxis(np.linalg.inv(gm), (-2, -1), (0, 1))
    for m in range(4):
        for n in range(4):
            np.testing.assert_allclose(geom.gCov[m][n], g[m][n], err_msg="gCov[%d][%d]" % (m, n))
            np.testing.assert_allclose(geom.gCon[m][n], gcon[m][n], atol=1e-14, err_msg="gCon[%d][%d]" % (m, n))
    np.testing.assert_allclose(geom.g, np.sqrt(-np.linalg.det(gm)))
    np.testing.assert_allclose(geom.alpha, 1. / np.sqrt(-gcon[0][0]))


def test_modified_kerr_schild_connection(mks):
    """test_geometry.py:407-...: gammaUpDownDown after
    computeConnectionCoeffs, all 64 components, against the exact
    connection of the analytic metric: the library's are central
    differences with eps = 1e-5 (geometry.cpp:61-119), so they agree to
    1e-7 relative plus 1e-7 absolute (the reference test's own tolerances
    for its components that vanish)."""
    geom, X1, X2, _ = mks
    geom.computeConnectionCoeffs()
    exact = _connection(X1, X2, SPIN, H_SLOPE)
    for idx in np.ndindex(4, 4, 4):
        np.testing.assert_allclose(geom.gammaUpDownDown[idx], exact[idx], rtol=1e-7, atol=1e-7,
                                   err_msg="gammaUpDownDown%s" % (list(idx),))


# ---- periodic communication (grid/test_mpi.py) --------------------------------
@pytest.mark.parametrize("dim", [1, 2, 3])
def test_periodic_communicate(dim):
    """grid/test_mpi.py:1-200: sin(2 pi X1) sin(2 pi X2) sin(2 pi X3) on the
    interior of a grid periodic in every direction, gridPy.communicate, then
    central differences over the whole array: at the first and last
    interior planes of each direction (where the stencil reaches into the
    ghosts) the mean error of the derivative equals the bulk's within the
    reference's 0.1 (a missing or wrong exchange makes it ~0.6).  Here the
    ghosts are also checked to be exact periodic images of the interior."""
    N = 32
    N2, N3 = (N if dim >= 2 else 1), (N if dim == 3 else 1)
    prim = gridPy.gridPy(N, N2, N3, dim, 1, NUM_GHOST, True, True, True)
    X = gridPy.coordinatesGridPy(N, N2, N3, dim, NUM_GHOST, 0., 1., 0., 1., 0., 1.)
    X1, X2, X3 = X.getCoords(gridPy.CENTER)
    g = (prim.numGhostX1, prim.numGhostX2, prim.numGhostX3)
    bulk = tuple(slice(gg, -gg) if gg else slice(None) for gg in reversed(g))  # (k, j, i)
    # sin(2 pi X) in each active direction (an inactive one holds one zone)
    S = [np.sin(2 * np.pi * X1), np.sin(2 * np.pi * X2) if dim >= 2 else 1., np.sin(2 * np.pi * X3) if dim == 3 else 1.]
    D = [2 * np.pi * np.cos(2 * np.pi * X1), 2 * np.pi * np.cos(2 * np.pi * X2), 2 * np.pi * np.cos(2 * np.pi * X3)]
    f = S[0] * S[1] * S[2]
    v = prim.getVars()
    v[(0,) + bulk] = f[bulk]
    prim.setVars(v)
    prim.communicate()
    v = prim.getVars()[0]
    # the ghosts hold the periodic images
    idx = [np.arange(n) for n in v.shape]
    for ax, gg in zip((2, 1, 0), g):
        if gg:
            n = v.shape[ax] - 2 * gg
            idx[ax] = (idx[ax] - gg) % n + gg
    np.testing.assert_array_equal(v, v[np.ix_(*idx)])
    # the derivatives at the interior's edge planes against the bulk
    dX = (1. / N, 1. / N2, 1. / N3)
    exact = [D[0] * S[1] * S[2], S[0] * D[1] * S[2], S[0] * S[1] * D[2]]
    for d in range(dim):
        ax = 2 - d
        num = np.gradient(v, dX[d], axis=ax)
        err = np.abs(num - exact[d])[bulk]
        sl = [slice(None)] * 3
        sl[ax] = 0
        first = float(np.mean(err[tuple(sl)]))
        sl[ax] = -1
        last = float(np.mean(err[tuple(sl)]))
        mid = float(np.mean(err))
        assert abs(first - mid) < 0.1 and abs(last - mid) < 0.1, (d, first, last, mid)
