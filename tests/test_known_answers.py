"""Known-answer tests re-expressed from the reference's own unit tests
(test/quadrature_test.cpp, test/basis_test.cpp, test/math_test.cpp,
test/flux_test.cpp), run against the CPU oracle and, for the host-side pieces
the product exposes (Gauss-Legendre rule, Lagrange basis), against the product
library too.  No GPU needed."""
import math

import numpy as np
import pytest

import dgpr_b200 as dg
import oracle

O = oracle.restatement()


def _gl_oracle(n, a, b):
    x = np.zeros(n)
    w = np.zeros(n)
    O.lib.oracle_gauss_legendre(n, a, b, oracle._p(x), oracle._p(w))
    return x, w


GL_IMPLS = {"oracle": _gl_oracle, "product": dg.gauss_legendre}


def _npts(order):  # quadrature.cpp:189
    return int(math.ceil((order + 1.0) / 2.0))


def ord2_1d(x):
    return 1.2785 * x * x + 4.382 * x + 0.3854


def ord5_1d(x):
    return 2.394 * x ** 5 + 8.371 * x ** 3 + 0.23444 * x + 3.223


def ord16_1d(x):
    return 5.76594 * x ** 16 + 3.7694 * x ** 9 + 1.7674 * x ** 2 + 4.11854


def ord32_1d(x):
    return 7.584 * x ** 32 + 2.69 * x ** 17 + 10.9473


def ord2_2d(x, y):
    return 1.2785 * x * x + 4.1854 * y * y + 9.43 * x * y + 4.382 * x + 2.333 * y + 0.3854


def ord16_2d(x, y):
    return 5.76594 * x ** 16 - 0.5542 * y ** 16 + 4.2833 * x ** 10 * y ** 8 + 3.7694 * x ** 9 * y ** 3 \
        + 1.7674 * x ** 2 + 4.11854


def ord32_2d(x, y):
    return 10.3874 * x ** 32 * y ** 32 + 3.452 * x ** 4 * y ** 20 + 3.6654


def ord2_3d(x, y, z):
    return 5.2038 * x * x * y * y * z * z - 2.3385 * y * z + 1.224


def ord16_3d(x, y, z):
    return 5.76594 * x ** 16 - 0.5542 * y ** 16 * z ** 16 + 4.2833 * x ** 10 * y ** 8 * z ** 6 \
        + 3.7694 * x ** 9 * y ** 3 + 1.7674 * x * x * z * z + 4.11854


# (order, interval, function, expected) from quadrature_test.cpp:177-244
CASES_1D = [(2, (-1, 1), ord2_1d, 1.62313333333333), (2, (0, 1), ord2_1d, 3.00256666666667),
            (5, (-1, 1), ord5_1d, 6.44600000000000), (5, (0.68834, 1), ord5_1d, 3.04565071481875),
            (16, (-1, 1), ord16_1d, 10.0936925490196), (16, (-0.22954, 1), ord16_1d, 6.37628085636999),
            (32, (-1, 1), ord32_1d, 22.3542363636364), (32, (0.78452, 1), ord32_1d, 2.73621651233878)]
CASES_2D = [(2, (-1, 1), ord2_2d, 8.82680000000000), (2, (0, 1), ord2_2d, 7.92170000000000),
            (16, (-1, 1), ord16_2d, 20.2300477243018), (16, (0, 1), ord16_2d, 5.15174693107546),
            (32, (-1, 1), ord32_2d, 14.8312586645678), (32, (0, 1), ord32_2d, 3.70781466614194)]
CASES_3D = [(2, (-1, 1), ord2_3d, 11.3338666666667), (2, (0, 1), ord2_3d, 0.832108333333333),
            (16, (-1, 1), ord16_3d, 37.2668310398099), (16, (0, 1), ord16_3d, 4.75258887997623)]


@pytest.mark.parametrize("impl", list(GL_IMPLS))
def test_gauss_legendre_integrals(impl):
    gl = GL_IMPLS[impl]
    for order, (a, b), f, want in CASES_1D:
        x, w = gl(_npts(order), a, b)
        assert abs(np.dot(w, f(x)) - want) < 2e-14 * abs(want) + 1e-14
    for order, (a, b), f, want in CASES_2D:
        x, w = gl(_npts(order), a, b)
        X, Y = np.meshgrid(x, x, indexing="ij")
        W = np.outer(w, w)
        assert abs(np.sum(W * f(X, Y)) - want) < 2e-14 * abs(want) + 1e-14
    for order, (a, b), f, want in CASES_3D:
        x, w = gl(_npts(order), a, b)
        X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
        W = np.einsum("i,j,k->ijk", w, w, w)
        assert abs(np.sum(W * f(X, Y, Z)) - want) < 2e-14 * abs(want) + 1e-14


def test_gauss_legendre_matches_reference_rule():
    ref = oracle.reference()
    if ref is None:
        pytest.skip("reference not built here")
    for n in range(1, 12):
        order = 2 * n - 1
        xr, wr = np.zeros(n), np.zeros(n)
        ref.lib.ref_gauss_legendre_1d(order, 0.0, 1.0, oracle._p(xr), oracle._p(wr))
        for impl in GL_IMPLS.values():
            x, w = impl(n, 0.0, 1.0)
            assert np.max(np.abs(x - xr)) < 2e-16 and np.max(np.abs(w - wr)) < 4e-16


LAG = {"oracle": (O.lagrange1d, O.lagrange1d_deriv), "product": (dg.lagrange1d, dg.lagrange1d_deriv)}
PNTS = (0.223, 0.437, 0.945)  # basis_test.cpp:26-28


@pytest.mark.parametrize("impl", list(LAG))
def test_lagrange_values_and_derivatives(impl):
    lag, dlag = LAG[impl]
    hand = {1: [lambda x: 1 - x, lambda x: x], 2: [lambda x: 2 * x * x - 3 * x + 1, lambda x: -4 * x * x + 4 * x,
                                                   lambda x: 2 * x * x - x]}
    dhand = {1: [lambda x: -1.0, lambda x: 1.0], 2: [lambda x: 4 * x - 3, lambda x: -8 * x + 4, lambda x: 4 * x - 1]}
    for x in PNTS:
        assert lag(0, 0, x) == 1.0 and dlag(0, 0, x) == 0.0
        for p in (1, 2):
            for i in range(p + 1):
                assert abs(lag(i, p, x) - hand[p][i](x)) < 1e-15
                assert abs(dlag(i, p, x) - dhand[p][i](x)) < 1e-14
    for p in range(1, 9):  # Lagrange property at the equispaced nodes
        for i in range(p + 1):
            for j in range(p + 1):
                assert abs(lag(i, p, j / p) - (1.0 if i == j else 0.0)) < 1e-13


@pytest.mark.parametrize("p", [0, 2, 7])
@pytest.mark.parametrize("impl", list(LAG))
def test_partition_of_unity_at_quadrature_points(p, impl):
    """basis_test.cpp:380-476: sum of all basis values is 1 and of all
    gradients is 0 at every volume quadrature point."""
    lag, dlag = LAG[impl]
    x, _ = dg.gauss_legendre(p + 1)
    for q in x:
        s = sum(lag(i, p, q) for i in range(p + 1))
        ds = sum(dlag(i, p, q) for i in range(p + 1))
        assert abs(s - 1.0) < 1e-13 and abs(ds) < 5e-12


# ------------------------------------------------------------------ dense math

A = np.array([4.20, -3.60, 3.14, 2.71, 8.33, -4.44, 5.22, 1.01, 5.55])
B = np.array([9.88, -5.50, -1.22, 5.22, 9.52, -0.22, 8.22, 4.73, -3.22])


def test_det_and_inverse_3x3():
    """math_test.cpp:166-191."""
    for M, det in ((A, 2.2264818999999997e+02), (B, -3.0973650800000019e+02)):
        assert abs(O.lib.oracle_det3(oracle._p(M)) - det) < 1e-13 * abs(det)
        inv = np.zeros(9)
        O.lib.oracle_inv3(oracle._p(M), oracle._p(inv))
        assert np.max(np.abs(inv - np.linalg.inv(M.reshape(3, 3)).ravel())) < 1e-15


@pytest.mark.parametrize("N", [10, 100])
def test_gauss_jordan_inverse(N):
    """math_test.cpp:262-307; matrices from MT19937(42) as scripts/linalg.py."""
    rng = np.random.Generator(np.random.MT19937(42))
    C = rng.random((10, 10))
    D = rng.random((100, 100))
    M = (C if N == 10 else D).ravel().copy()
    og = M.copy()
    assert O.lib.oracle_invert(N, oracle._p(M)) == 0
    I = og.reshape(N, N) @ M.reshape(N, N)
    assert np.max(np.abs(I - np.eye(N))) < (5e-15 if N == 10 else 5e-13)


def test_symmetric_packed_matvec():
    """math_test.cpp:204-249."""
    full = np.array([
        [-10, 18, -8, -1, -1, 11, 0, 3, 4, 5], [18, -2, 3, 15, -3, -9, 9, 6, 2, 10],
        [-8, 3, 0, 6, 7, 6, 8, 7, -3, -4], [-1, 15, 6, 16, 14, 7, -3, -1, 5, 3],
        [-1, -3, 7, 14, 18, 3, 3, -2, 9, -8], [11, -9, 6, 7, 3, 14, -1, 2, 15, 0],
        [0, 9, 8, -3, 3, -1, 14, 5, 2, 4], [3, 6, 7, -1, -2, 2, 5, -8, -3, 2],
        [4, 2, -3, 5, 9, 15, 2, -3, 12, 6], [5, 10, -4, 3, -8, 0, 4, 2, 6, 10]], dtype=np.float64)
    packed = np.concatenate([full[i, i:] for i in range(10)])
    vec = np.array([8, 6, -3, 2, -5, -5, 8, 8, -1, -3], dtype=np.float64)
    sol = np.array([5, 301, 36, -55, -101, -62, 152, 10, -95, 170], dtype=np.float64)
    out = np.zeros(10)
    O.lib.oracle_symm_packed_mv(10, oracle._p(packed), oracle._p(vec), 1.0, oracle._p(out))
    assert np.array_equal(out, sol)


# ------------------------------------------------------------------------ flux

def _roe_states():
    """flux_test.cpp:25-88: supersonic (M 2.2) left/right states and a normal."""
    g, Minf, c = 1.4, 2.2, 1.0
    d = math.pi / 180.0
    f32 = np.float32
    phl, thl, phr, thr, phn, thn = 5 * d, 85 * d, 3 * d, 87 * d, 2 * d, 83 * d
    Ml, Mr, rl, rr = Minf + 0.01, Minf - 0.02, 1.02, 1.04
    ul, vl, wl = Ml * float(np.cos(f32(phl))) * float(np.sin(f32(thl))), Ml * float(np.sin(f32(phl))) * float(
        np.sin(f32(thl))), Ml * float(np.cos(f32(thl)))
    ur, vr, wr = Mr * float(np.cos(f32(phr))) * float(np.sin(f32(thr))), Mr * float(np.sin(f32(phr))) * float(
        np.sin(f32(thr))), Mr * float(np.cos(f32(thr)))
    Ul = np.array([rl, rl * ul, rl * vl, rl * wl, rl * c * c / (g * (g - 1)) + 0.5 * rl * Ml * Ml])
    Ur = np.array([rr, rr * ur, rr * vr, rr * wr, rr * c * c / (g * (g - 1)) + 0.5 * rr * Mr * Mr])
    n = np.array([float(np.cos(f32(phn))) * float(np.sin(f32(thn))),
                  float(np.sin(f32(phn))) * float(np.sin(f32(thn))), float(np.cos(f32(thn)))])
    F = O.analytical_flux(Ul, g)
    return g, Ul, Ur, n, F.T @ n


def test_roe_equal_states_is_the_analytic_flux():
    g, Ul, Ur, n, fl = _roe_states()
    f, _ = O.roe(Ul, Ul, n, g)
    assert np.max(np.abs(f - fl)) < 1e-14 * np.max(np.abs(fl))


def test_roe_flip_antisymmetry():
    g, Ul, Ur, n, _ = _roe_states()
    ff, _ = O.roe(Ul, Ur, n, g)
    fr, _ = O.roe(Ur, Ul, -n, g)
    assert np.max(np.abs(ff + fr)) < 1e-14 * np.max(np.abs(ff))


def test_roe_supersonic_upwind():
    g, Ul, Ur, n, fl = _roe_states()
    f, _ = O.roe(Ul, Ur, n, g)
    assert np.max(np.abs(f - fl)) < 1e-14 * np.max(np.abs(fl))


def test_roe_matches_reference_including_entropy_fix():
    ref = oracle.reference()
    if ref is None:
        pytest.skip("reference not built here")
    rng = np.random.default_rng(3)
    for k in range(200):
        rho = 1 + 0.1 * rng.standard_normal(2)
        vel = 0.3 * rng.standard_normal((2, 3))
        if k % 2:  # near-sonic / stagnant normal speeds exercise the entropy fix
            vel *= 0.01
        p = 0.7 + 0.05 * rng.standard_normal(2)
        U = [np.array([r, *(r * v), pp / 0.4 + 0.5 * r * v @ v]) for r, v, pp in zip(rho, vel, p)]
        n = rng.standard_normal(3)
        n /= np.linalg.norm(n)
        fo, so = O.roe(U[0], U[1], n, 1.4)
        fr, sr = ref.roe(U[0], U[1], n, 1.4)
        assert np.max(np.abs(fo - fr)) < 1e-14 * max(1.0, np.max(np.abs(fr)))
        assert abs(so - sr) < 1e-15 * max(1.0, sr)
