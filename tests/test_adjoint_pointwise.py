"""The hand-written reverse mode of every pointwise function in the residual
(Euler flux, viscous flux and its rank-one forms, with and without the
optional heat flux, Roe flux with entropy fix, ghost states) against central
finite differences, on the CPU through the
check hooks (include/dgb200_check.h).  Also pins the forward functions to the
reference's own implementations where it is built here.

Check: <ybar, (y(x + h v) - y(x - h v)) / 2h>  vs  <xbar, v>  with random v,
ybar; relative tolerance 1e-7 (central differences at h = 1e-6 in FP64)."""
import ctypes

import numpy as np
import pytest

import dgpr_b200 as dg
import oracle

_dp = ctypes.POINTER(ctypes.c_double)


def _fn():
    f = dg.lib().dgb_check_pointwise
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_int, _dp, _dp, _dp, _dp, _dp]
    return f


def _p(a):
    return a.ctypes.data_as(_dp)


NOUT = {0: 15, 1: 5, 2: 15, 3: 15, 4: 5, 5: 5, 6: 5, 7: 15, 8: 15, 9: 5}
NIN = {0: 5, 1: 5, 2: 20, 3: 10, 4: 10, 5: 10, 6: 5, 7: 20, 8: 10, 9: 10}


def call(which, x, aux, ybar=None):
    x = np.ascontiguousarray(x, np.float64)
    aux = np.ascontiguousarray(aux, np.float64)
    y = np.zeros(NOUT[which])
    xbar = np.zeros(NIN[which])
    rc = _fn()(which, _p(x), _p(np.ascontiguousarray(ybar, np.float64)) if ybar is not None else None, _p(aux),
               _p(y), _p(xbar) if ybar is not None else None)
    assert rc == 0, rc
    return y, xbar


def state(rng, rho=1.0, vel=0.3, p=0.8, g=1.4):
    r = rho * (1 + 0.1 * rng.standard_normal())
    v = vel * rng.standard_normal(3)
    pp = p * (1 + 0.1 * rng.standard_normal())
    return np.array([r, *(r * v), pp / (g - 1) + 0.5 * r * v @ v])


def unit(rng):
    n = rng.standard_normal(3)
    return n / np.linalg.norm(n)


def fd_check(which, x, aux, rng, h=1e-6, tol=1e-7):
    ybar = rng.standard_normal(NOUT[which])
    v = rng.standard_normal(NIN[which])
    _, xbar = call(which, x, aux, ybar)
    yp, _ = call(which, x + h * v, aux)
    ym, _ = call(which, x - h * v, aux)
    fd = ybar @ (yp - ym) / (2 * h)
    an = xbar @ v
    assert abs(fd - an) <= tol * max(1.0, abs(an), np.abs(ybar).max() * np.abs(yp - ym).max() / (2 * h)), (fd, an)


@pytest.mark.parametrize("seed", range(8))
def test_euler_flux_vjp(seed):
    rng = np.random.default_rng(seed)
    fd_check(0, state(rng), [1.4], rng)
    fd_check(1, state(rng), [1.4, *unit(rng)], rng)


@pytest.mark.parametrize("seed", range(8))
def test_viscous_flux_vjp(seed):
    rng = np.random.default_rng(100 + seed)
    x = np.concatenate([state(rng), 0.5 * rng.standard_normal(15)])
    fd_check(2, x, [0.01 + 0.01 * seed], rng)


@pytest.mark.parametrize("seed", range(8))
def test_rank_one_viscous_vjps(seed):
    rng = np.random.default_rng(200 + seed)
    x = np.concatenate([state(rng), 0.1 * rng.standard_normal(5)])
    aux = [0.02, *unit(rng)]
    fd_check(3, x, aux, rng)
    fd_check(4, x, aux, rng)


@pytest.mark.parametrize("seed", range(16))
def test_roe_vjp(seed):
    rng = np.random.default_rng(300 + seed)
    UL, UR = state(rng), state(rng)
    if seed % 4 == 1:  # near-stagnant normal speed: the entropy fix on the contact wave
        UL[1:4] *= 0.01
        UR[1:4] *= 0.01
    if seed % 4 == 2:  # supersonic
        UL[1:4] *= 8.0
        UR[1:4] *= 8.0
        UL[4] += 0.5 * (UL[1:4] @ UL[1:4]) / UL[0] * 0.9
        UR[4] += 0.5 * (UR[1:4] @ UR[1:4]) / UR[0] * 0.9
    fd_check(5, np.concatenate([UL, UR]), [1.4, *unit(rng)], rng, h=1e-7, tol=2e-6)


@pytest.mark.parametrize("bt", [-3, -4, -7, -8])
def test_wall_and_freestream_state_vjp(bt):
    """-8: the isothermal wall (an extension), wall temperature in aux[14]."""
    rng = np.random.default_rng(17)
    aux = [bt, *unit(rng), 1.4, 287.0, 0.7, 0.9, 0.003, 1.0, 0.1, 0.0, 0.0, 1.8, 0.0021]
    for _ in range(4):
        fd_check(6, state(rng), aux, rng)


@pytest.mark.parametrize("bt,normal", [(-5, (-1.0, 0.0, 0.0)), (-6, (1.0, 0.0, 0.0))],
                         ids=["subsonic_inflow", "subsonic_outflow"])
def test_inflow_outflow_state_vjp(bt, normal):
    """The characteristic inflow / outflow ghost states (bound_states.cpp:53-130):
    total conditions of a Mach 0.3 freestream, interior states near it,
    normals near the side's axis."""
    rng = np.random.default_rng(40 + bt)
    g, R, rho, u, c = 1.4, 287.0, 1.0, 0.3, 1.0
    P = c * c * rho / g
    T = P / (rho * R)
    M = u / c
    Tt = T * (1 + 0.5 * (g - 1) * M * M)
    Pt = P * (Tt / T) ** (g / (g - 1))
    Ufr = [rho, rho * u, 0.0, 0.0, P / (g - 1) + 0.5 * rho * u * u]
    checked = 0
    for _ in range(60):
        n = np.array(normal) + 0.2 * rng.standard_normal(3)
        n /= np.linalg.norm(n)
        x = state(rng, rho=1.0, vel=0.3, p=P)
        x[1] += 0.3 * x[0]
        aux = [bt, *n, g, R, P, Pt, Tt, *Ufr]
        y = np.zeros(5)
        if _fn()(6, _p(x), None, _p(np.array(aux, np.float64)), _p(y), None) == dg.ERR_BOUNDARY:
            continue  # the forward has no boundary Mach root for this state (it reports that)
        fd_check(6, x, aux, rng)
        checked += 1
        if checked == 6:
            break
    assert checked == 6


def test_forward_pointwise_matches_reference():
    ref = oracle.reference()
    if ref is None:
        pytest.skip("reference not built here")
    rng = np.random.default_rng(5)
    for _ in range(50):
        UL, UR, n = state(rng), state(rng), unit(rng)
        f, _ = call(5, np.concatenate([UL, UR]), [1.4, *n])
        fr, _ = ref.roe(UL, UR, n, 1.4)
        assert np.max(np.abs(f - fr)) <= 1e-14 * max(1, np.max(np.abs(fr)))
        F, _ = call(0, UL, [1.4])
        assert np.max(np.abs(F.reshape(3, 5) - ref.analytical_flux(UL, 1.4))) <= 1e-14 * np.max(np.abs(F))
        G = 0.3 * rng.standard_normal(15)
        Q, _ = call(2, np.concatenate([UL, G]), [0.02])
        Qr = ref.A(UL, G[:5], G[5:10], G[10:], 0.02)
        assert np.max(np.abs(Q.reshape(3, 5) - Qr)) <= 1e-14 * max(1, np.max(np.abs(Qr)))


# ---------------------------------------------------------------- heat flux
# The optional heat flux kq = mu gamma / Pr (an extension: the reference's
# viscous flux conducts no heat): hooks 7-9 are hooks 2-4 with kq appended.

def _temperature(S, g=1.4, R=287.0):
    return (g - 1) * (S[4] - 0.5 * (S[1:4] @ S[1:4]) / S[0]) / (S[0] * R)


@pytest.mark.parametrize("seed", range(8))
def test_heat_flux_vjps(seed):
    rng = np.random.default_rng(500 + seed)
    kq = 0.02 * 1.4 / 0.71
    x = np.concatenate([state(rng), 0.5 * rng.standard_normal(15)])
    fd_check(7, x, [0.02, kq], rng)
    x = np.concatenate([state(rng), 0.1 * rng.standard_normal(5)])
    aux = [0.02, *unit(rng), kq]
    fd_check(8, x, aux, rng)
    fd_check(9, x, aux, rng)


@pytest.mark.parametrize("seed", range(6))
def test_heat_flux_is_kappa_grad_T(seed):
    """A(S, G) with the heat flux minus A(S, G) without it is kappa dT/dx_c in
    the energy row only, kappa = mu c_p / Pr with c_p = gamma R / (gamma - 1);
    dT/dx_c = grad_S T . G[c] with grad_S T by central differences of the
    temperature of the state (independent of the closed form in the kernels)."""
    rng = np.random.default_rng(600 + seed)
    g, R, mu, Pr = 1.4, 287.0, 0.015, 0.71
    S = state(rng)
    G = 0.5 * rng.standard_normal((3, 5))
    x = np.concatenate([S, G.reshape(-1)])
    Qh, _ = call(7, x, [mu, mu * g / Pr])
    Q0, _ = call(2, x, [mu])
    dT = np.zeros(5)
    for r in range(5):
        e = np.zeros(5)
        e[r] = 1e-6 * max(1.0, abs(S[r]))
        dT[r] = (_temperature(S + e, g, R) - _temperature(S - e, g, R)) / (2 * e[r])
    kappa = mu * g * R / ((g - 1) * Pr)
    diff = (Qh - Q0).reshape(3, 5)
    assert np.all(diff[:, :4] == 0.0)
    np.testing.assert_allclose(diff[:, 4], kappa * (G @ dT), rtol=1e-7, atol=1e-12)


@pytest.mark.parametrize("seed", range(6))
def test_heat_flux_rank_one_forms_agree_with_the_full_flux(seed):
    """A(S, d n^T) (hook 8) and its normal component (hook 9) equal the full
    flux (hook 7) of the gradient G[c] = n_c d."""
    rng = np.random.default_rng(700 + seed)
    S, d, n = state(rng), 0.1 * rng.standard_normal(5), unit(rng) * (0.5 + rng.random())
    mu, kq = 0.02, 0.02 * 1.4 / 0.71
    Qf, _ = call(7, np.concatenate([S, np.outer(n, d).reshape(-1)]), [mu, kq])
    Q1, _ = call(8, np.concatenate([S, d]), [mu, *n, kq])
    Qn, _ = call(9, np.concatenate([S, d]), [mu, *n, kq])
    np.testing.assert_allclose(Q1, Qf, rtol=1e-13, atol=1e-15)
    np.testing.assert_allclose(Qn, Qf.reshape(3, 5).T @ n, rtol=1e-12, atol=1e-15)


def test_zero_heat_flux_is_the_plain_flux_bit_for_bit():
    rng = np.random.default_rng(9)
    for _ in range(10):
        x = np.concatenate([state(rng), 0.5 * rng.standard_normal(15)])
        assert np.array_equal(call(7, x, [0.02, 0.0])[0], call(2, x, [0.02])[0])
        x = np.concatenate([state(rng), 0.1 * rng.standard_normal(5)])
        n = unit(rng)
        assert np.array_equal(call(8, x, [0.02, *n, 0.0])[0], call(3, x, [0.02, *n])[0])
        assert np.array_equal(call(9, x, [0.02, *n, 0.0])[0], call(4, x, [0.02, *n])[0])


def test_isothermal_wall_ghost_state():
    """Interior density, zero velocity, temperature Tw: p_b = rho R Tw."""
    rng = np.random.default_rng(18)
    g, R, Tw = 1.4, 287.0, 0.0021
    for _ in range(5):
        UL = state(rng)
        aux = [-8, *unit(rng), g, R, 0.7, 0.9, 0.003, 1.0, 0.1, 0.0, 0.0, 1.8, Tw]
        Ub, _ = call(6, UL, aux)
        assert Ub[0] == UL[0] and np.all(Ub[1:4] == 0.0)
        np.testing.assert_allclose((g - 1) * Ub[4] / (Ub[0] * R), Tw, rtol=1e-14)
