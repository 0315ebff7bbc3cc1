"""The optional heat flux (dgb_set_prandtl) on the GPU, through the C ABI.

The reference's viscous flux conducts no heat (flux.cpp:185-201); the heat
flux kappa grad T, kappa = mu c_p / Pr, is an extension and its parity is
unpinned: no reference output exists to compare with.  What pins it instead:

  off            Pr = 0 and Pr = inf run the plain kernels: bit-identical to a
                 handle that never set a Prandtl number
  affine in kq   every term of the residual is linear in the heat
                 coefficient, so R(2 kq) - R(0) = 2 (R(kq) - R(0)), on every
                 residual case (all boundary types, affine and curved)
  conservation   periodic boxes: the heat flux moves energy, it creates none
  heat equation  a quiescent gas at uniform pressure with a temperature wave
                 has dE/dt = kappa T'' and no mass or momentum change; the DG
                 rate converges to it under refinement
  adjoint        dot-product tests of the residual VJP on every residual case,
                 one RK step and N recorded steps against central differences
  mixed form     the FP32 form with heat stays within 1e-6 of FP64 with heat
  invalidation   changing Pr drops captured graphs and the recorded run
"""
import math

import numpy as np
import pytest

import dgpr_b200 as dg
from tests import cases as C

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

PR = 0.71


def solver(c, precision=dg.FP64):
    return dg.Solver(dg.Mesh(c.nx, c.ny, c.nz, c.p, c.q, c.nodes, c.bounds), dg.Params.from_array(c.prm), precision)


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


CASES = C.residual_cases()


def _tgv_case(n=3, p=2, mu=2e-2):
    nodes = C.box_nodes(n, n, n, 1, 2 * math.pi, 2 * math.pi, 2 * math.pi)
    xyz = C.node_coords(n, n, n, p, 1, nodes)
    prm = C.params(mu=mu, c=1.0 / 0.3, u=0.0, v=0.0, w=0.0)
    U = C.taylor_green(xyz, Ma=0.3).reshape(-1)
    return C.Case("tgv", n, n, n, p, 1, nodes, [C.P_] * 6, prm, U)


def _step(s, U, scheme, dt, n=1):
    s.set_state(U)
    s.step(scheme, dt, n, norms=False)
    return s.get_state()


@pytest.mark.parametrize("precision", [dg.FP64, dg.MIXED_FP32], ids=["fp64", "mixed"])
def test_zero_and_infinite_prandtl_are_the_plain_physics(precision):
    case = next(c for c in CASES if c.name == "noslip_p3")
    with solver(case, precision) as s:
        R0, f0 = s.residual(case.U)
        s.set_prandtl(PR)
        R1, _ = s.residual(case.U)
        assert not np.array_equal(R1, R0)
        for off in (0.0, math.inf):
            s.set_prandtl(off)
            R, f = s.residual(case.U)
            assert np.array_equal(R, R0) and np.array_equal(f, f0)
        for bad in (-1.0, math.nan):
            with pytest.raises(dg.DgbError):
                s.set_prandtl(bad)


@pytest.mark.parametrize("case", CASES, ids=lambda c: c.name)
def test_residual_is_affine_in_the_heat_coefficient(case):
    with solver(case) as s:
        R0, _ = s.residual(case.U)
        s.set_prandtl(PR)
        R1, _ = s.residual(case.U)
        s.set_prandtl(PR / 2)
        R2, _ = s.residual(case.U)
    if case.prm[2] == 0.0:  # inviscid: mu gamma / Pr = 0
        assert np.array_equal(R1, R0) and np.array_equal(R2, R0)
        return
    d1, d2 = R1 - R0, R2 - R0
    assert np.linalg.norm(d1) > 1e-6 * np.linalg.norm(R0)
    assert rel(d2, 2.0 * d1) < 1e-9, rel(d2, 2.0 * d1)


@pytest.mark.parametrize("case", [c for c in CASES if all(b == C.P_ for b in c.bounds) and c.prm[2] > 0
                                  and not any(c.prm[11:16])], ids=lambda c: c.name)
def test_heat_flux_conserves_energy_on_periodic_meshes(case):
    """sum over all nodes of R[e][r][b] is the rate of the integral of
    variable r (the Lagrange basis sums to one)."""
    with solver(case) as s:
        s.set_prandtl(PR)
        R, _ = s.residual(case.U)
    R = R.reshape(case.nelem, 5, case.nb)
    tot = R.sum(axis=(0, 2))
    scale = np.abs(R).sum(axis=(0, 2))
    assert np.all(np.abs(tot) < 1e-11 * scale), tot / scale


def _temperature_wave(nx, p, eps=0.1, mu=1e-2):
    """Periodic [0,1]^3, nx x 1 x 1 elements; u = 0, p = p0, T = T0 (1 + eps
    sin 2 pi x), rho = p0 / (R T).  Returns the case and dE/dt = kappa T''."""
    g, R = 1.4, 287.0
    prm = C.params(gamma=g, gcnst=R, mu=mu, c=1.0, u=0.0)
    p0 = prm[5]
    T0 = p0 / R  # rho = 1 at T0
    nodes = C.box_nodes(nx, 1, 1, 1, 1.0, 1.0, 1.0)
    x = C.node_coords(nx, 1, 1, p, 1, nodes)[..., 0]
    T = T0 * (1.0 + eps * np.sin(2 * np.pi * x))
    rho = p0 / (R * T)
    z = 0.0 * x
    U = C.state_from_primitives(rho, z, z, z, p0 + z, g).reshape(-1)
    kappa = mu * g * R / ((g - 1.0) * PR)
    rate = -kappa * T0 * eps * (2 * np.pi) ** 2 * np.sin(2 * np.pi * x)
    return C.Case("twave", nx, 1, 1, p, 1, nodes, [C.P_] * 6, prm, U), rate


def test_temperature_wave_follows_the_heat_equation():
    errs = []
    for nx in (8, 16):
        case, rate = _temperature_wave(nx, 3)
        with solver(case) as s:
            _, f0 = s.residual(case.U)
            s.set_prandtl(PR)
            _, f = s.residual(case.U)
        f = f.reshape(case.nelem, 5, case.nb)
        scale = np.abs(rate).max()
        # no jumps at the faces (the interpolant is exact there), uniform
        # pressure, no velocity: only the heat flux acts, on the energy
        assert np.abs(f0).max() < 1e-10 * scale
        assert np.abs(f[:, :4]).max() < 1e-10 * scale
        errs.append(np.linalg.norm(f[:, 4] - rate) / np.linalg.norm(rate))
    assert errs[0] < 0.05 and errs[1] < errs[0] / 3.0, errs


@pytest.mark.parametrize("case", CASES, ids=lambda c: c.name)
def test_residual_vjp_dot_product_with_heat(case):
    rng = np.random.default_rng(12)
    with solver(case) as s:
        s.set_prandtl(PR)
        U = case.U
        for _ in range(2):
            lam = rng.standard_normal(U.size)
            v = rng.standard_normal(U.size) * np.maximum(np.abs(U), 1.0)
            h = 1e-6
            fd = lam @ (s.residual(U + h * v)[1] - s.residual(U - h * v)[1]) / (2 * h)
            an = s.residual_vjp(U, lam) @ v
            assert abs(fd - an) <= 1e-7 * abs(an), (fd, an)


@pytest.mark.parametrize("case_name", ["noslip_p3", "walls_inout_p2", "bump_p2_q2"])
def test_step_vjp_with_heat_matches_fd(case_name):
    case = next(c for c in CASES if c.name == case_name)
    rng = np.random.default_rng(13)
    dt = 1e-3
    with solver(case) as s:
        s.set_prandtl(PR)
        U = case.U
        w, v = rng.standard_normal(U.size), rng.standard_normal(U.size)
        h = 1e-6
        fd = w @ (_step(s, U + h * v, dg.RK4, dt) - _step(s, U - h * v, dg.RK4, dt)) / (2 * h)
        Ud = torch.tensor(U, device="cuda")
        lam = torch.tensor(w, device="cuda")
        torch.cuda.synchronize()
        s.step_vjp_device(dg.RK4, dt, Ud.data_ptr(), lam.data_ptr())
        an = lam.cpu().numpy() @ v
    assert abs(fd - an) <= 1e-7 * abs(an), (fd, an)


def test_n_step_adjoint_with_heat_matches_fd():
    case = _tgv_case()
    N, dt = 10, 5e-3
    rng = np.random.default_rng(14)
    w, v = rng.standard_normal(case.U.size), rng.standard_normal(case.U.size)
    with solver(case) as s:
        s.set_prandtl(PR)
        s.set_state(case.U)
        s.forward_record(dg.RK4, dt, N, 3)
        g = s.backward(w)
        s.set_state(case.U)
        s.forward_record_stages(dg.RK4, dt, N)
        assert np.array_equal(s.backward(w), g)
        h = 1e-6
        fd = w @ (_step(s, case.U + h * v, dg.RK4, dt, N) - _step(s, case.U - h * v, dg.RK4, dt, N)) / (2 * h)
    assert abs(fd - g @ v) <= 1e-6 * abs(fd), (fd, g @ v)


def test_mixed_form_with_heat_tracks_fp64():
    """TGV 8^3, p = 3, Re 1600, Pr 0.71, 200 RK4 steps: the mixed form stays
    within 1e-6 relative L2 of the FP64 form, both with the heat flux."""
    n, p = 8, 3
    nodes = C.box_nodes(n, n, n, 1, 2 * math.pi, 2 * math.pi, 2 * math.pi)
    prm = C.params(mu=1.0 / 1600.0, c=10.0, u=0.0)
    U0 = C.taylor_green(C.node_coords(n, n, n, p, 1, nodes)).reshape(-1)
    case = C.Case("tgv8", n, n, n, p, 1, nodes, [C.P_] * 6, prm, U0)
    out = {}
    for prec in (dg.FP64, dg.MIXED_FP32):
        with solver(case, prec) as s:
            s.set_prandtl(PR)
            out[prec] = _step(s, U0, dg.RK4, 1e-3, 200)
    with solver(case) as s:
        plain = _step(s, U0, dg.RK4, 1e-3, 200)
    assert rel(out[dg.FP64], plain) > 1e-9, "the heat flux changes the run"
    assert rel(out[dg.MIXED_FP32], out[dg.FP64]) < 1e-6, rel(out[dg.MIXED_FP32], out[dg.FP64])


def test_changing_prandtl_drops_graphs_and_the_record():
    case = _tgv_case()
    dt, N = 5e-3, 4
    with solver(case) as s:
        s.set_prandtl(PR)
        fresh = _step(s, case.U, dg.RK4, dt, N)
    with solver(case) as s:
        plain = _step(s, case.U, dg.RK4, dt, N)  # captures the plain step graph
        s.set_prandtl(PR)
        assert np.array_equal(_step(s, case.U, dg.RK4, dt, N), fresh)
        s.set_prandtl(0.0)
        assert np.array_equal(_step(s, case.U, dg.RK4, dt, N), plain)
        s.set_state(case.U)
        s.forward_record(dg.RK4, dt, N, 2)
        s.set_prandtl(PR)
        with pytest.raises(dg.DgbError):
            s.backward(np.ones(case.U.size))


# ------------------------------------------------------ isothermal walls (-8)
# An extension: the reference's no-slip wall keeps the interior energy
# (bound_states.cpp:42-49).  Ghost state: interior density, zero velocity,
# temperature Tw.

ISO = dg.ISOTHERMAL_WALL


def _channel(T_gas_over_Tw=1.0, n=(3, 4, 2), p=3, mu=2e-2, rng_amp=0.0, seed=0):
    """Periodic x/z, isothermal walls at y = 0, 1; gas at rest at uniform
    pressure and temperature T_gas_over_Tw * Tw (Tw = the reference T)."""
    nx, ny, nz = n
    prm = C.params(mu=mu, c=1.0, u=0.0)
    p0, Tref = prm[5], prm[4]
    nodes = C.box_nodes(nx, ny, nz, 1, 1.0, 1.0, 1.0)
    E, nb = nx * ny * nz, (p + 1) ** 3
    Tg = T_gas_over_Tw * Tref
    rho = np.full((E, nb), p0 / (prm[1] * Tg))
    z = np.zeros((E, nb))
    U = C.state_from_primitives(rho, z, z, z, p0 + z, prm[0])
    if rng_amp:
        rng = np.random.default_rng(seed)
        U = U * (1 + rng_amp * rng.standard_normal(U.shape))
        U[:, 1:4] += rng_amp * rng.standard_normal(U[:, 1:4].shape)
    return C.Case("iso", nx, ny, nz, p, 1, nodes, [C.P_, C.P_, ISO, ISO, C.P_, C.P_], prm, U.reshape(-1))


@pytest.mark.parametrize("Pr", [0.0, PR])
def test_isothermal_wall_keeps_gas_at_its_temperature_at_rest(Pr):
    case = _channel(1.0)
    with solver(case) as s:
        s.set_prandtl(Pr)
        _, f = s.residual(case.U)
    assert np.abs(f).max() < 1e-12 * np.abs(case.U).max()


def test_hot_isothermal_wall_heats_only_with_a_heat_flux():
    """Walls at twice the gas temperature: with the heat flux the total
    energy rises; without it the walls only push (momentum), mass and energy
    stay (sum over nodes of R is the rate of each integral)."""
    case = _channel(0.5)
    tot = {}
    for Pr in (0.0, PR):
        with solver(case) as s:
            s.set_prandtl(Pr)
            R, _ = s.residual(case.U)
        R = R.reshape(case.nelem, 5, case.nb)
        tot[Pr] = (R.sum(axis=(0, 2)), np.abs(R).sum(axis=(0, 2)))
    rate, scale = tot[0.0]
    assert abs(rate[0]) <= 1e-12 * scale[0] and abs(rate[4]) <= 1e-12 * scale[4]
    rate, scale = tot[PR]
    assert abs(rate[0]) <= 1e-12 * scale[0]
    assert -rate[4] > 1e-3 * scale[4], "energy flows in (R is minus the rate)"


def test_wall_temperature_setter():
    case = _channel(1.0)
    with solver(case) as s:
        _, f0 = s.residual(case.U)
        s.set_wall_temperature(2.0 * case.prm[4])
        _, f1 = s.residual(case.U)
        assert np.abs(f1).max() > 0.0
        s.set_wall_temperature(case.prm[4])
        assert np.array_equal(s.residual(case.U)[1], f0)
        for bad in (0.0, -1.0, math.nan, math.inf):
            with pytest.raises(dg.DgbError):
                s.set_wall_temperature(bad)


@pytest.mark.parametrize("Pr", [0.0, PR])
def test_residual_vjp_dot_product_with_isothermal_walls(Pr):
    case = _channel(0.8, rng_amp=0.05)
    rng = np.random.default_rng(15)
    with solver(case) as s:
        s.set_prandtl(Pr)
        s.set_wall_temperature(1.2 * case.prm[4])
        U = case.U
        for _ in range(2):
            lam = rng.standard_normal(U.size)
            v = rng.standard_normal(U.size) * np.maximum(np.abs(U), 1.0)
            h = 1e-6
            fd = lam @ (s.residual(U + h * v)[1] - s.residual(U - h * v)[1]) / (2 * h)
            an = s.residual_vjp(U, lam) @ v
            assert abs(fd - an) <= 1e-7 * abs(an), (fd, an)


def test_wall_temperature_gradient_matches_fd():
    """dJ/dTw (dgb_backward_params) against central differences of the run
    with the wall temperature moved, with the heat flux on; J = w . U_N."""
    case = _channel(0.8, rng_amp=0.02)
    N, dt = 6, 1e-3
    Tw = 1.2 * case.prm[4]
    w = np.random.default_rng(16).standard_normal(case.U.size)
    with solver(case) as s:
        s.set_prandtl(PR)
        s.set_wall_temperature(Tw)
        s.set_state(case.U)
        s.forward_record(dg.TVDRK3, dt, N, 2)
        _, dp = s.backward_params(w)

        def J(t):
            s.set_wall_temperature(t)
            return float(w @ _step(s, case.U, dg.TVDRK3, dt, N))

        h = 1e-4 * Tw
        fd = (J(Tw + h) - J(Tw - h)) / (2 * h)
    assert abs(dp[dg.DPARAM_TWALL] - fd) <= 1e-6 * abs(fd), (dp[dg.DPARAM_TWALL], fd)


def test_mesh_without_isothermal_walls_has_zero_wall_gradient():
    case = _tgv_case()
    with solver(case) as s:
        s.set_state(case.U)
        s.forward_record(dg.RK4, 5e-3, 2, 2)
        _, dp = s.backward_params(np.ones(case.U.size))
    assert dp[dg.DPARAM_TWALL] == 0.0
