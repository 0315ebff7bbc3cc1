"""Parameter gradients of the recorded run (dgb_backward_params): dJ/dmu at
a fixed Prandtl number and dJ/dsource[0..4], through the C ABI, against
central differences of the forward run with the parameter moved by
dgb_set_params.

  J = w . U_N after N RK steps, relative tolerance 1e-6 (FD step 1e-5;
  f is affine in mu and in the source, so the central difference is exact
  up to the stepping's own nonlinearity and roundoff).  Also: the gradient
  is bit-identical for every checkpoint budget and the stage-keeping
  record, dJ/dU_0 equals dgb_backward's, and the torch wrapper returns the
  same numbers.
"""
import math

import numpy as np
import pytest

import dgpr_b200 as dg
from tests import cases as C

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def solver(c, precision=dg.FP64):
    return dg.Solver(dg.Mesh(c.nx, c.ny, c.nz, c.p, c.q, c.nodes, c.bounds), dg.Params.from_array(c.prm), precision)


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _tgv_case(n=3, p=2, mu=2e-2, source=(0, 0, 0, 0, 0)):
    nodes = C.box_nodes(n, n, n, 1, 2 * math.pi, 2 * math.pi, 2 * math.pi)
    xyz = C.node_coords(n, n, n, p, 1, nodes)
    prm = C.params(mu=mu, c=1.0 / 0.3, u=0.0, v=0.0, w=0.0, source=source)
    U = C.taylor_green(xyz, Ma=0.3).reshape(-1)
    return C.Case("tgv", n, n, n, p, 1, nodes, [C.P_] * 6, prm, U)


def _J(s, prm, U0, w, scheme, dt, N):
    s.set_params(prm)
    s.set_state(U0)
    s.step(scheme, dt, N, norms=False)
    return float(w @ s.get_state())


def _fd_params(s, case, w, scheme, dt, N, which):
    """Central differences of J in the parameters `which` (indices into
    [mu, source[0..4]])."""
    base = np.array(case.prm, dtype=np.float64)
    out = {}
    for k in which:
        idx = 2 if k == 0 else 10 + k  # mu, or source[k - 1] at 11..15
        h = 1e-5
        pp, pm = base.copy(), base.copy()
        pp[idx] += h
        pm[idx] -= h
        out[k] = (_J(s, pp, case.U, w, scheme, dt, N) - _J(s, pm, case.U, w, scheme, dt, N)) / (2 * h)
    s.set_params(base)
    return out


def _check(an, fd, which, tol=1e-6):
    scale = max(abs(fd[k]) for k in which)
    for k in which:
        assert abs(an[k] - fd[k]) <= tol * max(abs(fd[k]), 1e-2 * scale), (k, an[k], fd[k])


@pytest.mark.parametrize("scheme", [dg.RK4, dg.TVDRK3], ids=["rk4", "tvdrk3"])
def test_param_gradient_matches_fd_and_is_budget_independent(scheme):
    case = _tgv_case(source=(0.0, 0.1, 0.0, 0.0, 0.05))
    N, dt = 8, 5e-3
    rng = np.random.default_rng(31)
    w = rng.standard_normal(case.U.size)
    with solver(case) as s:
        grads = {}
        for slots in (1, 3, N, "stages"):
            s.set_state(case.U)
            if slots == "stages":
                s.forward_record_stages(scheme, dt, N)
            else:
                s.forward_record(scheme, dt, N, slots)
            grads[slots] = s.backward_params(w)
        g_plain = s.backward(w)
        fd = _fd_params(s, case, w, scheme, dt, N, range(6))
    for slots, (g, dp) in grads.items():
        assert np.array_equal(g, grads[N][0]) and np.array_equal(dp, grads[N][1]), slots
    assert np.array_equal(grads[N][0], g_plain), "dJ/dU_0 equals dgb_backward's"
    _check(grads[N][1], fd, range(6))


def test_viscosity_gradient_with_heat_flux():
    """mu at a fixed Prandtl number: the heat coefficient mu gamma / Pr moves
    with it, in the forward run and in the gradient."""
    case = _tgv_case()
    N, dt = 8, 5e-3
    w = np.random.default_rng(32).standard_normal(case.U.size)
    with solver(case) as s:
        s.set_prandtl(0.71)
        s.set_state(case.U)
        s.forward_record(dg.RK4, dt, N, 3)
        _, dp = s.backward_params(w)
        fd = _fd_params(s, case, w, dg.RK4, dt, N, [0])
        s.set_prandtl(0.0)
        s.set_state(case.U)
        s.forward_record(dg.RK4, dt, N, 3)
        _, dp0 = s.backward_params(w)
    _check(dp, fd, [0])
    assert abs(dp[0] - dp0[0]) > 1e-6 * abs(dp0[0]), "the heat flux changes dJ/dmu"


def test_viscosity_gradient_of_an_inviscid_run():
    """An Euler handle (mu = 0) still has dJ/dmu: the derivative of the run
    at zero viscosity (the FD run at -h has negative viscosity, which the
    affine residual does not mind)."""
    case = _tgv_case(mu=0.0)
    N, dt = 6, 5e-3
    w = np.random.default_rng(33).standard_normal(case.U.size)
    with solver(case) as s:
        s.set_state(case.U)
        s.forward_record(dg.RK4, dt, N, 2)
        _, dp = s.backward_params(w)
        fd = _fd_params(s, case, w, dg.RK4, dt, N, [0, 2])
    _check(dp, fd, [0, 2])


def test_param_gradient_on_walls_and_curved_elements():
    cases = C.residual_cases()
    ns = next(c for c in cases if c.name == "noslip_p3")
    ns.prm = np.array(ns.prm)
    ns.prm[12] = 0.1  # body force in x
    curved = next(c for c in cases if c.name == "bump_p2_q2")
    for case, dt in ((ns, 1e-3), (curved, 1e-3)):
        N = 4
        w = np.random.default_rng(34).standard_normal(case.U.size)
        with solver(case) as s:
            s.set_state(case.U)
            s.forward_record(dg.TVDRK3, dt, N, 2)
            _, dp = s.backward_params(w)
            fd = _fd_params(s, case, w, dg.TVDRK3, dt, N, [0, 2, 5])
        _check(dp, fd, [0, 2, 5])


def test_mixed_precision_param_gradient_tracks_fp64():
    case = _tgv_case(source=(0.0, 0.1, 0.0, 0.0, 0.0))
    N, dt = 8, 5e-3
    w = np.random.default_rng(35).standard_normal(case.U.size)
    out = {}
    for prec in (dg.FP64, dg.MIXED_FP32):
        with solver(case, prec) as s:
            s.set_state(case.U)
            s.forward_record(dg.RK4, dt, N, 3)
            out[prec] = s.backward_params(w)[1]
    assert rel(out[dg.MIXED_FP32], out[dg.FP64]) < 1e-5, (out[dg.MIXED_FP32], out[dg.FP64])


def test_torch_theta_gradient_matches_the_c_abi():
    from dgpr_b200 import autograd as dga
    case = _tgv_case()
    N, dt = 6, 5e-3
    rng = np.random.default_rng(36)
    w = torch.tensor(rng.standard_normal(case.U.size), device="cuda")
    theta = torch.tensor([3e-2, 0.0, 0.05, 0.0, 0.0, 0.01], dtype=torch.float64, requires_grad=True)
    with solver(case) as s:
        U0 = torch.tensor(case.U, device="cuda", requires_grad=True)
        J = (w * dga.integrate(U0, s, dg.RK4, dt, N, slots=2, theta=theta)).sum()
        J.backward()
        assert s.params.mu == 3e-2 and list(s.params.source) == [0.0, 0.05, 0.0, 0.0, 0.01]
        s.set_state(case.U)
        s.forward_record(dg.RK4, dt, N, 2)
        g, dp = s.backward_params(w.cpu().numpy())
    assert np.array_equal(U0.grad.cpu().numpy(), g)
    assert np.array_equal(theta.grad.numpy(), dp[:6])


def test_set_params_keeps_geometry_and_drops_the_record():
    case = _tgv_case()
    with solver(case) as s:
        s.set_state(case.U)
        s.forward_record(dg.RK4, 5e-3, 3, 2)
        s.set_params(case.prm)  # unchanged parameters: the record stays
        s.backward(np.ones(case.U.size))
        p = np.array(case.prm)
        p[2] *= 2.0
        s.set_params(p)
        with pytest.raises(dg.DgbError):
            s.backward(np.ones(case.U.size))
        s.set_state(case.U)
        s.step(dg.RK4, 5e-3, 3, norms=False)
        a = s.get_state()
    c2 = _tgv_case(mu=case.prm[2] * 2.0)
    with solver(c2) as s2:
        s2.set_state(case.U)
        s2.step(dg.RK4, 5e-3, 3, norms=False)
        b = s2.get_state()
    assert np.array_equal(a, b), "set_params equals creating the handle with those parameters"
