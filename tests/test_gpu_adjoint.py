"""The hand-written discrete adjoint on the GPU, through the C ABI.

  residual VJP   the full vector (df/dU)^T lam against central-difference
                 Jacobians of dgb_residual on tiny meshes (every entry), and
                 dot-product tests <lam, J v> = <J^T lam, v> on every residual
                 case (all boundary types, affine and curved, p = 0..6)
  step VJP       one RK4 / TVD-RK3 step against central differences of dgb_step
  N steps        dgb_forward_record / dgb_backward against central differences,
                 bit-identical gradients for every checkpoint budget, and the
                 recomputation count of the binomial plan
  torch          the autograd.Function wrappers
  functional     gradient of the final enstrophy w.r.t. Fourier-mode amplitudes
                 against central differences of the same runs and against
                 central differences of the reference's own FP64 CPU solver

Tolerance: relative 1e-7 for the VJPs (central differences in FP64 at
h ~ 1e-6 leave ~1e-9), 1e-6 over N steps, 1e-5 (the bound asked of the
adjoint) for the enstrophy gradient.
"""
import math

import numpy as np
import pytest

import dgpr_b200 as dg
import oracle
from tests import cases as C

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def solver(c, precision=dg.FP64):
    return dg.Solver(dg.Mesh(c.nx, c.ny, c.nz, c.p, c.q, c.nodes, c.bounds), dg.Params.from_array(c.prm), precision)


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def tiny_cases():
    rng = np.random.default_rng(77)
    visc = C.params(mu=2e-2, c=1.0, u=0.3, v=0.1, w=-0.2)
    out = []
    for name, dims, p, L, bounds, prm, shear in [
        ("periodic_p1", (2, 1, 1), 1, (1.0, 0.5, 0.5), [C.P_] * 6, visc, 0.0),
        ("walls_p1", (2, 2, 1), 1, (1.0, 1.0, 0.5), [C.F_, C.F_, C.W_, C.NS_, C.P_, C.P_], visc, 0.0),
        ("sheared_p1", (1, 2, 1), 1, (0.5, 1.0, 0.5), [C.P_] * 6, visc, 0.25),
        ("euler_p2", (1, 1, 2), 2, (0.5, 0.5, 1.0), [C.P_] * 6, C.params(mu=0.0, u=0.3, v=0.2), 0.0),
    ]:
        nodes = C.box_nodes(*dims, 1, *L, shear=shear)
        U = C.random_state(prm, dims[0] * dims[1] * dims[2], (p + 1) ** 3, rng, 0.05)
        out.append(C.Case(name, *dims, p, 1, nodes, bounds, prm, U))
    # curved: sinusoidally mapped q = 2 elements, periodic; bump channel with walls
    nodes = C.sine_nodes(2, 1, 1, 2, 1.0, 0.5, 0.5, 0.03)
    out.append(C.Case("curved_sine_p1", 2, 1, 1, 1, 2, nodes, [C.P_] * 6, visc,
                      C.random_state(visc, 2, 8, rng, 0.05)))
    nodes = C.bump_nodes(2, 1, 1, 2, 2.0, 1.0, 0.5)
    prm = C.params(mu=2e-2, u=0.3)
    out.append(C.Case("curved_bump_p1", 2, 1, 1, 1, 2, nodes, [C.F_, C.F_, C.NS_, C.W_, C.P_, C.P_], prm,
                      C.random_state(prm, 2, 8, rng, 0.05)))
    return out


@pytest.mark.parametrize("case", tiny_cases(), ids=lambda c: c.name)
def test_residual_vjp_equals_transposed_fd_jacobian(case):
    rng = np.random.default_rng(1)
    with solver(case) as s:
        U = case.U
        lam = rng.standard_normal(U.size)
        vjp = s.residual_vjp(U, lam)
        assert s.last_launch_count == 3
        fd = np.zeros(U.size)
        for j in range(U.size):
            h = 1e-6 * max(1.0, abs(U[j]))
            Up, Um = U.copy(), U.copy()
            Up[j] += h
            Um[j] -= h
            fd[j] = lam @ (s.residual(Up)[1] - s.residual(Um)[1]) / (2 * h)
    assert rel(vjp, fd) < 1e-7, rel(vjp, fd)


ADJ_CASES = C.residual_cases()


@pytest.mark.parametrize("case", ADJ_CASES, ids=lambda c: c.name)
def test_residual_vjp_dot_product(case):
    rng = np.random.default_rng(2)
    with solver(case) as s:
        U = case.U
        for _ in range(3):
            lam = rng.standard_normal(U.size)
            v = rng.standard_normal(U.size) * np.maximum(np.abs(U), 1.0)
            h = 1e-6
            fd = lam @ (s.residual(U + h * v)[1] - s.residual(U - h * v)[1]) / (2 * h)
            an = s.residual_vjp(U, lam) @ v
            assert abs(fd - an) <= 1e-7 * abs(an), (fd, an)


def test_residual_vjp_is_linear_in_lam():
    case = ADJ_CASES[0]
    rng = np.random.default_rng(3)
    with solver(case) as s:
        a, b = rng.standard_normal(case.U.size), rng.standard_normal(case.U.size)
        va, vb = s.residual_vjp(case.U, a), s.residual_vjp(case.U, b)
        vab = s.residual_vjp(case.U, 2.0 * a - 3.0 * b)
    assert rel(vab, 2.0 * va - 3.0 * vb) < 1e-13


def _step(s, U, scheme, dt, n=1):
    s.set_state(U)
    s.step(scheme, dt, n, norms=False)
    return s.get_state()


STEP_CASES = [
    ("periodic_visc", "periodic_p2", 2e-3),
    ("walls_visc", "freestream_p2", 2e-3),
    ("noslip", "noslip_p3", 1e-3),
    ("euler", "euler_p2", 2e-3),
    ("inflow_outflow", "walls_inout_p2", 2e-3),
]


@pytest.mark.parametrize("form", [dg.STEP_GAUSS, dg.STEP_NODAL], ids=["gauss", "nodal"])
@pytest.mark.parametrize("scheme", [dg.RK4, dg.TVDRK3], ids=["rk4", "tvdrk3"])
@pytest.mark.parametrize("name,case_name,dt", STEP_CASES, ids=[c[0] for c in STEP_CASES])
def test_step_vjp_matches_fd(scheme, name, case_name, dt, form):
    """dgb_step_vjp_device is the VJP of dgb_step in its form."""
    case = next(c for c in C.residual_cases() if c.name == case_name)
    rng = np.random.default_rng(4)
    with solver(case) as s:
        s.set_step_form(form)
        U = case.U
        w = rng.standard_normal(U.size)
        v = rng.standard_normal(U.size)
        h = 1e-6
        fd = w @ (_step(s, U + h * v, scheme, dt) - _step(s, U - h * v, scheme, dt)) / (2 * h)
        Ud = torch.tensor(U, device="cuda")
        lam = torch.tensor(w, device="cuda")
        torch.cuda.synchronize()
        s.step_vjp_device(scheme, dt, Ud.data_ptr(), lam.data_ptr())
        an = lam.cpu().numpy() @ v
        assert torch.equal(Ud.cpu(), torch.tensor(U)), "U must be unchanged"
    assert abs(fd - an) <= 1e-7 * abs(an), (fd, an)


def _tgv_case(n=3, p=2, mu=2e-2):
    nodes = C.box_nodes(n, n, n, 1, 2 * math.pi, 2 * math.pi, 2 * math.pi)
    xyz = C.node_coords(n, n, n, p, 1, nodes)
    prm = C.params(mu=mu, c=1.0 / 0.3, u=0.0, v=0.0, w=0.0)
    U = C.taylor_green(xyz, Ma=0.3).reshape(-1)
    return C.Case("tgv", n, n, n, p, 1, nodes, [C.P_] * 6, prm, U)


@pytest.mark.parametrize("form", [dg.STEP_GAUSS, dg.STEP_NODAL], ids=["gauss", "nodal"])
@pytest.mark.parametrize("scheme", [dg.RK4, dg.TVDRK3], ids=["rk4", "tvdrk3"])
def test_n_step_adjoint_fd_and_checkpoint_invariance(scheme, form):
    """The recorded run steps in dgb_step's form (Gauss-point or nodal) and
    the backward sweep reverses that form."""
    case = _tgv_case()
    N, dt = 12, 5e-3
    rng = np.random.default_rng(5)
    with solver(case) as s:
        s.set_step_form(form)
        U0 = case.U
        w = rng.standard_normal(U0.size)
        grads = {}
        for slots in (1, 3, 5, N):
            s.set_state(U0)
            s.forward_record(scheme, dt, N, slots)
            UN = s.get_state()
            grads[slots] = s.backward(w)
            fwd, rev, planned = s.adjoint_stats()
            ops, pfwd, _ = dg.checkpoint_plan(N, slots)
            first = next(k for k, (kind, _) in enumerate(ops) if kind == "reverse")
            rec = sum(a for kind, a in ops[:first] if kind == "forward")
            assert rev == N and planned == pfwd and fwd == pfwd - rec
            assert np.array_equal(s.get_state(), UN), "backward leaves the final state resident"
        s.set_state(U0)
        s.forward_record_stages(scheme, dt, N)
        assert np.array_equal(s.get_state(), UN), "the stage-keeping record computes the same states"
        grads["stages"] = s.backward(w)
        fwd, rev, _ = s.adjoint_stats()
        assert fwd == 0 and rev == N
        ref = _step(s, U0, scheme, dt, N)
        assert np.array_equal(UN, ref), "recorded run equals dgb_step"
        for slots, g in grads.items():
            assert np.array_equal(g, grads[N]), f"gradient depends on the checkpoint budget ({slots})"
        v = rng.standard_normal(U0.size)
        h = 1e-6
        fd = w @ (_step(s, U0 + h * v, scheme, dt, N) - _step(s, U0 - h * v, scheme, dt, N)) / (2 * h)
        an = grads[N] @ v
    assert abs(fd - an) <= 1e-6 * abs(an), (fd, an)


def test_adjoint_forms_agree():
    """The Gauss-point and the nodal forms are one discretisation: their
    recorded runs and gradients agree to rounding (affine TGV, RK4, and the
    sinusoidally mapped mesh, TVD-RK3)."""
    cases = [(_tgv_case(), dg.RK4)]
    n, p, q = 2, 2, 3
    L = 2 * math.pi
    nodes = C.sine_nodes(n, n, n, q, L, L, L, 0.1)
    prm = C.params(mu=2e-2, c=1.0 / 0.3, u=0.0, v=0.0, w=0.0)
    U0 = C.taylor_green(C.node_coords(n, n, n, p, q, nodes), Ma=0.3).reshape(-1)
    cases.append((C.Case("tgv_sine", n, n, n, p, q, nodes, [C.P_] * 6, prm, U0), dg.TVDRK3))
    for case, scheme in cases:
        w = np.random.default_rng(10).standard_normal(case.U.size)
        out = {}
        for form in (dg.STEP_GAUSS, dg.STEP_NODAL):
            with solver(case) as s:
                s.set_step_form(form)
                s.set_state(case.U)
                s.forward_record(scheme, 5e-3, 8, 3)
                out[form] = (s.get_state(), s.backward(w))
        assert rel(out[dg.STEP_GAUSS][0], out[dg.STEP_NODAL][0]) < 1e-13
        assert rel(out[dg.STEP_GAUSS][1], out[dg.STEP_NODAL][1]) < 1e-12, rel(out[dg.STEP_GAUSS][1],
                                                                             out[dg.STEP_NODAL][1])


def test_curved_n_step_adjoint_fd():
    """Sinusoidally mapped (q = 3) periodic TGV, p = 2: every stored-stage and
    checkpointed budget gives the same gradient, which matches central
    differences of the forward run."""
    n, p, q = 2, 2, 3
    L = 2 * math.pi
    nodes = C.sine_nodes(n, n, n, q, L, L, L, 0.1)
    prm = C.params(mu=2e-2, c=1.0 / 0.3, u=0.0, v=0.0, w=0.0)
    U0 = C.taylor_green(C.node_coords(n, n, n, p, q, nodes), Ma=0.3).reshape(-1)
    case = C.Case("tgv_sine", n, n, n, p, q, nodes, [C.P_] * 6, prm, U0)
    N, dt = 8, 5e-3
    rng = np.random.default_rng(8)
    w, v = rng.standard_normal(U0.size), rng.standard_normal(U0.size)
    with solver(case) as s:
        s.set_state(U0)
        s.forward_record(dg.RK4, dt, N, 3)
        g = s.backward(w)
        s.set_state(U0)
        s.forward_record_stages(dg.RK4, dt, N)
        assert np.array_equal(s.backward(w), g)
        h = 1e-6
        fd = w @ (_step(s, U0 + h * v, dg.RK4, dt, N) - _step(s, U0 - h * v, dg.RK4, dt, N)) / (2 * h)
    assert abs(fd - g @ v) <= 1e-6 * abs(fd), (fd, g @ v)


def test_backward_can_repeat_and_needs_a_record():
    case = _tgv_case(n=2)
    with solver(case) as s:
        with pytest.raises(dg.DgbError):
            s.backward(np.ones(case.U.size))
        s.set_state(case.U)
        s.forward_record(dg.RK4, 5e-3, 4, 2)
        a = s.backward(np.ones(case.U.size))
        b = s.backward(np.ones(case.U.size))
    assert np.array_equal(a, b)


def test_torch_wrappers_match_the_c_abi():
    from dgpr_b200 import autograd as dga
    case = _tgv_case()
    rng = np.random.default_rng(6)
    w = torch.tensor(rng.standard_normal(case.U.size), device="cuda")
    with solver(case) as s:
        U0 = torch.tensor(case.U, device="cuda", requires_grad=True)
        J = (w * dga.integrate(U0, s, dg.RK4, 5e-3, 6, slots=2)).sum()
        J.backward()
        s.set_state(case.U)
        s.forward_record(dg.RK4, 5e-3, 6, 2)
        ref = s.backward(w.cpu().numpy())
        assert np.array_equal(U0.grad.cpu().numpy(), ref)
        U1 = torch.tensor(case.U, device="cuda", requires_grad=True)
        (w * dga.residual(U1, s)).sum().backward()
        assert np.array_equal(U1.grad.cpu().numpy(), s.residual_vjp(case.U, w.cpu().numpy()))
        f = dga.residual(torch.tensor(case.U, device="cuda"), s)
        assert np.array_equal(f.cpu().numpy(), s.residual(case.U)[1])


def test_stale_record_raises():
    from dgpr_b200 import autograd as dga
    case = _tgv_case(n=2)
    with solver(case) as s:
        U0 = torch.tensor(case.U, device="cuda", requires_grad=True)
        y1 = dga.integrate(U0, s, dg.RK4, 5e-3, 3)
        dga.integrate(U0.detach(), s, dg.RK4, 5e-3, 3)
        with pytest.raises(dg.DgbError):
            y1.sum().backward()


def _fourier_setup(n, p, Re=500.0, Ma=0.3):
    from dgpr_b200 import functionals as F
    L = 2 * math.pi
    c = 1.0 / Ma
    prm = C.params(mu=1.0 / Re, c=c, u=1.0, v=0.0, w=0.0)
    nodes = C.box_nodes(n, n, n, 1, L, L, L)
    xyz = F.box_node_coords(n, n, n, p, L, L, L)
    gamma, rho = 1.4, 1.0
    modes = F.FourierModes(xyz, gamma, rho, prm[5], (1.0, 0.0, 0.0), nmodes=8, kmax=4, amp=0.05, seed=0,
                           device="cuda")
    quad = F.BoxQuadrature(n, n, n, p, L, L, L, device="cuda")
    case = C.Case("fourier", n, n, n, p, 1, nodes, [C.P_] * 6, prm, None)
    return case, modes, quad, F


def test_enstrophy_gradient_wrt_mode_amplitudes():
    from dgpr_b200 import autograd as dga
    case, modes, quad, F = _fourier_setup(4, 2)
    N, dt = 20, 4e-3
    with solver(case) as s:
        a = modes.amplitudes("cuda").requires_grad_(True)
        J = F.enstrophy(dga.integrate(modes.state(a), s, dg.RK4, dt, N, slots=5), quad)
        J.backward()
        g = a.grad.cpu().numpy()

        def Jof(av):
            with torch.no_grad():
                return float(F.enstrophy(dga.integrate(modes.state(av), s, dg.RK4, dt, N), quad))

        fd = np.zeros_like(g)
        h = 1e-5
        for m in range(g.shape[0]):
            for c in range(3):
                ap, am = a.detach().clone(), a.detach().clone()
                ap[m, c] += h
                am[m, c] -= h
                fd[m, c] = (Jof(ap) - Jof(am)) / (2 * h)
    assert np.max(np.abs(g - fd)) <= 1e-5 * np.max(np.abs(fd)), (g, fd)


def test_enstrophy_gradient_against_reference_solver_fd():
    ref = oracle.reference()
    if ref is None:
        pytest.skip("reference solver not built here")
    from dgpr_b200 import autograd as dga
    case, modes, quad, F = _fourier_setup(3, 2)
    N, dt = 8, 4e-3
    rng = np.random.default_rng(7)
    d = rng.standard_normal((8, 3))
    mesh = oracle.Mesh(case.nx, case.ny, case.nz, case.p, case.q, case.nodes, case.bounds)
    with solver(case) as s:
        a = modes.amplitudes("cuda").requires_grad_(True)
        J = F.enstrophy(dga.integrate(modes.state(a), s, dg.RK4, dt, N), quad)
        J.backward()
        an = float((a.grad.cpu().numpy() * d).sum())

    def Jref(av):
        U0 = modes.state(av).cpu().numpy()
        UN, _ = ref.run(mesh, case.prm, U0, dg.RK4, dt, N)
        return float(F.enstrophy(torch.tensor(UN, device="cuda"), quad))

    h = 1e-5
    a0 = modes.amplitudes("cuda")
    dd = torch.tensor(d, device="cuda")
    fd = (Jref(a0 + h * dd) - Jref(a0 - h * dd)) / (2 * h)
    assert abs(fd - an) <= 1e-5 * abs(fd), (fd, an)


def test_mixed_precision_adjoint_tracks_the_fp64_gradient():
    """A mixed-precision handle recomputes its states in FP32 and applies the
    FP64 adjoint at them (FP32 forward, FP64 adjoint accumulation): its
    gradient stays within 1e-5 relative L2 of the FP64 handle's, for the
    checkpointed and the stage-keeping records alike."""
    case = _tgv_case()
    N, dt = 12, 5e-3
    w = np.random.default_rng(9).standard_normal(case.U.size)
    grads = {}
    for prec in (dg.FP64, dg.MIXED_FP32):
        with solver(case, prec) as s:
            s.set_state(case.U)
            s.forward_record(dg.RK4, dt, N, 4)
            g = s.backward(w)
            s.set_state(case.U)
            s.forward_record_stages(dg.RK4, dt, N)
            assert np.array_equal(s.backward(w), g)
            grads[prec] = g
    assert rel(grads[dg.MIXED_FP32], grads[dg.FP64]) < 1e-5, rel(grads[dg.MIXED_FP32], grads[dg.FP64])
