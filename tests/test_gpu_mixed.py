"""The mixed form (FP32 contractions, traces and fluxes; FP64 geometry,
inverse mass matrix, RK accumulation and state) against the FP64 form and the
oracle.

Tolerances:
  one residual, relative L2 vs the FP64 oracle       2e-5  (FP32 arithmetic;
      the flux divergence of the large background pressure cancels, so f is
      relatively less accurate than the state)
  state after 1000 RK4 steps of a Taylor-Green vortex,
      relative L2 vs the FP64 form                    1e-6  (the required bound)
"""
import numpy as np
import pytest

import dgpr_b200 as dg
import oracle
from tests import cases as C

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def solver(c, precision):
    return dg.Solver(dg.Mesh(c.nx, c.ny, c.nz, c.p, c.q, c.nodes, c.bounds), dg.Params.from_array(c.prm), precision)


@pytest.mark.parametrize("case", [c for c in C.residual_cases() if c.name in
                                  ("periodic_p2", "periodic_p3_q2", "sheared_p2", "walls_inout_p2",
                                   "freestream_p2", "noslip_p3", "p4", "euler_p2", "source_p2",
                                   "bump_p2_q2", "sine_periodic_p2_q2")],
                         ids=lambda c: c.name)
def test_mixed_residual_close_to_oracle(case):
    with solver(case, dg.MIXED_FP32) as s:
        R, f = s.residual(case.U)
    Ro, fo = oracle.restatement().residual(oracle.Mesh(case.nx, case.ny, case.nz, case.p, case.q, case.nodes,
                                                       case.bounds), case.prm, case.U)
    assert rel(R, Ro) < 2e-5, rel(R, Ro)
    assert rel(f, fo) < 2e-5, rel(f, fo)


def _tgv(n, p):
    L = 2 * np.pi
    nodes = C.box_nodes(n, n, n, 1, L, L, L)
    prm = C.params(mu=1.0 / 1600.0, c=10.0, u=0.0)
    U = C.taylor_green(C.node_coords(n, n, n, p, 1, nodes)).reshape(-1)
    dt = 0.2 * (L / n) / ((2 * p + 1) * 11.0)
    return C.Case("tgv", n, n, n, p, 1, nodes, [C.P_] * 6, prm, U), dt


@pytest.mark.parametrize("n,p", [(8, 3), (6, 4)])
def test_mixed_tgv_1000_steps_within_1e6_of_fp64(n, p):
    c, dt = _tgv(n, p)
    out = {}
    for prec in (dg.FP64, dg.MIXED_FP32):
        with solver(c, prec) as s:
            s.set_state(c.U)
            s.step(dg.RK4, dt, 1000, norms=False)
            out[prec] = s.get_state()
    err = rel(out[dg.MIXED_FP32], out[dg.FP64])
    assert err < 1e-6, err


def test_mixed_time_steps_track_reference_fixture():
    c = [k for k in C.run_cases() if k.name == "channel_tvdrk3"][0]
    gold = np.load(__import__("os").path.join(__import__("os").path.dirname(__file__), "golden", "golden.npz"))
    with solver(c, dg.MIXED_FP32) as s:
        s.set_state(c.U)
        s.step(c.scheme, c.dt, c.nsteps)
        U = s.get_state()
    assert rel(U, gold[f"{c.name}/UN"]) < 1e-7


def test_mixed_at_the_48_cubed_p4_configuration():
    """The mixed-precision configuration's size (TGV, 48^3 hexes, p = 4): after
    200 RK4 steps the mixed state is within 1e-6 (relative L2) of the FP64
    form's, and the kinetic-energy history (dissipation) agrees to 1e-7."""
    import math

    import torch

    from dgpr_b200 import functionals as F
    c, dt = _tgv(48, 4)
    L = 2 * math.pi
    quad = F.BoxQuadrature(48, 48, 48, 4, L, L, L, device="cuda")
    out, ke = {}, {}
    for prec in (dg.FP64, dg.MIXED_FP32):
        with solver(c, prec) as s:
            s.set_state(c.U)
            hist = []
            for _ in range(4):
                s.step(dg.RK4, dt, 50, norms=False)
                hist.append(float(F.kinetic_energy(torch.tensor(s.get_state(), device="cuda"), quad)))
            out[prec] = s.get_state()
            ke[prec] = np.array(hist)
    err = rel(out[dg.MIXED_FP32], out[dg.FP64])
    assert err < 1e-6, err
    assert np.max(np.abs(ke[dg.MIXED_FP32] - ke[dg.FP64])) < 1e-7 * np.max(np.abs(ke[dg.FP64]))
    assert np.all(np.diff(ke[dg.FP64]) < 0), "viscous TGV dissipates kinetic energy"
