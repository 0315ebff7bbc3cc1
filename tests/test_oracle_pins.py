"""Pins the CPU oracle (oracle/dg_oracle.c) to the reference: against the
committed fixtures made by the unmodified reference solver
(tests/golden/make_golden.py), and, where the reference has been built here,
against live reference runs including curved (bump) geometry."""
import os

import numpy as np
import pytest

import oracle
from tests import cases as C

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "golden.npz"))
O = oracle.restatement()


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def omesh(c):
    return oracle.Mesh(c.nx, c.ny, c.nz, c.p, c.q, c.nodes, c.bounds)


@pytest.mark.parametrize("case", C.residual_cases(), ids=lambda c: c.name)
def test_oracle_residual_matches_reference_fixture(case):
    assert np.array_equal(GOLD[f"{case.name}/U"], case.U)
    R, f = O.residual(omesh(case), case.prm, case.U)
    assert rel(R, GOLD[f"{case.name}/R"]) < 1e-13
    # f = -Minv R: both invert the dense mass matrix by Gauss-Jordan, with
    # different pivot arithmetic; at p = 6 its condition number reaches ~1e3
    assert rel(f, GOLD[f"{case.name}/f"]) < 1e-12


@pytest.mark.parametrize("case", C.run_cases(), ids=lambda c: c.name)
def test_oracle_time_steps_match_reference_fixture(case):
    U, norms = O.run(omesh(case), case.prm, case.U, case.scheme, case.dt, case.nsteps)
    assert rel(U, GOLD[f"{case.name}/UN"]) < 1e-14
    assert rel(norms, GOLD[f"{case.name}/norms"]) < 1e-12


def test_oracle_matches_live_reference_on_curved_bump_mesh():
    ref = oracle.reference()
    if ref is None:
        pytest.skip("reference not built here")
    rng = np.random.default_rng(11)
    for (nx, ny, nz, p, q, bounds) in [(3, 2, 2, 2, 2, [-5, -6, -4, -4, -2, -2]),
                                       (2, 3, 1, 3, 3, [-3, -3, -7, -4, -2, -2])]:
        nodes = np.zeros(nx * ny * nz * (q + 1) ** 3 * 3)
        ref.lib.ref_bump_nodes(nx, ny, nz, p, q, 2.0, 1.0, 1.0, 0.3, 0.1, 1.0, 0.05, oracle._p(nodes))
        m = oracle.Mesh(nx, ny, nz, p, q, nodes, bounds)
        prm = C.params(mu=1e-2, u=0.3)
        U = C.random_state(prm, m.nelem, m.nb, rng, 0.03)
        Ro, fo = O.residual(m, prm, U)
        Rr, fr = ref.residual(m, prm, U)
        assert rel(Ro, Rr) < 1e-13 and rel(fo, fr) < 1e-13


def test_oracle_detects_planted_mistake():
    """The checker can fail: a planted error in the oracle's input (one state
    coefficient perturbed) is visible in the residual comparison."""
    c = C.residual_cases()[0]
    U = c.U.copy()
    U[17] *= 1.0 + 1e-9
    _, f = O.residual(omesh(c), c.prm, U)
    assert rel(f, GOLD[f"{c.name}/f"]) > 1e-13
