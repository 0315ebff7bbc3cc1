"""The mixed form's stage with tensor-core volume contractions
(DGB_STEP_GAUSS_TC: tcgen05 kind::tf32, three TF32 products per term, FP32
accumulation) against the FP64 form and the FP32x2 mixed stage.

Tolerances:
  state after 1000 RK4 steps of a Taylor-Green vortex,
      relative L2 vs the FP64 form                    1e-6  (the mixed form's bound)
  state after 10 steps, relative L2 vs the default
      mixed stage (same arithmetic but the contractions)  2e-7
"""
import numpy as np
import pytest

import dgpr_b200 as dg
from tests import cases as C
from tests.test_gpu_mixed import _tgv, rel, solver

pytestmark = pytest.mark.gpu


def _run(c, dt, precision, form, nsteps, scheme=dg.RK4):
    with solver(c, precision) as s:
        s.set_step_form(form)
        s.set_state(c.U)
        s.step(scheme, dt, nsteps, norms=False)
        return s.get_state()


@pytest.mark.parametrize("n,p", [(8, 3), (6, 4)])
def test_tc_tgv_1000_steps_within_1e6_of_fp64(n, p):
    c, dt = _tgv(n, p)
    ref = _run(c, dt, dg.FP64, dg.STEP_GAUSS, 1000)
    err = rel(_run(c, dt, dg.MIXED_FP32, dg.STEP_GAUSS_TC, 1000), ref)
    assert err < 1e-6, err


@pytest.mark.parametrize("n,p,scheme", [(6, 3, dg.RK4), (5, 3, dg.TVDRK3), (4, 4, dg.RK4)])
def test_tc_close_to_the_ffma_mixed_stage(n, p, scheme):
    """Odd element counts take the scalar FP32 stage; even ones the paired one."""
    c, dt = _tgv(n, p)
    a = _run(c, dt, dg.MIXED_FP32, dg.STEP_GAUSS_TC, 10, scheme)
    b = _run(c, dt, dg.MIXED_FP32, dg.STEP_GAUSS, 10, scheme)
    assert rel(a, b) < 2e-7, rel(a, b)
    assert rel(a, b) > 0  # a different kernel ran


@pytest.mark.parametrize("name", ["noslip_p3", "p4"])
def test_tc_walls_and_general_states(name):
    """No-slip walls and a non-uniform sheared state through the tensor-core
    stage (the face and boundary code is the FP32 stage's own), against the
    FP64 form after 5 steps."""
    c = [k for k in C.residual_cases() if k.name == name][0]
    a = _run(c, 1e-4, dg.MIXED_FP32, dg.STEP_GAUSS_TC, 5)
    b = _run(c, 1e-4, dg.FP64, dg.STEP_GAUSS, 5)
    assert rel(a, b) < 1e-6, rel(a, b)


def test_tc_form_rejected_where_not_built():
    c, dt = _tgv(4, 3)
    with solver(c, dg.FP64) as s:
        with pytest.raises(dg.DgbError) as ex:
            s.set_step_form(dg.STEP_GAUSS_TC)
        assert ex.value.code == dg.ERR_UNSUPPORTED
    c2, _ = _tgv(4, 2)
    with solver(c2, dg.MIXED_FP32) as s:
        with pytest.raises(dg.DgbError):
            s.set_step_form(dg.STEP_GAUSS_TC)
    with solver(c, dg.MIXED_FP32) as s:  # the heat flux cannot be switched on under the form
        s.set_step_form(dg.STEP_GAUSS_TC)
        with pytest.raises(dg.DgbError) as ex:
            s.set_prandtl(0.71)
        assert ex.value.code == dg.ERR_UNSUPPORTED
        s.set_step_form(dg.STEP_GAUSS)
        s.set_prandtl(0.71)


@pytest.mark.parametrize("n", [4, 3], ids=["even", "odd"])
def test_tc_step_host_equals_set_step_get(n):
    """dgb_step_host runs the tensor-core stage in pieces of elements (its
    last stage): the same bits as the plain calls."""
    c, dt = _tgv(n, 3)
    with solver(c, dg.MIXED_FP32) as s:
        s.set_step_form(dg.STEP_GAUSS_TC)
        s.set_state(c.U)
        norms_a = s.step(dg.RK4, dt, 2)
        Ua = s.get_state()
    with solver(c, dg.MIXED_FP32) as s:
        s.set_step_form(dg.STEP_GAUSS_TC)
        Uout = np.zeros(c.U.size)
        norms_b = s.step_host(dg.RK4, dt, 2, np.array(c.U, dtype=np.float64), Uout)
    assert np.array_equal(Uout, Ua)
    assert np.array_equal(norms_b, norms_a[:2])
