"""dgb_residual_noalloc: the residual for callers that may not allocate GPU
memory (a host application owning the device memory pool, or a solver that
has claimed all of HBM).  It keeps its scratch in a fixed 32 MiB device array
built into the library instead of cudaMalloc'd per-mesh buffers.

Checked through the C ABI against the ordinary entry point (dgb_residual),
within the parity tolerance of the FP64 tests (1e-11 relative L2; in practice
the two run the same kernels and agree exactly), on two calls in a row with
different meshes, so stale contents of the shared array would show.  This
file is collected last; it also passes alone in a fresh process.  Each call
looks up the static array's device address itself (no cached set-up)."""
import ctypes

import numpy as np
import pytest

import dgpr_b200 as dg
from tests import cases as C

pytestmark = pytest.mark.gpu


def _noalloc(c, U):
    import torch
    L = dg.lib()
    fn = L.dgb_residual_noalloc
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.POINTER(dg.MeshDesc), ctypes.POINTER(dg.Params), ctypes.c_void_p, ctypes.c_void_p,
                   ctypes.c_void_p]
    mesh = dg.Mesh(c.nx, c.ny, c.nz, c.p, c.q, c.nodes, c.bounds)
    desc = mesh.desc()
    prm = dg.Params.from_array(c.prm)
    Ud = torch.tensor(U, dtype=torch.float64, device="cuda")
    fd = torch.full_like(Ud, float("nan"))
    torch.cuda.synchronize()
    rc = fn(ctypes.byref(desc), ctypes.byref(prm), ctypes.c_void_p(Ud.data_ptr()), ctypes.c_void_p(fd.data_ptr()),
            ctypes.c_void_p(0))
    dg._check(rc)
    torch.cuda.synchronize()
    return fd.cpu().numpy()


def _reference_entry(c, U):
    with dg.Solver(dg.Mesh(c.nx, c.ny, c.nz, c.p, c.q, c.nodes, c.bounds), dg.Params.from_array(c.prm)) as s:
        return s.residual(U)[1]


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def test_noalloc_residual_matches_the_allocating_entry_point_on_two_calls():
    cases = {c.name: c for c in C.residual_cases()}
    first, second = cases["walls_inout_p2"], cases["periodic_p3_q2"]
    f1 = _noalloc(first, first.U)
    f2 = _noalloc(second, second.U)
    assert np.all(np.isfinite(f1)) and np.all(np.isfinite(f2))
    assert rel(f1, _reference_entry(first, first.U)) < 1e-11
    assert rel(f2, _reference_entry(second, second.U)) < 1e-11


def test_noalloc_rejects_meshes_beyond_its_scratch():
    n = 20  # 8000 elements at p = 3 need about 64 MB of scratch, over the 32 MiB array
    c = C.Case("big", n, n, n, 3, 1, C.box_nodes(n, n, n, 1, 1.0, 1.0, 1.0), [C.P_] * 6, C.params(),
               np.zeros(n ** 3 * 5 * 64))
    with pytest.raises(dg.DgbError) as e:
        _noalloc(c, c.U)
    assert e.value.code == dg.ERR_ARG and "32 MiB" in str(e.value)


def test_noalloc_residual_on_curved_meshes():
    """Curved elements: the per-point geometry shares the static array."""
    cases = {c.name: c for c in C.residual_cases()}
    for name in ("bump_p2_q2", "sine_periodic_p2_q2"):
        c = cases[name]
        f = _noalloc(c, c.U)
        assert rel(f, _reference_entry(c, c.U)) < 1e-11, name
