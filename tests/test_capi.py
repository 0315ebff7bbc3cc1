"""The C-ABI library on a machine without a GPU: it loads, exports every entry
point include/dgb200.h declares, its host-side helpers agree with the
reference's setup functions and .dg format, and invalid meshes are rejected
with status codes before any device work."""
import ctypes
import os
import re

import numpy as np
import pytest

import dgpr_b200 as dg
import oracle
from tests import cases as C

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "dgb200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(dgb_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_entry_point():
    names = declared_symbols()
    assert len(names) >= 20
    lib = ctypes.CDLL(dg.LIB_PATH)
    for n in names:
        assert hasattr(lib, n), n


def test_library_is_built_for_sm100a():
    out = os.popen(f"cuobjdump --list-elf {dg.LIB_PATH} 2>/dev/null").read()
    if not out:
        pytest.skip("cuobjdump unavailable")
    assert "sm_100a" in out


def test_make_reference_state_matches_reference():
    p = dg.make_reference_state(gamma=1.4, gcnst=287.0, mu=1e-3, c=1.3, rho=1.1, u=0.2, v=-0.1, w=0.05, eta=6.0,
                                source=(0.0, 0.4, 0.0, 0.0, 0.0))
    ref = oracle.reference()
    if ref is not None:
        out = np.zeros(17)
        src = np.array([0.0, 0.4, 0.0, 0.0, 0.0])
        ref.lib.ref_make_reference_state(1.4, 287.0, 1e-3, 1.3, 1.1, 0.2, -0.1, 0.05, 6.0, oracle._p(src),
                                         oracle._p(out))
        assert np.max(np.abs(p.as_array() - out)) == 0.0
    assert np.allclose(p.as_array(), C.params(1.4, 287.0, 1e-3, 1.3, 1.1, 0.2, -0.1, 0.05, 6.0,
                                              (0.0, 0.4, 0.0, 0.0, 0.0)), rtol=1e-15)


@pytest.mark.parametrize("args", [(3, 2, 2, 2, 2.0, 1.0, 1.0, 0.0, 0.1, 1.0, 0.05),
                                  (4, 3, 2, 3, 2.0, 1.0, 0.5, 0.5, 0.2, 0.8, 0.1),
                                  (2, 2, 2, 1, 1.0, 1.0, 1.0, 0.0, 0.0, 1.0, 1.0)])
def test_bump_nodes_match_reference_generator(args):
    nx, ny, nz, q = args[:4]
    mine = dg.bump_nodes(nx, ny, nz, q, *args[4:])
    ref = oracle.reference()
    if ref is None:
        pytest.skip("reference not built here")
    theirs = np.zeros_like(mine)
    ref.lib.ref_bump_nodes(nx, ny, nz, 1, q, *args[4:], oracle._p(theirs))
    assert np.max(np.abs(mine - theirs)) < 1e-15


def test_dg_file_round_trip_and_reference_byte_compatibility(tmp_path):
    nodes = C.box_nodes(2, 3, 1, 2, 1.0, 2.0, 0.5)
    m = dg.Mesh(2, 3, 1, 3, 2, nodes, [dg.SUBSONIC_INFLOW, dg.SUBSONIC_OUTFLOW, dg.INVISCID_WALL,
                                       dg.INVISCID_WALL, dg.PERIODIC, dg.PERIODIC])
    rng = np.random.default_rng(0)
    outs = {"state": rng.standard_normal(m.state_size), "mean": rng.standard_normal(m.state_size)}
    f = str(tmp_path / "a.dg")
    dg.write_state(f, 17, m, outs)
    t, m2, U = dg.read_state(f, "state")
    assert t == 17 and (m2.nx, m2.ny, m2.nz, m2.p, m2.q) == (2, 3, 1, 3, 2) and m2.bounds == m.bounds
    assert np.array_equal(m2.nodes, nodes) and np.array_equal(U, outs["state"])
    _, _, M = dg.read_state(f, "mean")
    assert np.array_equal(M, outs["mean"])
    ref = oracle.reference()
    if ref is not None:
        g = str(tmp_path / "b.dg")
        keys = (ctypes.c_char_p * 2)(b"state", b"mean")
        data = (ctypes.POINTER(ctypes.c_double) * 2)(oracle._p(outs["state"]), oracle._p(outs["mean"]))
        b = np.array(m.bounds, dtype=np.int64)
        ref.lib.ref_write_state.argtypes = None
        ref.lib.ref_write_state(g.encode(), ctypes.c_ulonglong(17), 2, 3, 1, 3, 2, oracle._lpp(b),
                                oracle._p(nodes), 2, keys, data)
        assert open(f, "rb").read() == open(g, "rb").read()


def test_truncated_dg_file_is_an_io_error(tmp_path):
    nodes = C.box_nodes(1, 1, 1, 1, 1.0, 1.0, 1.0)
    m = dg.Mesh(1, 1, 1, 1, 1, nodes, [dg.PERIODIC] * 6)
    f = str(tmp_path / "t.dg")
    dg.write_state(f, 0, m, {"state": np.ones(m.state_size)})
    raw = open(f, "rb").read()
    open(f, "wb").write(raw[:-8])
    with pytest.raises(dg.DgbError) as e:
        dg.read_state(f)
    assert e.value.code == dg.ERR_IO


def _try_create(nx, ny, nz, p, q, nodes, bounds):
    with pytest.raises(dg.DgbError) as e:
        dg.Solver(dg.Mesh(nx, ny, nz, p, q, nodes, bounds), dg.make_reference_state())
    return e.value.code


def test_invalid_meshes_are_rejected_before_device_work():
    box = C.box_nodes(2, 2, 2, 1, 1.0, 1.0, 1.0)
    assert _try_create(2, 2, 2, 2, 1, box, [dg.PERIODIC, dg.FREESTREAM] + [dg.PERIODIC] * 4) == dg.ERR_GEOMETRY
    assert _try_create(2, 2, 2, 7, 1, box, [dg.PERIODIC] * 6) == dg.ERR_UNSUPPORTED
    assert _try_create(2, 2, 2, 2, 1, box, [dg.INTERIOR] + [dg.PERIODIC] * 5) == dg.ERR_ARG
    # singular and mismatched element geometry is found by the device builder
    # (tests/test_geometry.py checks it against the host builder's messages)


def test_noalloc_residual_rejects_oversized_meshes_before_device_work():
    """The 32 MiB static scratch bounds the mesh; the size check comes before
    any CUDA call (curved meshes need more per element than affine ones)."""
    import ctypes
    prm = dg.make_reference_state()
    fn = dg.lib().dgb_residual_noalloc
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.POINTER(dg.MeshDesc), ctypes.POINTER(dg.Params), ctypes.c_void_p, ctypes.c_void_p,
                   ctypes.c_void_p]
    for n, q, nodes in [(20, 1, C.box_nodes(20, 20, 20, 1, 1.0, 1.0, 1.0)),
                        (12, 2, C.sine_nodes(12, 12, 12, 2, 1.0, 1.0, 1.0, 0.02))]:
        desc = dg.Mesh(n, n, n, 3, q, nodes, [dg.PERIODIC] * 6).desc()
        # device pointers are never touched: the mesh is refused first
        assert fn(ctypes.byref(desc), ctypes.byref(prm), ctypes.c_void_p(16), ctypes.c_void_p(16), None) == \
            dg.ERR_ARG
        assert "32 MiB" in dg.lib().dgb_last_error_message().decode()

def test_read_state_finds_a_key_without_copying(tmp_path):
    import ctypes
    mesh = dg.Mesh(1, 1, 1, 1, 1, C.box_nodes(1, 1, 1, 1, 1.0, 1.0, 1.0), [dg.PERIODIC] * 6)
    f = str(tmp_path / "k.dg")
    dg.write_state(f, 3, mesh, {"state": np.ones(40)})
    t = ctypes.c_ulonglong()
    rc = dg.lib().dgb_read_state(f.encode(), ctypes.byref(t), None, None, None, None, None, None, None, b"state", None)
    assert rc == dg.OK and t.value == 3
    rc = dg.lib().dgb_read_state(f.encode(), None, None, None, None, None, None, None, None, b"other", None)
    assert rc == dg.ERR_IO
