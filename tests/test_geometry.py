"""Element geometry: the host builder (dgb_geometry_host) against the oracle's
restatement of the reference's precompute (core_geometry::precompute,
geometry_common.cpp:292-395, and the face geometry of
geometry_common.cpp:416-454), and the device builder dgb_create uses
(geometry.cu, read back by dgb_get_geometry) bit for bit against the host
builder, including its error checks and messages.

Tolerance against the oracle: 1e-13 relative for determinants and surface
Jacobians, 1e-13 absolute for unit normals (the oracle takes the Jacobian
through the 3D basis and the face tangents through the 2D face interpolant;
mathematically the same numbers, summed in another order)."""
import numpy as np
import pytest

import dgpr_b200 as dg
import oracle
from tests import cases as C

KGEO, KVOL, KFACE = 36, 10, 14
GEO_DETJ, GEO_N, GEO_FJ = 9, 10, 28
FACE_N, FACE_FJ, FACE_LIFT = 9, 12, 13


def _mesh(c):
    return dg.Mesh(c.nx, c.ny, c.nz, c.p, c.q, c.nodes, c.bounds)


def _oracle_geometry(c):
    m = oracle.Mesh(c.nx, c.ny, c.nz, c.p, c.q, c.nodes, c.bounds)
    P = c.p + 1
    E = m.nelem
    nfmax = 3 * E + c.nx * c.ny + c.ny * c.nz + c.nz * c.nx
    vJ = np.zeros(E * P ** 3)
    fJ = np.zeros(nfmax * P * P)
    fn = np.zeros(nfmax * P * P * 3)
    faces = np.zeros(nfmax * 4, dtype=np.int64)
    nf = oracle.restatement().lib.oracle_geometry(*m.args(), oracle._p(vJ), None, oracle._p(fJ), oracle._p(fn),
                                                  oracle._lpp(faces))
    return vJ.reshape(E, P ** 3), fJ[:nf * P * P].reshape(nf, P * P), fn[:nf * P * P * 3].reshape(nf, P * P, 3), \
        faces[:4 * nf].reshape(nf, 4)


def _oracle_point_order(lf, P):
    """Index into the oracle's face points (surf2vol's (s, t), s fastest) of
    each of this library's face points (tangential axes in axis order)."""
    idx = np.arange(P * P)
    if lf in (2, 3):  # y faces: the oracle's s runs along z, t along x
        t1, t2 = idx % P, idx // P
        return t2 + P * t1
    return idx


def _face_geometry(c, geo, gf):
    """(normals [E][6][P^2][3], surface Jacobians [E][6][P^2]) from either part."""
    E, P = c.nx * c.ny * c.nz, c.p + 1
    if gf is not None:
        g = gf.reshape(E, 6, KFACE, P * P)
        return np.moveaxis(g[:, :, FACE_N:FACE_N + 3, :], 2, 3), g[:, :, FACE_FJ, :]
    g = geo.reshape(E, KGEO)
    n = g[:, GEO_N:GEO_N + 18].reshape(E, 6, 1, 3).repeat(P * P, axis=2)
    return n, g[:, GEO_FJ:GEO_FJ + 6, None].repeat(P * P, axis=2)


def _check_against_oracle(c):
    curved, geo, gv, gf = dg.geometry_host(_mesh(c))
    E, P = c.nx * c.ny * c.nz, c.p + 1
    vJ, fJ, fn, faces = _oracle_geometry(c)
    if curved:
        dJ = gv.reshape(E, KVOL, P ** 3)[:, 9, :]
    else:
        dJ = np.repeat(geo.reshape(E, KGEO)[:, GEO_DETJ, None], P ** 3, axis=1)
    assert np.max(np.abs(dJ - vJ) / np.abs(vJ)) < 1e-13
    n, fj = _face_geometry(c, geo, gf)
    for f in range(faces.shape[0]):
        e, lf = int(faces[f, 0]), int(faces[f, 2])
        o = _oracle_point_order(lf, P)
        assert np.max(np.abs(n[e, lf] - fn[f, o])) < 1e-13, (c.name, f)
        assert np.max(np.abs(fj[e, lf] - fJ[f, o]) / fJ[f, o]) < 1e-13, (c.name, f)
    return curved


def test_host_geometry_matches_the_oracle():
    kinds = {}
    for c in C.residual_cases():
        kinds[c.name] = _check_against_oracle(c)
    assert kinds["bump_p2_q2"] and kinds["sine_periodic_p2_q2"] and not kinds["sheared_p2"]


def test_host_geometry_lifting_scale_of_affine_elements():
    """The face lifting scale of a curved element with straight sides is
    cend / detJ, the affine value (E_f Minv E_f^T with a constant Jacobian)."""
    c = C.Case("q2box", 2, 2, 2, 3, 2, C.box_nodes(2, 2, 2, 2, 1.0, 1.0, 1.0), [C.P_] * 6, C.params(), None)
    nodes = c.nodes.reshape(-1, 3).copy()
    nodes[:, 1] += 0.03 * np.sin(2 * np.pi * nodes[:, 0]) * np.sin(2 * np.pi * nodes[:, 2])
    curved, geo, gv, gf = dg.geometry_host(dg.Mesh(2, 2, 2, 3, 2, nodes.ravel(), [C.P_] * 6))
    assert curved
    P = 4
    x, w = dg.gauss_legendre(P)
    el1 = np.array([np.prod([(1.0 - x[m]) / (x[q] - x[m]) for m in range(P) if m != q]) for q in range(P)])
    g = gf.reshape(8, 6, KFACE, P * P)
    dJ = gv.reshape(8, KVOL, P, P, P)[:, 9]  # [e][k][j][i]
    # +x face (lf 1), point (t1 = j, t2 = k): sum over i of EL1[i]^2 / (w_i detJ(i, j, k))
    lift = np.einsum("i,ekji->ejk", el1 ** 2 / w, 1.0 / dJ)
    assert np.allclose(g[:, 1, FACE_LIFT, :].reshape(8, P, P), lift.transpose(0, 2, 1), rtol=1e-13, atol=0)


def test_host_geometry_errors():
    box = C.box_nodes(2, 2, 2, 1, 1.0, 1.0, 1.0)
    flat = box.copy().reshape(-1, 3)
    flat[:, 0] = 0.0
    with pytest.raises(dg.DgbError) as e:
        dg.geometry_host(dg.Mesh(2, 2, 2, 2, 1, flat.ravel(), [C.P_] * 6))
    assert e.value.code == dg.ERR_GEOMETRY and "element 0 has a singular Jacobian" in str(e.value)
    bump = dg.bump_nodes(2, 2, 2, 2, 2.0, 1.0, 1.0, 0.0, 0.2, 0.7, 0.05)
    with pytest.raises(dg.DgbError) as e:
        dg.geometry_host(dg.Mesh(2, 2, 2, 2, 2, bump, [C.P_, C.P_] + [C.F_] * 4))
    assert e.value.code == dg.ERR_GEOMETRY and "does not match its neighbour" in str(e.value)
    folded = _folded_nodes()
    with pytest.raises(dg.DgbError) as e:
        dg.geometry_host(dg.Mesh(3, 1, 1, 2, 2, folded, [C.F_] * 6))
    assert e.value.code == dg.ERR_GEOMETRY and "element 1 has a non-positive Jacobian determinant" in str(e.value)


def _folded_nodes():
    """Three q = 2 elements in x; the middle one's mid-edge nodes pushed past
    its far side, so its Jacobian changes sign inside it."""
    nodes = C.box_nodes(3, 1, 1, 2, 3.0, 1.0, 1.0).reshape(3, 3, 3, 3, 3)  # [e][k][j][i][xyz]
    nodes[1, :, :, 1, 0] += 0.9
    return nodes.ravel()


# ----------------------------------------------------------- device builder


def _device_cases():
    out = list(C.residual_cases())
    out.append(C.Case("sine_walls_p3_q2", 6, 4, 5, 3, 2, C.sine_nodes(6, 4, 5, 2, 2.0, 2.0, 1.0, 0.05, walls=True),
                      [C.P_, C.P_, C.NS_, C.NS_, C.P_, C.P_], C.params(), None))
    out.append(C.Case("bump_p4_q3", 4, 3, 2, 4, 3, dg.bump_nodes(4, 3, 2, 3, 2.0, 1.0, 0.5, 0.6),
                      [C.F_, C.F_, C.NS_, C.W_, C.P_, C.P_], C.params(), None))
    out.append(C.Case("stretched_p3", 5, 4, 3, 3, 1, dg.bump_nodes(5, 4, 3, 1, 2.0, 1.0, 0.5, 0.7, 0.0),
                      [C.P_] * 6, C.params(), None))
    return out


@pytest.mark.gpu
def test_device_geometry_is_bit_identical_to_the_host_builder():
    for c in _device_cases():
        curved, geo, gv, gf = dg.geometry_host(_mesh(c))
        with dg.Solver(_mesh(c), C.params()) as s:
            cv, build_s = s.geometry_stats()
            assert cv == curved and build_s > 0.0, c.name
            assert np.array_equal(s.geometry(dg.GEO_ELEMENT), geo), c.name
            if curved:
                assert np.array_equal(s.geometry(dg.GEO_VOLUME), gv), c.name
                assert np.array_equal(s.geometry(dg.GEO_FACE), gf), c.name
            else:
                with pytest.raises(dg.DgbError):
                    s.geometry(dg.GEO_VOLUME)


@pytest.mark.gpu
def test_device_geometry_errors_match_the_host_builder():
    box = C.box_nodes(2, 2, 2, 1, 1.0, 1.0, 1.0)
    flat = box.copy().reshape(-1, 3)
    flat[:, 0] = 0.0
    bad = [dg.Mesh(2, 2, 2, 2, 1, flat.ravel(), [C.P_] * 6),
           dg.Mesh(2, 2, 2, 2, 2, dg.bump_nodes(2, 2, 2, 2, 2.0, 1.0, 1.0, 0.0, 0.2, 0.7, 0.05),
                   [C.P_, C.P_] + [C.F_] * 4),
           dg.Mesh(3, 1, 1, 2, 2, _folded_nodes(), [C.F_] * 6)]
    for m in bad:
        with pytest.raises(dg.DgbError) as host:
            dg.geometry_host(m)
        with pytest.raises(dg.DgbError) as dev:
            dg.Solver(m, C.params())
        assert dev.value.code == host.value.code == dg.ERR_GEOMETRY
        assert str(dev.value) == str(host.value)


def test_face_match_predicate_flags_degenerate_faces():
    """The face-match test both builders run (host.cpp, geometry.cu) through
    the check hook: matching sides pass; a normal or surface Jacobian that is
    off by more than 1e-10, a NaN normal, and a zero or NaN surface
    Jacobian (a collapsed face, 0/0) are mismatches."""
    import ctypes
    dp = ctypes.POINTER(ctypes.c_double)
    f = dg.lib().dgb_check_pointwise
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_int, dp, dp, dp, dp, dp]

    def mismatch(ng, nh, fg, fh):
        x = np.array([*ng, *nh, fg, fh], dtype=np.float64)
        aux, y = np.zeros(1), np.zeros(1)
        assert f(10, x.ctypes.data_as(dp), None, aux.ctypes.data_as(dp), y.ctypes.data_as(dp), None) == 0
        return bool(y[0])

    n = np.array([0.6, 0.8, 0.0])
    assert not mismatch(n, -n, 2.0, 2.0)
    assert not mismatch(n, -n + 1e-12, 2.0, 2.0 * (1 + 1e-12))
    assert mismatch(n, -n + 1e-8, 2.0, 2.0)
    assert mismatch(n, -n, 2.0, 2.0 * (1 + 1e-8))
    assert mismatch(np.array([np.nan, 0.8, 0.0]), -n, 2.0, 2.0)
    assert mismatch(n, np.array([-0.6, np.nan, 0.0]), 2.0, 2.0)
    assert mismatch(n, -n, 0.0, 0.0)
    assert mismatch(n, -n, np.nan, 2.0)
