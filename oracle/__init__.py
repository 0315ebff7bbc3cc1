"""ctypes bindings for the parity checkers (test infrastructure only).

`restatement()` loads liboracle.so, the C restatement of the reference's FP64
residual / RK path (dg_oracle.c).  `reference()` loads _ref/libdgref.so, the
unmodified reference solver compiled in place, when it has been built here.
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
module; the product never imports it.

Parameter vectors use one layout everywhere (17 doubles):
    [0] gamma [1] R [2] mu [3] c [4] T [5] P [6:11] Ufr [11:16] source [16] eta
Boundary codes follow the reference's btype enum (boundaries.cpp:26-35).
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_dp = ctypes.POINTER(ctypes.c_double)
_lp = ctypes.POINTER(ctypes.c_longlong)

PERIODIC, FREESTREAM, INVISCID_WALL, SUBSONIC_INFLOW, SUBSONIC_OUTFLOW, NO_SLIP_WALL = -2, -3, -4, -5, -6, -7


def _p(a):
    return a.ctypes.data_as(_dp)


def _lpp(a):
    return a.ctypes.data_as(_lp)


def build_restatement():
    """Compile liboracle.so from dg_oracle.c (gcc only; works on any box)."""
    subprocess.check_call(["make", "-s", "-C", HERE, os.path.join(HERE, "liboracle.so")])


_cache = {}


def _load(path, sigs):
    lib = ctypes.CDLL(path)
    for name, (res, args) in sigs.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


_mesh_args = [ctypes.c_int] * 5 + [_dp, _lp]
_SIGS_COMMON = {
    "residual": (ctypes.c_int, _mesh_args + [_dp, _dp, _dp, _dp]),
    "run": (ctypes.c_int, _mesh_args + [_dp, ctypes.c_int, ctypes.c_double, ctypes.c_int, _dp, _dp]),
    "roe": (None, [_dp, _dp, _dp, ctypes.c_double, _dp, _dp]),
    "A": (None, [_dp, _dp, _dp, _dp, ctypes.c_double, _dp]),
    "analytical_flux": (None, [_dp, ctypes.c_double, _dp]),
    "lagrange1d": (ctypes.c_double, [ctypes.c_int, ctypes.c_int, ctypes.c_double]),
    "lagrange1d_deriv": (ctypes.c_double, [ctypes.c_int, ctypes.c_int, ctypes.c_double]),
}


class _Solver:
    """Uniform Python face over either library (prefix 'oracle_' or 'ref_')."""

    def __init__(self, lib, prefix):
        self.lib = lib
        self.prefix = prefix

    def _f(self, name):
        return getattr(self.lib, self.prefix + name)

    def residual(self, mesh, params, U):
        U = np.ascontiguousarray(U, dtype=np.float64).ravel()
        R = np.zeros_like(U)
        f = np.zeros_like(U)
        rc = self._f("residual")(*mesh.args(), _p(np.ascontiguousarray(params, np.float64)), _p(U), _p(R), _p(f))
        if rc != 0:
            raise RuntimeError(f"{self.prefix}residual failed ({rc})")
        return R, f

    def run(self, mesh, params, U, scheme, dt, nsteps):
        U = np.ascontiguousarray(U, dtype=np.float64).ravel().copy()
        norms = np.zeros(max(nsteps, 1))
        rc = self._f("run")(*mesh.args(), _p(np.ascontiguousarray(params, np.float64)), int(scheme),
                            float(dt), int(nsteps), _p(U), _p(norms))
        if rc != 0:
            raise RuntimeError(f"{self.prefix}run failed ({rc})")
        return U, norms[:nsteps]

    def roe(self, UL, UR, n, gamma):
        f = np.zeros(5)
        smax = np.zeros(1)
        self._f("roe")(_p(np.asarray(UL, np.float64)), _p(np.asarray(UR, np.float64)),
                       _p(np.asarray(n, np.float64)), float(gamma), _p(f), _p(smax))
        return f, smax[0]

    def A(self, s, sx, sy, sz, mu):
        Q = np.zeros(15)
        self._f("A")(*(_p(np.asarray(a, np.float64)) for a in (s, sx, sy, sz)), float(mu), _p(Q))
        return Q.reshape(3, 5)

    def analytical_flux(self, U, gamma):
        F = np.zeros(15)
        self._f("analytical_flux")(_p(np.asarray(U, np.float64)), float(gamma), _p(F))
        return F.reshape(3, 5)

    def lagrange1d(self, i, p, x):
        return self._f("lagrange1d")(i, p, x)

    def lagrange1d_deriv(self, i, p, x):
        return self._f("lagrange1d_deriv")(i, p, x)


def restatement():
    if "o" not in _cache:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build_restatement()
        sigs = {"oracle_" + k: v for k, v in _SIGS_COMMON.items()}
        sigs.update({
            "oracle_gauss_legendre": (None, [ctypes.c_int, ctypes.c_double, ctypes.c_double, _dp, _dp]),
            "oracle_det3": (ctypes.c_double, [_dp]),
            "oracle_inv3": (None, [_dp, _dp]),
            "oracle_invert": (ctypes.c_int, [ctypes.c_int, _dp]),
            "oracle_symm_packed_mv": (None, [ctypes.c_int, _dp, _dp, ctypes.c_double, _dp]),
            "oracle_bc_state": (ctypes.c_int, [ctypes.c_int, _dp, _dp] + [ctypes.c_double] * 5 + [_dp, _dp]),
            "oracle_geometry": (ctypes.c_int, _mesh_args + [_dp, _dp, _dp, _dp, _lp]),
            "oracle_box_nodes": (None, [ctypes.c_int] * 4 + [ctypes.c_double] * 3 + [_dp]),
        })
        _cache["o"] = _Solver(_load(path, sigs), "oracle_")
    return _cache["o"]


def reference_path():
    return os.path.join(HERE, "_ref", "libdgref.so")


def reference():
    """The unmodified reference solver, or None when it was not built here."""
    if "r" not in _cache:
        path = reference_path()
        if not os.path.exists(path):
            return None
        sigs = {"ref_" + k: v for k, v in _SIGS_COMMON.items()}
        sigs.update({
            "ref_make_reference_state": (None, [ctypes.c_double] * 9 + [_dp, _dp]),
            "ref_bump_nodes": (None, [ctypes.c_int] * 5 + [ctypes.c_double] * 7 + [_dp]),
            "ref_gauss_legendre_1d": (None, [ctypes.c_int, ctypes.c_double, ctypes.c_double, _dp, _dp]),
            "ref_bc_state": (None, [ctypes.c_longlong, _dp, _dp] + [ctypes.c_double] * 5 + [_dp]),
            "ref_basis_tables": (None, [ctypes.c_int, _dp, _dp, _dp, _dp]),
            "ref_geometry": (ctypes.c_int, _mesh_args + [_dp] * 5 + [_lp, _lp]),
            "ref_num_faces": (ctypes.c_longlong, [ctypes.c_int] * 4 + [_lp]),
        })
        _cache["r"] = _Solver(_load(path, sigs), "ref_")
    return _cache["r"]


class Mesh:
    """nx*ny*nz hexes of order p (solution) and q (geometry) with explicit
    geometry nodes [E][(q+1)^3][3] and six boundary codes."""

    def __init__(self, nx, ny, nz, p, q, nodes, bounds):
        self.nx, self.ny, self.nz, self.p, self.q = int(nx), int(ny), int(nz), int(p), int(q)
        self.nodes = np.ascontiguousarray(nodes, dtype=np.float64).ravel()
        self.bounds = np.ascontiguousarray(bounds, dtype=np.int64)
        assert self.nodes.size == self.nelem * (q + 1) ** 3 * 3
        assert self.bounds.size == 6

    @property
    def nelem(self):
        return self.nx * self.ny * self.nz

    @property
    def nb(self):
        return (self.p + 1) ** 3

    def args(self):
        return (self.nx, self.ny, self.nz, self.p, self.q, _p(self.nodes), _lpp(self.bounds))


def box_mesh(nx, ny, nz, p, q, lx, ly, lz, bounds):
    nodes = np.zeros(nx * ny * nz * (q + 1) ** 3 * 3)
    restatement().lib.oracle_box_nodes(nx, ny, nz, q, lx, ly, lz, _p(nodes))
    return Mesh(nx, ny, nz, p, q, nodes, bounds)


def make_reference_state(gamma=1.4, gcnst=287.0, mu=1e-3, c=1.0, rho=1.0, u=0.1, v=0.0, w=0.0,
                         eta=6.0, source=(0, 0, 0, 0, 0)):
    """solver_params.cpp:40-70 restated: P = c^2 rho / gamma, T = P / (rho R)."""
    P = c * c * (rho / gamma)
    out = np.zeros(17)
    out[0], out[1], out[2], out[3] = gamma, gcnst, mu, c
    out[4] = P / (rho * gcnst)
    out[5] = P
    out[6:11] = [rho, rho * u, rho * v, rho * w, P / (gamma - 1.0) + 0.5 * rho * (u * u + v * v + w * w)]
    out[11:16] = source
    out[16] = eta
    return out
