"""dgpr_b200: Python harness over the dgb200 C ABI (include/dgb200.h).

The product is the native library dgpr_b200/_lib/libdgb200.so (C++ host code
plus sm_100a CUDA kernels).  This module only binds it with ctypes so tests,
the benchmark and users in Python can drive it; there is no Python or CPU
compute path.  Importing fails loudly if the library has not been built
(`python -m dgpr_b200.build` or `__graft_entry__.build()`).
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# DGB200_LIB selects another build of the same library (e.g. a tuning variant)
LIB_PATH = os.environ.get("DGB200_LIB") or os.path.join(HERE, "_lib", "libdgb200.so")

OK, ERR_ARG, ERR_UNSUPPORTED, ERR_CUDA, ERR_GEOMETRY, ERR_NONFINITE, ERR_IO, ERR_BOUNDARY = range(8)
INTERIOR, PERIODIC, FREESTREAM, INVISCID_WALL, SUBSONIC_INFLOW, SUBSONIC_OUTFLOW, NO_SLIP_WALL = \
    -1, -2, -3, -4, -5, -6, -7
ISOTHERMAL_WALL = -8  # an extension: no-slip wall at Solver.set_wall_temperature (default: params T)
RK4, TVDRK3 = 0, 1
FP64, MIXED_FP32 = 0, 1
STEP_GAUSS, STEP_NODAL, STEP_GAUSS_TC = 0, 1, 2  # dgb_set_step_form
GEO_ELEMENT, GEO_VOLUME, GEO_FACE = 0, 1, 2  # dgb_get_geometry parts
DPARAM_MU, DPARAM_SOURCE, DPARAM_TWALL, NDPARAMS = 0, 1, 6, 7  # dgb_backward_params: dJ/d[mu, source[0..4], Tw]

BOUNDARY_TYPES = {  # the reference's boundary_types map (boundaries.cpp:37-44)
    "periodic": PERIODIC, "freestream": FREESTREAM, "inviscid_wall": INVISCID_WALL,
    "subsonic_inflow": SUBSONIC_INFLOW, "subsonic_outflow": SUBSONIC_OUTFLOW, "no_slip_wall": NO_SLIP_WALL,
    "isothermal_wall": ISOTHERMAL_WALL,
}
TIME_SCHEMES = {"RK4": RK4, "tvdRK3": TVDRK3}  # multistage_schemes (time.cpp:29-31)


class DgbError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"dgb200 error {code}: {msg}")
        self.code = code


_dp = ctypes.POINTER(ctypes.c_double)


class MeshDesc(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int), ("p", ctypes.c_int),
                ("q", ctypes.c_int), ("nodes", _dp), ("bounds", ctypes.c_longlong * 6)]


class Params(ctypes.Structure):
    """The reference's `parameters` struct (solver_params.cpp:22-36)."""
    _fields_ = [("gamma", ctypes.c_double), ("R", ctypes.c_double), ("mu", ctypes.c_double),
                ("c", ctypes.c_double), ("T", ctypes.c_double), ("P", ctypes.c_double),
                ("Ufr", ctypes.c_double * 5), ("source", ctypes.c_double * 5), ("eta", ctypes.c_double)]

    def as_array(self):
        """17-vector [gamma R mu c T P Ufr(5) source(5) eta]."""
        return np.array([self.gamma, self.R, self.mu, self.c, self.T, self.P, *self.Ufr, *self.source, self.eta])

    @classmethod
    def from_array(cls, a):
        a = [float(v) for v in a]
        p = cls()
        p.gamma, p.R, p.mu, p.c, p.T, p.P = a[:6]
        for i in range(5):
            p.Ufr[i] = a[6 + i]
            p.source[i] = a[11 + i]
        p.eta = a[16]
        return p


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m dgpr_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        vp = ctypes.c_void_p
        sig = {
            "dgb_error_string": (ctypes.c_char_p, [ctypes.c_int]),
            "dgb_last_error_message": (ctypes.c_char_p, []),
            "dgb_create": (ctypes.c_int, [ctypes.POINTER(MeshDesc), ctypes.POINTER(Params), ctypes.c_int,
                                          ctypes.POINTER(vp)]),
            "dgb_destroy": (ctypes.c_int, [vp]),
            "dgb_set_stream": (ctypes.c_int, [vp, vp]),
            "dgb_set_prandtl": (ctypes.c_int, [vp, ctypes.c_double]),
            "dgb_state_size": (ctypes.c_longlong, [vp]),
            "dgb_set_state": (ctypes.c_int, [vp, _dp]),
            "dgb_get_state": (ctypes.c_int, [vp, _dp]),
            "dgb_state_device_ptr": (ctypes.c_int, [vp, ctypes.POINTER(vp)]),
            "dgb_residual": (ctypes.c_int, [vp, _dp, _dp, _dp]),
            "dgb_residual_device": (ctypes.c_int, [vp, vp, vp, vp]),
            "dgb_step": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_double, ctypes.c_ulonglong, _dp]),
            "dgb_step_host": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_double, ctypes.c_ulonglong, _dp, _dp,
                                             _dp]),
            "dgb_step_host_async": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_double, ctypes.c_ulonglong, _dp,
                                                   _dp, _dp]),
            "dgb_last_launch_count": (ctypes.c_longlong, [vp]),
            "dgb_profile_step": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_double, ctypes.c_int, _dp,
                                                ctypes.POINTER(ctypes.c_int)]),
            "dgb_synchronize": (ctypes.c_int, [vp]),
            "dgb_mean_update": (ctypes.c_int, [vp, ctypes.c_ulonglong, ctypes.c_ulonglong]),
            "dgb_set_mean": (ctypes.c_int, [vp, _dp]),
            "dgb_get_mean": (ctypes.c_int, [vp, _dp]),
            "dgb_set_state_device": (ctypes.c_int, [vp, vp]),
            "dgb_get_state_device": (ctypes.c_int, [vp, vp]),
            "dgb_residual_vjp": (ctypes.c_int, [vp, _dp, _dp, _dp]),
            "dgb_residual_vjp_device": (ctypes.c_int, [vp, vp, vp, vp]),
            "dgb_step_vjp_device": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_double, vp, vp]),
            "dgb_forward_record": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_double, ctypes.c_ulonglong,
                                                  ctypes.c_int, _dp]),
            "dgb_forward_record_stages": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_double, ctypes.c_ulonglong,
                                                         _dp]),
            "dgb_backward": (ctypes.c_int, [vp, _dp, _dp]),
            "dgb_backward_device": (ctypes.c_int, [vp, vp, vp]),
            "dgb_backward_params": (ctypes.c_int, [vp, _dp, _dp, _dp]),
            "dgb_backward_params_device": (ctypes.c_int, [vp, vp, vp, vp]),
            "dgb_set_params": (ctypes.c_int, [vp, ctypes.POINTER(Params)]),
            "dgb_set_wall_temperature": (ctypes.c_int, [vp, ctypes.c_double]),
            "dgb_set_step_form": (ctypes.c_int, [vp, ctypes.c_int]),
            "dgb_adjoint_stats": (ctypes.c_int, [vp] + [ctypes.POINTER(ctypes.c_longlong)] * 3),
            "dgb_checkpoint_plan": (ctypes.c_int, [ctypes.c_longlong, ctypes.c_int,
                                                   ctypes.POINTER(ctypes.c_longlong), ctypes.c_longlong,
                                                   ctypes.POINTER(ctypes.c_longlong),
                                                   ctypes.POINTER(ctypes.c_longlong),
                                                   ctypes.POINTER(ctypes.c_int)]),
            "dgb_gauss_legendre": (ctypes.c_int, [ctypes.c_int, ctypes.c_double, ctypes.c_double, _dp, _dp]),
            "dgb_lagrange1d": (ctypes.c_double, [ctypes.c_int, ctypes.c_int, ctypes.c_double]),
            "dgb_lagrange1d_deriv": (ctypes.c_double, [ctypes.c_int, ctypes.c_int, ctypes.c_double]),
            "dgb_bump_nodes": (ctypes.c_int, [ctypes.c_int] * 4 + [ctypes.c_double] * 7 + [_dp]),
            "dgb_get_geometry": (ctypes.c_int, [vp, ctypes.c_int, _dp, ctypes.c_size_t]),
            "dgb_geometry_stats": (ctypes.c_int, [vp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)]),
            "dgb_geometry_host": (ctypes.c_int, [ctypes.POINTER(MeshDesc), ctypes.POINTER(ctypes.c_int),
                                                 _dp, ctypes.c_size_t, _dp, ctypes.c_size_t, _dp,
                                                 ctypes.c_size_t]),
            "dgb_make_reference_state": (ctypes.c_int, [ctypes.c_double] * 9 + [_dp, ctypes.POINTER(Params)]),
            "dgb_write_state": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_ulonglong, ctypes.POINTER(MeshDesc),
                                               ctypes.c_int, ctypes.POINTER(ctypes.c_char_p),
                                               ctypes.POINTER(_dp)]),
            "dgb_read_state": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(ctypes.c_ulonglong)]
                               + [ctypes.POINTER(ctypes.c_int)] * 5
                               + [ctypes.POINTER(ctypes.c_longlong), _dp, ctypes.c_char_p, _dp]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _check(rc):
    if rc != OK:
        msg = lib().dgb_last_error_message().decode(errors="replace")
        raise DgbError(rc, f"{lib().dgb_error_string(rc).decode()}: {msg}")


def _p(a):
    return a.ctypes.data_as(_dp)


# ----------------------------------------------------------------- setup helpers


def checkpoint_plan(nsteps, slots):
    """The binomial checkpoint plan of dgb_forward_record / dgb_backward:
    (ops, forward_steps, peak_slots) with ops a list of (kind, arg), kind
    "forward" (arg steps), "store" / "restore" (arg buffer), "reverse" (arg
    step index).  Host only."""
    n = ctypes.c_longlong()
    fw = ctypes.c_longlong()
    pk = ctypes.c_int()
    _check(lib().dgb_checkpoint_plan(int(nsteps), int(slots), None, 0, ctypes.byref(n), ctypes.byref(fw),
                                     ctypes.byref(pk)))
    buf = (ctypes.c_longlong * (2 * n.value))()
    _check(lib().dgb_checkpoint_plan(int(nsteps), int(slots), buf, 2 * n.value, ctypes.byref(n),
                                     ctypes.byref(fw), ctypes.byref(pk)))
    kinds = ("forward", "store", "restore", "reverse")
    ops = [(kinds[buf[2 * k]], buf[2 * k + 1]) for k in range(n.value)]
    return ops, fw.value, pk.value

def make_reference_state(gamma=1.4, gcnst=287.0, mu=1e-3, c=1.0, rho=1.0, u=0.1, v=0.0, w=0.0, eta=6.0,
                         source=(0.0, 0.0, 0.0, 0.0, 0.0)):
    """make_reference_state (solver_params.cpp:40-70); defaults are the
    reference's solver_inputs defaults (input.cpp:46-65)."""
    out = Params()
    src = np.ascontiguousarray(source, dtype=np.float64)
    _check(lib().dgb_make_reference_state(gamma, gcnst, mu, c, rho, u, v, w, eta, _p(src), ctypes.byref(out)))
    return out


def gauss_legendre(n, a=0.0, b=1.0):
    x = np.zeros(n)
    w = np.zeros(n)
    _check(lib().dgb_gauss_legendre(n, a, b, _p(x), _p(w)))
    return x, w


def lagrange1d(i, p, x):
    return lib().dgb_lagrange1d(i, p, x)


def lagrange1d_deriv(i, p, x):
    return lib().dgb_lagrange1d_deriv(i, p, x)


def bump_nodes(nx, ny, nz, q, lx=2.0, ly=1.0, lz=1.0, a=0.0, bmp_height=0.1, bmp_center=1.0, bmp_variance=0.05):
    """generate_bump_nodes (geometry_common.cpp:494-576); defaults from input.cpp:23-38."""
    nodes = np.zeros(nx * ny * nz * (q + 1) ** 3 * 3)
    _check(lib().dgb_bump_nodes(nx, ny, nz, q, lx, ly, lz, a, bmp_height, bmp_center, bmp_variance, _p(nodes)))
    return nodes


def _geometry_sizes(mesh):
    E = mesh.nx * mesh.ny * mesh.nz
    P = mesh.p + 1
    return {GEO_ELEMENT: E * 36, GEO_VOLUME: E * 10 * P ** 3, GEO_FACE: E * 6 * 14 * P ** 2}


def geometry_host(mesh, curved=None):
    """Element geometry built on the host (dgb_geometry_host): (curved,
    element records, per-point volume part or None, per-point face part or
    None), flat arrays in dgb_get_geometry's layouts.  `curved` True
    allocates the per-point parts up front (one build); None finds out with
    a first build."""
    n = _geometry_sizes(mesh)
    d = mesh.desc()
    cv = ctypes.c_int()
    if curved:
        cv.value = 1
    else:
        _check(lib().dgb_geometry_host(ctypes.byref(d), ctypes.byref(cv), None, 0, None, 0, None, 0))
    geo = np.zeros(n[GEO_ELEMENT])
    gv = np.zeros(n[GEO_VOLUME]) if cv.value else None
    gf = np.zeros(n[GEO_FACE]) if cv.value else None
    _check(lib().dgb_geometry_host(ctypes.byref(d), ctypes.byref(cv), _p(geo), geo.size,
                                   _p(gv) if gv is not None else None, gv.size if gv is not None else 0,
                                   _p(gf) if gf is not None else None, gf.size if gf is not None else 0))
    if not cv.value:
        gv = gf = None
    return bool(cv.value), geo, gv, gf


def box_nodes(nx, ny, nz, q, lx, ly, lz):
    return bump_nodes(nx, ny, nz, q, lx, ly, lz, 0.0, 0.0, 1.0, 1.0)


class Mesh:
    def __init__(self, nx, ny, nz, p, q, nodes, bounds):
        self.nx, self.ny, self.nz, self.p, self.q = int(nx), int(ny), int(nz), int(p), int(q)
        self.nodes = np.ascontiguousarray(nodes, dtype=np.float64).ravel()
        self.bounds = [int(b) for b in bounds]
        if self.nodes.size != self.nelem * (self.q + 1) ** 3 * 3 or len(self.bounds) != 6:
            raise ValueError("mesh nodes / bounds have the wrong size")

    @property
    def nelem(self):
        return self.nx * self.ny * self.nz

    @property
    def nb(self):
        return (self.p + 1) ** 3

    @property
    def state_size(self):
        return self.nelem * 5 * self.nb

    def desc(self):
        d = MeshDesc()
        d.nx, d.ny, d.nz, d.p, d.q = self.nx, self.ny, self.nz, self.p, self.q
        d.nodes = _p(self.nodes)
        for i, b in enumerate(self.bounds):
            d.bounds[i] = b
        return d


def write_state(fname, tstep, mesh, outputs):
    """.dg writer (io.cpp:33-90); outputs: dict key -> state array."""
    keys = list(outputs.keys())
    arrs = [np.ascontiguousarray(outputs[k], dtype=np.float64).ravel() for k in keys]
    karr = (ctypes.c_char_p * len(keys))(*[k.encode() for k in keys])
    darr = (_dp * len(keys))(*[_p(a) for a in arrs])
    d = mesh.desc()
    _check(lib().dgb_write_state(os.fsencode(fname), tstep, ctypes.byref(d), len(keys), karr, darr))


def read_state(fname, key="state"):
    """.dg reader (io.cpp:92-159): returns (tstep, Mesh, state array or None)."""
    t = ctypes.c_ulonglong()
    ints = [ctypes.c_int() for _ in range(5)]
    b = (ctypes.c_longlong * 6)()
    _check(lib().dgb_read_state(os.fsencode(fname), ctypes.byref(t), *[ctypes.byref(i) for i in ints], b,
                                None, None, None))
    nx, ny, nz, p, q = [i.value for i in ints]
    nodes = np.zeros(nx * ny * nz * (q + 1) ** 3 * 3)
    data = np.zeros(nx * ny * nz * 5 * (p + 1) ** 3)
    _check(lib().dgb_read_state(os.fsencode(fname), None, None, None, None, None, None, None, _p(nodes),
                                key.encode() if key else None, _p(data) if key else None))
    return t.value, Mesh(nx, ny, nz, p, q, nodes, list(b)), (data if key else None)


# ----------------------------------------------------------------------- solver

class Solver:
    """One device-resident mesh + state (dgb_create .. dgb_destroy).

    Mirrors the reference's GPU driver objects: the constructor plays
    cuda_device_geometry + cuda_residual_workspace (solve_cuda.cu:171,303),
    `residual` plays cuda_residual (solve_cuda.cu:1235) and `step` plays
    RK4_cuda / tvdRK3_cuda (time_cuda.cu:126-185)."""

    def __init__(self, mesh, params, precision=FP64):
        self.mesh = mesh
        self.params = params if isinstance(params, Params) else Params.from_array(params)
        self._desc = mesh.desc()
        h = ctypes.c_void_p()
        _check(lib().dgb_create(ctypes.byref(self._desc), ctypes.byref(self.params), precision, ctypes.byref(h)))
        self.h = h
        self.n = lib().dgb_state_size(h)
        self._pending = []  # host arrays that queued copies still read or write

    def close(self):
        if self.h:
            lib().dgb_destroy(self.h)  # waits for the queued copies
            self.h = None
            self._pending = []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_state(self, U):
        U = np.ascontiguousarray(U, dtype=np.float64).ravel()
        assert U.size == self.n
        _check(lib().dgb_set_state(self.h, _p(U)))

    def get_state(self):
        U = np.zeros(self.n)
        _check(lib().dgb_get_state(self.h, _p(U)))
        return U

    def geometry_stats(self):
        """(curved, seconds dgb_create spent building the geometry on the device)."""
        cv, t = ctypes.c_int(), ctypes.c_double()
        _check(lib().dgb_geometry_stats(self.h, ctypes.byref(cv), ctypes.byref(t)))
        return bool(cv.value), t.value

    def geometry(self, part=GEO_ELEMENT):
        """The device-built element geometry (dgb_get_geometry), flat."""
        out = np.zeros(_geometry_sizes(self.mesh)[part])
        _check(lib().dgb_get_geometry(self.h, part, _p(out), out.size))
        return out

    def residual(self, U):
        """(R, f) for host state U, f = -Minv R."""
        U = np.ascontiguousarray(U, dtype=np.float64).ravel()
        R = np.zeros(self.n)
        f = np.zeros(self.n)
        _check(lib().dgb_residual(self.h, _p(U), _p(R), _p(f)))
        return R, f

    def residual_device(self, U_ptr, R_ptr, f_ptr):
        """Device pointers (ints, e.g. torch tensor.data_ptr()); asynchronous."""
        _check(lib().dgb_residual_device(self.h, ctypes.c_void_p(U_ptr), ctypes.c_void_p(R_ptr or 0),
                                         ctypes.c_void_p(f_ptr)))

    def set_stream(self, stream_ptr):
        _check(lib().dgb_set_stream(self.h, ctypes.c_void_p(stream_ptr or 0)))

    def state_device_ptr(self):
        p = ctypes.c_void_p()
        _check(lib().dgb_state_device_ptr(self.h, ctypes.byref(p)))
        return p.value

    def step(self, scheme, dt, nsteps, norms=True):
        out = np.zeros(max(int(nsteps), 1))
        _check(lib().dgb_step(self.h, int(scheme), float(dt), int(nsteps), _p(out) if norms else None))
        return out[:nsteps]

    def step_host(self, scheme, dt, nsteps, U_in, U_out, norms=True, wait=True):
        """dgb_step_host: nsteps steps of the host state U_in into U_out
        (float64 numpy arrays, page-locked for the overlap), the copies
        overlapped with the work; returns the per-step norms.  wait=False:
        dgb_step_host_async, the arrays (and the returned norms array) are
        filled by the time synchronize() returns."""
        assert U_in.dtype == np.float64 and U_out.dtype == np.float64 and U_in.size == U_out.size == self.n
        out = np.zeros(max(int(nsteps), 1)) if norms else None
        fn = lib().dgb_step_host if wait else lib().dgb_step_host_async
        if not wait:
            self._pending.append((U_in, U_out, out))
        _check(fn(self.h, int(scheme), float(dt), int(nsteps), _p(U_in), _p(U_out), _p(out) if norms else None))
        return out[:nsteps] if norms else None

    def profile_step(self, scheme, dt, reps):
        """Mean per-launch durations (ms) of one RK step, CUDA events on the
        handle's stream, launch order: per stage trace, stage (+ norm after
        the first stage)."""
        out = np.zeros(64)
        nk = ctypes.c_int(64)
        _check(lib().dgb_profile_step(self.h, int(scheme), float(dt), int(reps), _p(out), ctypes.byref(nk)))
        return out[:nk.value]

    @property
    def last_launch_count(self):
        return lib().dgb_last_launch_count(self.h)

    def mean_update(self, tstep, mean_start):
        """Running mean after step tstep (the reference's update_mean)."""
        _check(lib().dgb_mean_update(self.h, int(tstep), int(mean_start)))

    def get_mean(self):
        M = np.zeros(self.n)
        _check(lib().dgb_get_mean(self.h, _p(M)))
        return M

    def synchronize(self):
        try:
            _check(lib().dgb_synchronize(self.h))
        finally:
            self._pending = []

    def set_prandtl(self, prandtl):
        """Heat conduction with Prandtl number `prandtl` (0 or inf: off, the
        reference's physics); drops captured step graphs and any recorded
        forward run."""
        _check(lib().dgb_set_prandtl(self.h, float(prandtl)))

    def set_state_device(self, U_ptr):
        _check(lib().dgb_set_state_device(self.h, ctypes.c_void_p(U_ptr)))

    def get_state_device(self, U_ptr):
        _check(lib().dgb_get_state_device(self.h, ctypes.c_void_p(U_ptr)))

    # ---- adjoint (no counterpart in the reference)

    def residual_vjp(self, U, lam):
        """(df/dU)^T lam at host state U, f = -Minv R(U)."""
        U = np.ascontiguousarray(U, dtype=np.float64).ravel()
        lam = np.ascontiguousarray(lam, dtype=np.float64).ravel()
        out = np.zeros(self.n)
        _check(lib().dgb_residual_vjp(self.h, _p(U), _p(lam), _p(out)))
        return out

    def residual_vjp_device(self, U_ptr, lam_ptr, out_ptr):
        _check(lib().dgb_residual_vjp_device(self.h, ctypes.c_void_p(U_ptr), ctypes.c_void_p(lam_ptr),
                                             ctypes.c_void_p(out_ptr)))

    def step_vjp_device(self, scheme, dt, U_ptr, lam_ptr):
        """Reverse of one RK step at device state U: lam (device) is the
        adjoint of the stepped state on entry and of U on return."""
        _check(lib().dgb_step_vjp_device(self.h, int(scheme), float(dt), ctypes.c_void_p(U_ptr),
                                         ctypes.c_void_p(lam_ptr)))

    def forward_record(self, scheme, dt, nsteps, slots, norms=True):
        self.record_id = getattr(self, "record_id", 0) + 1
        out = np.zeros(max(int(nsteps), 1))
        _check(lib().dgb_forward_record(self.h, int(scheme), float(dt), int(nsteps), int(slots),
                                        _p(out) if norms else None))
        return out[:nsteps]

    def forward_record_stages(self, scheme, dt, nsteps, norms=True):
        """Recorded run keeping every state and stage state: the backward
        sweep then recomputes nothing."""
        self.record_id = getattr(self, "record_id", 0) + 1
        out = np.zeros(max(int(nsteps), 1))
        _check(lib().dgb_forward_record_stages(self.h, int(scheme), float(dt), int(nsteps),
                                               _p(out) if norms else None))
        return out[:nsteps]

    def backward(self, lamN):
        lamN = np.ascontiguousarray(lamN, dtype=np.float64).ravel()
        out = np.zeros(self.n)
        _check(lib().dgb_backward(self.h, _p(lamN), _p(out)))
        return out

    def backward_device(self, lamN_ptr, out_ptr):
        _check(lib().dgb_backward_device(self.h, ctypes.c_void_p(lamN_ptr), ctypes.c_void_p(out_ptr)))

    def backward_params(self, lamN):
        """(dJ/dU_0, dJ/d[mu, source[0..4], Tw]) for J with dJ/dU_N = lamN."""
        lamN = np.ascontiguousarray(lamN, dtype=np.float64).ravel()
        out = np.zeros(self.n)
        dpar = np.zeros(NDPARAMS)
        _check(lib().dgb_backward_params(self.h, _p(lamN), _p(out), _p(dpar)))
        return out, dpar

    def backward_params_device(self, lamN_ptr, out_ptr, dpar_ptr):
        _check(lib().dgb_backward_params_device(self.h, ctypes.c_void_p(lamN_ptr), ctypes.c_void_p(out_ptr),
                                                ctypes.c_void_p(dpar_ptr)))

    def set_step_form(self, form):
        """STEP_GAUSS (default: dgb_step at the Gauss points) or STEP_NODAL."""
        _check(lib().dgb_set_step_form(self.h, int(form)))

    def set_wall_temperature(self, Tw):
        """Temperature of the isothermal walls (> 0); drops the recorded run."""
        _check(lib().dgb_set_wall_temperature(self.h, float(Tw)))

    def set_params(self, params):
        """New physical parameters (Params or its 17-vector) for this handle;
        mesh, state and Prandtl number stay.  Drops the recorded run."""
        p = params if isinstance(params, Params) else Params.from_array(params)
        _check(lib().dgb_set_params(self.h, ctypes.byref(p)))
        self.params = p

    def adjoint_stats(self):
        """(steps recomputed, steps reversed) by the last backward sweep and
        the forward steps of the whole checkpoint plan."""
        a, b, c = ctypes.c_longlong(), ctypes.c_longlong(), ctypes.c_longlong()
        _check(lib().dgb_adjoint_stats(self.h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)))
        return a.value, b.value, c.value
