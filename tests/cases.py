"""Seeded parity cases shared by the fixture generator and the tests.

Each case is a small mesh + reference parameters + initial state, sized so the
CPU checkers finish in well under a second.  Flow fields are synthetic
stand-ins with the shapes of the benchmark configurations: an isentropic
vortex (Euler), the Taylor-Green vortex (Navier-Stokes) and seeded random
perturbations of a freestream.
"""
import math

import numpy as np

P_, F_, W_, IN_, OUT_, NS_ = -2, -3, -4, -5, -6, -7


def params(gamma=1.4, gcnst=287.0, mu=1e-3, c=1.0, rho=1.0, u=0.1, v=0.0, w=0.0, eta=6.0, source=(0, 0, 0, 0, 0)):
    """make_reference_state (solver_params.cpp:40-70) as a 17-vector
    [gamma R mu c T P Ufr(5) source(5) eta]."""
    P = c * c * (rho / gamma)
    out = np.zeros(17)
    out[:6] = [gamma, gcnst, mu, c, P / (rho * gcnst), P]
    out[6:11] = [rho, rho * u, rho * v, rho * w, P / (gamma - 1.0) + 0.5 * rho * (u * u + v * v + w * w)]
    out[11:16] = source
    out[16] = eta
    return out


def box_nodes(nx, ny, nz, q, lx, ly, lz, shear=0.0):
    """Equispaced box elements, [z[y[x]]] node order; `shear` adds shear*y to x
    (an affine parallelepiped mesh)."""
    Q = q + 1
    X = np.zeros((nz, ny, nx, Q, Q, Q, 3))
    ex, ey, ez = lx / nx, ly / ny, lz / nz
    a = np.arange(Q) / q
    for k in range(nz):
        for j in range(ny):
            for i in range(nx):
                zz, yy, xx = np.meshgrid(k * ez + ez * a, j * ey + ey * a, i * ex + ex * a, indexing="ij")
                X[k, j, i, ..., 0] = xx + shear * yy
                X[k, j, i, ..., 1] = yy
                X[k, j, i, ..., 2] = zz
    return X.ravel()


def sine_nodes(nx, ny, nz, q, lx, ly, lz, amp, walls=False):
    """Curved order-q elements: equispaced box nodes with y displaced by
    amp sin(2 pi x / lx) sin(2 pi z / lz), times (1 - (2y/ly - 1)^2) when the
    y sides are walls (they stay flat).  Periodic in x and z, and in y too
    without the wall factor.  The reference has no generator for this mesh;
    its nodes reach it as a .dg node array (io.cpp:131-136)."""
    X = box_nodes(nx, ny, nz, q, lx, ly, lz).reshape(-1, 3)
    d = amp * np.sin(2 * math.pi * X[:, 0] / lx) * np.sin(2 * math.pi * X[:, 2] / lz)
    if walls:
        d *= 1.0 - (2.0 * X[:, 1] / ly - 1.0) ** 2
    X[:, 1] += d
    return X.ravel()


def bump_nodes(nx, ny, nz, q, lx, ly, lz, height=0.1, center=1.0, variance=0.05):
    """The reference's bump channel (generate_bump_nodes,
    geometry_common.cpp:494-576, no stretching), restated here so the cases
    need no library."""
    Q = q + 1
    X = np.zeros((nz, ny, nx, Q, Q, Q, 3))
    elx, ely, elz = lx / nx, ly / ny, lz / nz
    nsx, nsy, nsz = elx / q, ely / q, elz / q
    for ez in range(nz):
        for ey in range(ny):
            for ex in range(nx):
                for k in range(Q):
                    for j in range(Q):
                        for i in range(Q):
                            x = ex * elx + nsx * i
                            y = ey * ely + nsy * j
                            z = ez * elz + nsz * k
                            f = height * math.exp(-((x - center) * (x - center)) / (2.0 * variance))
                            X[ez, ey, ex, k, j, i] = (x, (y / ly) * (ly - f) + f, z)
    return X.ravel()


def node_coords(nx, ny, nz, p, q, nodes):
    """Physical coordinates of the solution nodes (equispaced reference nodes
    i/p mapped through the order-q geometry), shape [E][nb][3]."""
    Q, Pn = q + 1, p + 1
    E = nx * ny * nz
    X = nodes.reshape(E, Q, Q, Q, 3)  # [e][k][j][i]
    r = np.arange(Pn) / p if p > 0 else np.zeros(1)

    def lag(i, x):
        v = 1.0
        for j in range(Q):
            if j != i:
                v *= (x - j / q) / (i / q - j / q)
        return v

    L = np.array([[lag(i, x) for i in range(Q)] for x in r])  # [node][geo]
    out = np.einsum("ai,bj,ck,ekjid->ecbad", L, L, L, X)  # [e][z][y][x][3]
    return out.reshape(E, Pn ** 3, 3)


def state_from_primitives(rho, u, v, w, p, gamma):
    E = p / (gamma - 1.0) + 0.5 * rho * (u * u + v * v + w * w)
    return np.stack([rho, rho * u, rho * v, rho * w, E], axis=-2)  # [..., 5, nb]


def random_state(prm, E, nb, rng, amp=0.05):
    U = np.tile(prm[6:11][None, :, None], (E, 1, nb)).astype(np.float64)
    U *= 1.0 + amp * rng.standard_normal(U.shape)
    U[:, 1:4, :] += amp * rng.standard_normal(U[:, 1:4, :].shape)
    return U.ravel()


def isentropic_vortex(xyz, gamma=1.4, eps=5.0, xc=5.0, yc=5.0, u0=1.0, v0=1.0):
    """Shu's isentropic vortex on rho=1, p=1 freestream (z aligned)."""
    x, y = xyz[..., 0] - xc, xyz[..., 1] - yc
    r2 = x * x + y * y
    du = eps / (2 * math.pi) * np.exp(0.5 * (1 - r2))
    T = 1.0 - (gamma - 1.0) * eps * eps / (8 * gamma * math.pi ** 2) * np.exp(1 - r2)
    rho = T ** (1.0 / (gamma - 1.0))
    return state_from_primitives(rho, u0 - du * y, v0 + du * x, 0 * x, rho ** gamma, gamma)


def taylor_green(xyz, gamma=1.4, V0=1.0, rho0=1.0, Ma=0.1):
    """TGV: u = sin x cos y cos z, v = -cos x sin y cos z, w = 0,
    p = p0 + (cos 2x + cos 2y)(cos 2z + 2)/16, isothermal rho = p/p0 * rho0."""
    x, y, z = xyz[..., 0], xyz[..., 1], xyz[..., 2]
    p0 = rho0 * V0 * V0 / (gamma * Ma * Ma)
    u = V0 * np.sin(x) * np.cos(y) * np.cos(z)
    v = -V0 * np.cos(x) * np.sin(y) * np.cos(z)
    w = 0 * x
    p = p0 + rho0 * V0 * V0 / 16.0 * (np.cos(2 * x) + np.cos(2 * y)) * (np.cos(2 * z) + 2.0)
    rho = rho0 * p / p0
    return state_from_primitives(rho, u, v, w, p, gamma)


class Case:
    def __init__(self, name, nx, ny, nz, p, q, nodes, bounds, prm, U, scheme=None, dt=None, nsteps=0):
        self.name, self.nx, self.ny, self.nz, self.p, self.q = name, nx, ny, nz, p, q
        self.nodes, self.bounds, self.prm, self.U = nodes, list(bounds), prm, U
        self.scheme, self.dt, self.nsteps = scheme, dt, nsteps

    @property
    def nelem(self):
        return self.nx * self.ny * self.nz

    @property
    def nb(self):
        return (self.p + 1) ** 3


def residual_cases():
    rng = np.random.default_rng(20241203)
    out = []
    visc = params(mu=1e-2, c=1.0, u=0.3, v=0.1, w=-0.2)

    def add(name, nx, ny, nz, p, q, L, bounds, prm, shear=0.0, amp=0.05):
        nodes = box_nodes(nx, ny, nz, q, *L, shear=shear)
        U = random_state(prm, nx * ny * nz, (p + 1) ** 3, rng, amp)
        out.append(Case(name, nx, ny, nz, p, q, nodes, bounds, prm, U))

    add("periodic_p2", 2, 2, 2, 2, 1, (1.0, 1.0, 1.0), [P_] * 6, visc)
    add("periodic_p1_aniso", 3, 2, 1, 1, 1, (1.0, 2.0, 1.5), [P_] * 6, visc)
    add("periodic_p3_q2", 2, 2, 2, 3, 2, (1.0, 1.0, 1.0), [P_] * 6, params(mu=5e-3, u=0.2))
    add("sheared_p2", 2, 3, 2, 2, 1, (1.0, 1.0, 1.0), [P_] * 6, visc, shear=0.3)
    add("walls_inout_p2", 2, 3, 2, 2, 1, (2.0, 1.0, 1.0), [IN_, OUT_, W_, NS_, P_, P_], params(mu=1e-2, u=0.3))
    add("freestream_p2", 2, 2, 2, 2, 1, (1.0, 1.0, 1.0), [F_, F_, W_, W_, F_, F_], visc)
    add("noslip_p3", 2, 2, 2, 3, 1, (1.0, 1.0, 1.0), [P_, P_, NS_, NS_, P_, P_], params(mu=2e-2, u=0.3))
    add("p0", 3, 3, 3, 0, 1, (1.0, 1.0, 1.0), [P_] * 6, visc)
    add("p4", 2, 2, 1, 4, 1, (1.0, 1.0, 0.5), [P_] * 6, visc)
    add("p5", 1, 2, 1, 5, 1, (0.5, 1.0, 0.5), [P_] * 6, visc)
    add("p6", 1, 1, 2, 6, 1, (0.5, 0.5, 1.0), [P_] * 6, visc)
    add("euler_p2", 2, 2, 2, 2, 1, (1.0, 1.0, 1.0), [P_] * 6, params(mu=0.0, u=0.3, v=0.2))
    add("source_p2", 2, 2, 2, 2, 1, (1.0, 1.0, 1.0), [P_] * 6, params(mu=1e-2, source=(0.0, 0.3, 0.0, 0.0, 0.0)))

    # curved (non-affine) elements: per-point geometry
    def add_curved(name, nx, ny, nz, p, q, nodes, bounds, prm, amp=0.05):
        U = random_state(prm, nx * ny * nz, (p + 1) ** 3, rng, amp)
        out.append(Case(name, nx, ny, nz, p, q, nodes, bounds, prm, U))

    add_curved("bump_p2_q2", 3, 2, 2, 2, 2, bump_nodes(3, 2, 2, 2, 2.0, 1.0, 0.5),
               [F_, F_, NS_, W_, P_, P_], params(mu=1e-2, u=0.3))
    add_curved("bump_p3_q3", 3, 2, 1, 3, 3, bump_nodes(3, 2, 1, 3, 2.0, 1.0, 0.5),
               [F_, F_, W_, F_, P_, P_], params(mu=5e-3, u=0.3, source=(0.0, 0.2, 0.0, 0.0, 0.0)))
    add_curved("sine_periodic_p2_q2", 2, 2, 2, 2, 2, sine_nodes(2, 2, 2, 2, 1.0, 1.0, 1.0, 0.04),
               [P_] * 6, visc)
    add_curved("sine_euler_p3_q2", 2, 2, 2, 3, 2, sine_nodes(2, 2, 2, 2, 1.0, 1.0, 1.0, 0.04),
               [P_] * 6, params(mu=0.0, u=0.3, v=0.2))
    return out


def run_cases():
    out = []
    # isentropic vortex (Euler), periodic [0,10]^3, RK4 dt 0.01
    nx = ny = 4
    nz = 2
    nodes = box_nodes(nx, ny, nz, 1, 10.0, 10.0, 5.0)
    prm = params(mu=0.0, c=math.sqrt(1.4), u=1.0, v=1.0)  # rho = p = 1
    xyz = node_coords(nx, ny, nz, 2, 1, nodes)
    U = isentropic_vortex(xyz).reshape(-1)
    out.append(Case("vortex_rk4", nx, ny, nz, 2, 1, nodes, [P_] * 6, prm, U, scheme=0, dt=0.01, nsteps=10))
    # Taylor-Green vortex, Re 1600, Ma 0.1, periodic [0, 2pi]^3, p = 3
    n = 3
    L = 2 * math.pi
    nodes = box_nodes(n, n, n, 1, L, L, L)
    prm = params(mu=1.0 / 1600.0, c=10.0, u=0.0, v=0.0, w=0.0)  # rho0 = 1, p0 = 1/(gamma Ma^2)
    xyz = node_coords(n, n, n, 3, 1, nodes)
    U = taylor_green(xyz).reshape(-1)
    dt = 0.2 * (L / n) / ((2 * 3 + 1) * (10.0 + 1.0))
    out.append(Case("tgv_rk4", n, n, n, 3, 1, nodes, [P_] * 6, prm, U, scheme=0, dt=dt, nsteps=5))
    out.append(Case("tgv_tvdrk3", n, n, n, 3, 1, nodes, [P_] * 6, prm, U, scheme=1, dt=dt, nsteps=5))
    # channel with walls, inflow and outflow, TVD-RK3
    rng = np.random.default_rng(7)
    nodes = box_nodes(3, 2, 2, 1, 2.0, 1.0, 1.0)
    prm = params(mu=1e-2, u=0.3)
    U = random_state(prm, 12, 27, rng, 0.02)
    out.append(Case("channel_tvdrk3", 3, 2, 2, 2, 1, nodes, [IN_, OUT_, NS_, W_, P_, P_], prm, U,
                    scheme=1, dt=2e-3, nsteps=5))
    # sinusoidally mapped channel (curved q = 3 elements), no-slip walls, body force
    nodes = sine_nodes(3, 2, 2, 3, 2.0, 1.0, 1.0, 0.05, walls=True)
    prm = params(mu=1e-2, u=0.3, source=(0.0, 0.05, 0.0, 0.0, 0.0))
    U = random_state(prm, 12, 27, rng, 0.02)
    out.append(Case("sine_channel_tvdrk3", 3, 2, 2, 2, 3, nodes, [P_, P_, NS_, NS_, P_, P_], prm, U,
                    scheme=1, dt=2e-3, nsteps=5))
    return out


def long_run_cases():
    """The benchmark configurations at their own step counts, sized for the
    reference CPU solver: the isentropic vortex in full (8^3, p = 2, 100 RK4
    steps of dt 0.01 on [0,10]^3) and the Taylor-Green vortex (Re 1600,
    Ma 0.1) at 8^3 hexes, p = 3, for 1000 RK4 steps."""
    out = []
    n = 8
    nodes = box_nodes(n, n, n, 1, 10.0, 10.0, 10.0)
    prm = params(mu=0.0, c=math.sqrt(1.4), u=1.0, v=1.0)  # rho = p = 1
    U = isentropic_vortex(node_coords(n, n, n, 2, 1, nodes)).reshape(-1)
    out.append(Case("vortex_8_p2_100", n, n, n, 2, 1, nodes, [P_] * 6, prm, U, scheme=0, dt=0.01, nsteps=100))
    L = 2 * math.pi
    nodes = box_nodes(n, n, n, 1, L, L, L)
    prm = params(mu=1.0 / 1600.0, c=10.0, u=0.0, v=0.0, w=0.0)
    U = taylor_green(node_coords(n, n, n, 3, 1, nodes)).reshape(-1)
    dt = 0.2 * (L / n) / ((2 * 3 + 1) * (10.0 + 1.0))
    out.append(Case("tgv_8_p3_1000", n, n, n, 3, 1, nodes, [P_] * 6, prm, U, scheme=0, dt=dt, nsteps=1000))
    return out
