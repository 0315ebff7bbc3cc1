"""Flow functionals and seeded initial states for the adjoint checks, in torch
(float64), on uniform box meshes [0,lx]x[0,ly]x[0,lz] of nx x ny x nz
elements.

These sit on the harness side of the C ABI: the reference has no functionals,
no Fourier-mode initial state and no adjoint.  Every quantity is a quadrature
over the solver's own discretisation -- the order-p equispaced Lagrange basis
evaluated at the P = p+1 Gauss-Legendre points per direction
(basis.cpp:64-170, quadrature.cpp:187-205) -- so J(U) is a smooth function of
the nodal state U[e][r][b] that torch differentiates exactly.
"""
import math

import numpy as np
import torch

from . import gauss_legendre, lagrange1d, lagrange1d_deriv


class BoxQuadrature:
    """Values and physical gradients of a nodal state at the Gauss points of a
    uniform box mesh."""

    def __init__(self, nx, ny, nz, p, lx, ly, lz, device="cpu"):
        self.nx, self.ny, self.nz, self.p = nx, ny, nz, p
        self.h = (lx / nx, ly / ny, lz / nz)
        P = p + 1
        x, w = gauss_legendre(P, 0.0, 1.0)
        B = np.array([[lagrange1d(i, p, xq) for i in range(P)] for xq in x])
        Bd = np.array([[lagrange1d_deriv(i, p, xq) for i in range(P)] for xq in x])
        dd = dict(dtype=torch.float64, device=device)
        self.B, self.Bd = torch.tensor(B, **dd), torch.tensor(Bd, **dd)
        wq = torch.tensor(w, **dd)
        self.W = torch.einsum("a,b,c->abc", wq, wq, wq) * (self.h[0] * self.h[1] * self.h[2])  # [z][y][x]
        self.volume = lx * ly * lz

    def fields(self, U):
        """(V, dV/dx, dV/dy, dV/dz) at the Gauss points, each [E][5][z][y][x]."""
        P = self.p + 1
        Ue = U.reshape(-1, 5, P, P, P)
        B, Bd = self.B, self.Bd
        V = torch.einsum("ck,bj,ai,erkji->ercba", B, B, B, Ue)
        Dx = torch.einsum("ck,bj,ai,erkji->ercba", B, B, Bd, Ue) / self.h[0]
        Dy = torch.einsum("ck,bj,ai,erkji->ercba", B, Bd, B, Ue) / self.h[1]
        Dz = torch.einsum("ck,bj,ai,erkji->ercba", Bd, B, B, Ue) / self.h[2]
        return V, Dx, Dy, Dz

    def integrate(self, q):
        """Integral over the domain of a field q[E][z][y][x] at the Gauss points."""
        return (q * self.W).sum()


def kinetic_energy(U, quad):
    """Volume-averaged kinetic energy (1/|V|) int rho |u|^2 / 2 dV."""
    V, _, _, _ = quad.fields(U)
    rho, m = V[:, 0], V[:, 1:4]
    return quad.integrate(0.5 * (m * m).sum(1) / rho) / quad.volume


def enstrophy(U, quad):
    """Volume-averaged enstrophy (1/|V|) int rho |curl u|^2 / 2 dV, the
    Taylor-Green diagnostic."""
    V, Dx, Dy, Dz = quad.fields(U)
    rho = V[:, 0]
    u = V[:, 1:4] / rho[:, None]

    def grad_u(D):  # d u_i / d x_c = (d m_i - u_i d rho) / rho
        return (D[:, 1:4] - u * D[:, 0:1]) / rho[:, None]

    gx, gy, gz = grad_u(Dx), grad_u(Dy), grad_u(Dz)
    wx = gy[:, 2] - gz[:, 1]
    wy = gz[:, 0] - gx[:, 2]
    wz = gx[:, 1] - gy[:, 0]
    return quad.integrate(0.5 * rho * (wx * wx + wy * wy + wz * wz)) / quad.volume


def wall_shear(U, quad, mu, wall="-y"):
    """Mean wall shear stress tau_xy = mu (du/dy + dv/dx) over the wall y = 0
    ("-y") or y = ly ("+y") of a box mesh, from the wall elements' own
    polynomials (one-sided, as the solver's face terms take the interior
    trace), integrated with the P x P Gauss points of the face.  The channel
    diagnostic (config 5's skin friction); u = m / rho."""
    P = quad.p + 1
    nx, ny, nz = quad.nx, quad.ny, quad.nz
    hx, hy, hz = quad.h
    Ue = U.reshape(nz, ny, nx, 5, P, P, P)  # [k][j][i][r][z][y][x]
    j, end = (0, 0.0) if wall == "-y" else (ny - 1, 1.0)
    Uw = Ue[:, j]  # [k][i][r][z][y][x]
    dd = dict(dtype=torch.float64, device=U.device)
    p = quad.p
    Ev = torch.tensor([lagrange1d(a, p, end) for a in range(P)], **dd)
    Dv = torch.tensor([lagrange1d_deriv(a, p, end) for a in range(P)], **dd)
    B, Bd = quad.B, quad.Bd
    V = torch.einsum("cz,y,ax,kirzyx->kirca", B, Ev, B, Uw)
    Vy = torch.einsum("cz,y,ax,kirzyx->kirca", B, Dv, B, Uw) / hy
    Vx = torch.einsum("cz,y,ax,kirzyx->kirca", B, Ev, Bd, Uw) / hx
    rho = V[:, :, 0]
    u, v = V[:, :, 1] / rho, V[:, :, 2] / rho
    dudy = (Vy[:, :, 1] - u * Vy[:, :, 0]) / rho
    dvdx = (Vx[:, :, 2] - v * Vx[:, :, 0]) / rho
    x, w = gauss_legendre(P, 0.0, 1.0)
    wq = torch.tensor(w, **dd)
    W = torch.einsum("c,a->ca", wq, wq) * (hx * hz)
    area = nx * hx * nz * hz
    return (mu * (dudy + dvdx) * W).sum() / area


def box_node_coords(nx, ny, nz, p, lx, ly, lz):
    """Physical coordinates of the solution nodes of a uniform box mesh,
    [E][(p+1)^3][3], element e = i + nx (j + ny k), node b = x + P (y + P z)."""
    P = p + 1
    r = np.arange(P) / p if p > 0 else np.zeros(1)
    hx, hy, hz = lx / nx, ly / ny, lz / nz
    ez, ey, ex, kz, ky, kx = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), r, r, r, indexing="ij")
    X = np.stack([(ex + kx) * hx, (ey + ky) * hy, (ez + kz) * hz], axis=-1)
    return X.reshape(nx * ny * nz, P ** 3, 3)


class FourierModes:
    """Uniform flow plus M seeded Fourier velocity modes,
    u(x) = u0 + sum_m a_m sin(k_m . x + phi_m), uniform density and pressure;
    the amplitudes a (M x 3) are the parameters.  Wavevector components are
    integers in 1..kmax (periodic on [0, 2 pi]^3)."""

    def __init__(self, xyz, gamma, rho, p, u0, nmodes=8, kmax=4, amp=0.05, seed=0, device="cpu"):
        rng = np.random.default_rng(seed)
        self.k = rng.integers(1, kmax + 1, size=(nmodes, 3)).astype(np.float64)
        self.phi = rng.uniform(0.0, 2 * math.pi, size=nmodes)
        self.a0 = amp * rng.standard_normal((nmodes, 3))
        dd = dict(dtype=torch.float64, device=device)
        arg = np.einsum("enc,mc->enm", xyz, self.k) + self.phi  # [E][nb][M]
        self.S = torch.tensor(np.sin(arg), **dd)
        self.gamma, self.rho, self.p = gamma, rho, p
        self.u0 = torch.tensor(u0, **dd)

    def amplitudes(self, device="cpu"):
        return torch.tensor(self.a0, dtype=torch.float64, device=device)

    def state(self, a):
        """Nodal state U[E][5][nb] (flattened) for amplitudes a [M][3]."""
        u = self.u0 + torch.einsum("enm,mc->enc", self.S, a)  # [E][nb][3]
        rho = self.rho
        E = self.p / (self.gamma - 1.0) + 0.5 * rho * (u * u).sum(-1)
        cons = torch.cat([torch.full_like(E, rho)[..., None], rho * u, E[..., None]], dim=-1)  # [E][nb][5]
        return cons.transpose(1, 2).reshape(-1)
