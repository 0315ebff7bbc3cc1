"""The harness functionals (dgpr_b200/functionals.py) on the CPU, against
closed forms they must reproduce exactly (polynomial fields the order-p basis
holds): kinetic energy of a uniform flow, enstrophy of a solid-body
rotation, wall shear of a Poiseuille profile with a linear cross flow; and
torch's gradient of the wall shear against central differences."""
import numpy as np
import pytest
import torch

from dgpr_b200 import functionals as F


def _state(xyz, rho, u, v, w, p, gamma=1.4):
    E = p / (gamma - 1) + 0.5 * rho * (u * u + v * v + w * w)
    U = np.stack([rho + 0 * u, rho * u, rho * v, rho * w, E + 0 * u], axis=1)  # [E][5][nb]
    return torch.tensor(U.reshape(-1), dtype=torch.float64)


def test_kinetic_energy_of_uniform_flow():
    nx, ny, nz, p = 2, 3, 2, 2
    xyz = F.box_node_coords(nx, ny, nz, p, 1.0, 2.0, 1.5)
    x = xyz[..., 0]
    U = _state(xyz, 1.3, 0.2 + 0 * x, -0.1 + 0 * x, 0.05 + 0 * x, 0.7)
    quad = F.BoxQuadrature(nx, ny, nz, p, 1.0, 2.0, 1.5)
    ke = float(F.kinetic_energy(U, quad))
    assert abs(ke - 0.5 * 1.3 * (0.04 + 0.01 + 0.0025)) < 1e-14


@pytest.mark.parametrize("p", [1, 2, 3])
def test_enstrophy_of_solid_body_rotation(p):
    nx, ny, nz, Om = 2, 2, 1, 0.7
    xyz = F.box_node_coords(nx, ny, nz, p, 1.0, 1.0, 0.5)
    x, y = xyz[..., 0], xyz[..., 1]
    U = _state(xyz, 1.0, -Om * y, Om * x, 0 * x, 1.0)
    quad = F.BoxQuadrature(nx, ny, nz, p, 1.0, 1.0, 0.5)
    assert abs(float(F.enstrophy(U, quad)) - 0.5 * (2 * Om) ** 2) < 1e-12


@pytest.mark.parametrize("p", [2, 3])
def test_wall_shear_of_poiseuille_flow(p):
    """u = 4 Ub y (ly - y) / ly^2, v = c x: tau_xy = mu (4 Ub / ly + c) at
    y = 0 and mu (-4 Ub / ly + c) at y = ly, exactly (quadratic u, linear v)."""
    nx, ny, nz, lx, ly, lz = 3, 4, 2, 2.0, 1.0, 1.0
    Ub, c, mu = 1.5, 0.3, 2e-3
    xyz = F.box_node_coords(nx, ny, nz, p, lx, ly, lz)
    x, y = xyz[..., 0], xyz[..., 1]
    U = _state(xyz, 1.0, 4 * Ub * y * (ly - y) / ly ** 2, c * x, 0 * x, 1.0)
    quad = F.BoxQuadrature(nx, ny, nz, p, lx, ly, lz)
    assert abs(float(F.wall_shear(U, quad, mu, "-y")) - mu * (4 * Ub / ly + c)) < 1e-14
    assert abs(float(F.wall_shear(U, quad, mu, "+y")) - mu * (-4 * Ub / ly + c)) < 1e-14


def test_wall_shear_gradient_matches_fd():
    nx, ny, nz, p = 2, 2, 1, 2
    rng = np.random.default_rng(3)
    xyz = F.box_node_coords(nx, ny, nz, p, 1.0, 1.0, 1.0)
    x, y = xyz[..., 0], xyz[..., 1]
    U0 = _state(xyz, 1.0 + 0.1 * np.sin(x), y * (1 - y), 0.1 * x, 0 * x, 1.0)
    U0 = U0 * (1 + 0.01 * torch.tensor(rng.standard_normal(U0.shape)))
    quad = F.BoxQuadrature(nx, ny, nz, p, 1.0, 1.0, 1.0)
    U = U0.clone().requires_grad_(True)
    F.wall_shear(U, quad, 1e-2).backward()
    d = torch.tensor(rng.standard_normal(U0.shape))
    h = 1e-6
    fd = (F.wall_shear(U0 + h * d, quad, 1e-2) - F.wall_shear(U0 - h * d, quad, 1e-2)) / (2 * h)
    an = (U.grad * d).sum()
    assert abs(float(fd - an)) <= 1e-7 * abs(float(an))
