"""The block decomposition and halo exchange of dgpr_b200.halo on CPU ranks
(gloo): every rank extends its block with the element layers its neighbours
send, evaluates the residual of the extended block with the CPU oracle, and
its owned elements' residual f = -Minv R must equal the single-rank
residual of the whole mesh.  Bar: 1e-13 relative L2 per rank.  The owned
elements see the same states in the same order; a ghost element reached
across a periodic boundary is a translated copy whose Jacobian, formed from
node differences at coordinates shifted by the period, rounds differently
in the last bits (affine meshes agree bit for bit, the curved case to about
1e-14).

Cases: a periodic Taylor-Green box split along z and along x over two ranks
(each rank is then the other's neighbour on both sides), walls in y split
along y (a physical boundary on one side of each block), a curved (q = 2)
periodic mesh split along z, and four ranks in a 2 x 1 x 2 layout (edge and
corner ghosts)."""
import datetime
import math
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _case(name):
    from tests import cases as C
    L = 2 * math.pi
    if name == "tgv":
        n, p, q = 4, 2, 1
        nodes = C.box_nodes(n, n, n, q, L, L, L)
        prm = C.params(mu=1.0 / 100.0, c=3.0, u=0.0)
        U = C.taylor_green(C.node_coords(n, n, n, p, q, nodes))
        return (n, n, n, p, q), nodes, [-2] * 6, (L, L, L), prm, U
    if name == "walls":
        nx, ny, nz, p, q = 4, 4, 2, 2, 1
        nodes = C.box_nodes(nx, ny, nz, q, 2.0, 1.0, 1.0)
        prm = C.params(mu=1e-2, u=0.2)
        rng = np.random.default_rng(3)
        U = np.tile(prm[6:11], (nx * ny * nz, (p + 1) ** 3, 1)).transpose(0, 2, 1).copy()
        U *= 1.0 + 0.01 * rng.standard_normal(U.shape)
        return (nx, ny, nz, p, q), nodes, [-2, -2, -7, -4, -2, -2], (2.0, 1.0, 1.0), prm, U
    if name == "curved":
        n, p, q = 4, 2, 2
        nodes = C.sine_nodes(n, n, n, q, L, L, L, 0.1)
        prm = C.params(mu=1.0 / 100.0, c=3.0, u=0.0)
        U = C.taylor_green(C.node_coords(n, n, n, p, q, nodes))
        return (n, n, n, p, q), nodes, [-2] * 6, (L, L, L), prm, U
    raise KeyError(name)


def _rank_main(rank, world, port, name, dims, out):
    import torch.distributed as dist

    import oracle
    from dgpr_b200 import halo
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        (nx, ny, nz, p, q), nodes, bounds, period, prm, U = _case(name)
        nb, nq = (p + 1) ** 3, (q + 1) ** 3
        plan = halo.BlockPlan(nx, ny, nz, dims, rank, bounds, period)
        Ug = np.asarray(U, dtype=np.float64).reshape(nz, ny, nx, 5 * nb)
        block = np.ascontiguousarray(plan.owned(Ug))
        ghosts = halo.exchange(plan, block)
        fill = np.repeat(prm[6:11], nb)  # free-stream state, [5][nb]
        Ue = plan.assemble(block, ghosts, fill)
        Xe = plan.extended_nodes(np.asarray(nodes).reshape(nz, ny, nx, nq * 3))
        ex, ey, ez = plan.extended_shape()
        m = oracle.Mesh(ex, ey, ez, p, q, Xe.ravel(), plan.extended_bounds())
        _, f = oracle.restatement().residual(m, prm, Ue.ravel())
        f = f.reshape(ez, ey, ex, 5 * nb)[plan.owned_slices()]
        out.put((rank, plan.lo, plan.size, f))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("name,dims", [("tgv", (1, 1, 2)), ("tgv", (2, 1, 1)), ("walls", (1, 2, 1)),
                                       ("curved", (1, 1, 2)), ("tgv", (2, 1, 2))],
                         ids=["tgv-z2", "tgv-x2", "walls-y2", "curved-z2", "tgv-2x1x2"])
def test_block_halo_residual_equals_single_rank(name, dims):
    import torch.multiprocessing as mp

    import oracle
    world = dims[0] * dims[1] * dims[2]
    (nx, ny, nz, p, q), nodes, bounds, _, prm, U = _case(name)
    _, fg = oracle.restatement().residual(oracle.Mesh(nx, ny, nz, p, q, nodes, bounds), prm,
                                          np.asarray(U).ravel())
    fg = fg.reshape(nz, ny, nx, -1)
    ctx = mp.get_context("spawn")
    q_out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, name, dims, q_out)) for r in range(world)]
    for pr in procs:
        pr.start()
    res = [q_out.get(timeout=180) for _ in procs]
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    covered = np.zeros(fg.shape[:3], dtype=int)
    for rank, (i0, j0, k0), (sx, sy, sz), f in res:
        ref = fg[k0:k0 + sz, j0:j0 + sy, i0:i0 + sx]
        err = np.linalg.norm(f - ref) / np.linalg.norm(ref)
        assert err <= 1e-13, (rank, err)
        covered[k0:k0 + sz, j0:j0 + sy, i0:i0 + sx] += 1
    assert np.all(covered == 1), "the blocks tile the mesh once"


def test_block_plan_neighbours():
    from dgpr_b200 import halo
    # two ranks along periodic z: each is the other's neighbour on both z sides
    a = halo.BlockPlan(4, 4, 4, (1, 1, 2), 0, [-2] * 6, (1.0, 1.0, 1.0))
    assert a.nbr == [None, None, None, None, 1, 1] and a.extended_shape() == (4, 4, 4)
    # a wall direction: no ghost on the physical boundary
    b = halo.BlockPlan(4, 4, 2, (1, 2, 1), 1, [-2, -2, -7, -4, -2, -2], (1.0, 1.0, 1.0))
    assert b.nbr == [None, None, 0, None, None, None] and b.extended_bounds()[2:4] == [-3, -4]
    with pytest.raises(ValueError):
        halo.BlockPlan(5, 4, 4, (2, 1, 1), 0, [-2] * 6, (1.0, 1.0, 1.0))
