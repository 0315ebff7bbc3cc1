"""Block decomposition of a structured hex mesh over ranks, and the halo
exchange of one element layer per face, on the host (numpy arrays moved with
torch.distributed point-to-point calls; the gloo backend on CPU).

The reference decomposes its mesh into npx x npy x npz blocks
(geometry_distributed.cpp:504-579) and exchanges the face traces of the
partition faces every residual evaluation (solve.cpp:258-387: MPI_Issend of
each partition face's trace, MPI_Recv of the neighbour's).  This module keeps
the same decomposition -- contiguous blocks, rank = px + npx (py + npy pz) --
and exchanges the element states of the layer behind every partition face:
a rank extends its block by one ghost element on each partitioned side, so a
residual over the extended block gives the owned elements exactly the
single-rank residual (an element's residual reads only its own state and its
face neighbours').  On a GPU the same plan would move the partition faces'
trace slices [10][P^2] of the stage kernels' trace buffer instead (fewer
bytes: 10 P^2 against 5 P^3 values per face), between the stages; that path
is not built: this library runs on one GPU.

The geometry is static: every rank builds the nodes of its extended block
from the mesh description, translating elements reached across a periodic
boundary by the period so the extended block is geometrically continuous.
The states of ghost elements that touch the block only along an edge or a
corner are not exchanged (no owned element reads them); they are set to the
reference free-stream state so every ghost is a valid state.
"""
import numpy as np

PERIODIC = -2
_FREESTREAM = -3


class BlockPlan:
    """One rank's block of an nx x ny x nz mesh split over dims = (npx, npy,
    npz) ranks.  bounds: the global btype codes [-x, +x, -y, +y, -z, +z]
    (-2 periodic, negative btypes otherwise); period: the domain lengths, for
    ghosts across periodic boundaries."""

    def __init__(self, nx, ny, nz, dims, rank, bounds, period):
        self.n = (nx, ny, nz)
        self.dims = tuple(int(d) for d in dims)
        if any(self.n[a] % self.dims[a] for a in range(3)):
            raise ValueError("every direction's element count must divide by its rank count")
        npx, npy, _ = self.dims
        self.rank = rank
        self.coord = (rank % npx, (rank // npx) % npy, rank // (npx * npy))
        self.bounds = list(bounds)
        self.period = period
        self.size = tuple(self.n[a] // self.dims[a] for a in range(3))
        self.lo = tuple(self.coord[a] * self.size[a] for a in range(3))
        # per side: the neighbour rank across it, or None at a physical boundary
        self.nbr = []
        for a in range(3):
            for s in (-1, 1):
                c = list(self.coord)
                c[a] += s
                periodic = self.bounds[2 * a] == PERIODIC
                if 0 <= c[a] < self.dims[a]:
                    self.nbr.append(self._rank_of(c))
                elif periodic and self.dims[a] > 1:
                    c[a] %= self.dims[a]
                    self.nbr.append(self._rank_of(c))
                else:
                    self.nbr.append(None)
        # ghost layers on each side: where a neighbour rank sits across it
        self.ghost = [self.nbr[f] is not None for f in range(6)]

    def _rank_of(self, c):
        return c[0] + self.dims[0] * (c[1] + self.dims[1] * c[2])

    def extended_shape(self):
        """(nx, ny, nz) of the owned block with its ghost layers."""
        return tuple(self.size[a] + int(self.ghost[2 * a]) + int(self.ghost[2 * a + 1]) for a in range(3))

    def extended_bounds(self):
        """btype codes of the extended block: the global ones on undivided
        directions and physical boundaries; free-stream on the outer side of
        a ghost layer (it only bounds ghost elements)."""
        b = []
        for a in range(3):
            for s in range(2):
                f = 2 * a + s
                if self.dims[a] == 1:
                    b.append(self.bounds[f])
                else:
                    b.append(_FREESTREAM if self.ghost[f] else self.bounds[f])
        return b

    def owned_slices(self):
        """Index slices (z, y, x) of the owned elements inside the extended block."""
        return tuple(slice(int(self.ghost[2 * a]), int(self.ghost[2 * a]) + self.size[a]) for a in (2, 1, 0))

    # ---- element arrays in the reference's order e = i + nx (j + ny k), as
    # [nz][ny][nx][...] views
    def owned(self, glob):
        """The owned block of a global per-element array glob[nz][ny][nx][...]."""
        (i0, j0, k0), (sx, sy, sz) = self.lo, self.size
        return glob[k0:k0 + sz, j0:j0 + sy, i0:i0 + sx]

    def layer(self, block, f):
        """The element layer of an owned block next to side f (what the
        neighbour across f needs), as a contiguous array."""
        a, s = f // 2, f % 2
        idx = [slice(None)] * 3
        idx[2 - a] = slice(-1, None) if s else slice(0, 1)
        return np.ascontiguousarray(block[tuple(idx)])

    def assemble(self, block, ghosts, fill):
        """The extended block: the owned block, the received ghost layers
        (ghosts[f], or None where there is none) and `fill` on the edge and
        corner ghost elements."""
        ext = np.empty(self.extended_shape()[::-1] + block.shape[3:], dtype=block.dtype)
        ext[...] = fill
        ext[self.owned_slices()] = block
        for f in range(6):
            if not self.ghost[f]:
                continue
            a, s = f // 2, f % 2
            idx = list(self.owned_slices())
            idx[2 - a] = slice(-1, None) if s else slice(0, 1)
            ext[tuple(idx)] = ghosts[f]
        return ext

    def extended_nodes(self, nodes):
        """Node coordinates of the extended block, ghosts included, from the
        global node array nodes[nz][ny][nx][(q+1)^3 * 3]: the geometry is
        static, so every rank builds its halo's from the mesh description (as
        the reference's geometry_distributed.cpp does for its partition
        faces); an element reached across a periodic boundary is translated
        by the period."""
        g = [int(self.ghost[2 * a]) for a in range(3)]
        shape = self.extended_shape()
        out = np.empty(shape[::-1] + nodes.shape[3:], dtype=nodes.dtype)
        for ke in range(shape[2]):
            for je in range(shape[1]):
                for ie in range(shape[0]):
                    idx, shift = [], np.zeros(3)
                    for a, e in zip(range(3), (ie, je, ke)):
                        gi = self.lo[a] - g[a] + e
                        w = gi // self.n[a]
                        shift[a] = w * self.period[a]
                        idx.append(gi - w * self.n[a])
                    xyz = nodes[idx[2], idx[1], idx[0]].reshape(-1, 3) + shift
                    out[ke, je, ie] = xyz.reshape(nodes.shape[3:])
        return out


def exchange(plan, block, group=None):
    """Sends every partition-face layer of `block` (owned, [nz][ny][nx][...],
    float64) to the rank across it and receives that rank's layer facing this
    block: returns ghosts[f] for the six sides (None where there is no
    neighbour).  Non-blocking sends and receives, all posted before any wait,
    so ranks that are each other's neighbour on two sides (two ranks along a
    periodic direction) do not deadlock; a side's tag is the side index the
    receiver files it under."""
    import torch
    import torch.distributed as dist
    reqs, recv = [], {}
    for f in range(6):
        if plan.nbr[f] is None:
            continue
        lay = torch.from_numpy(plan.layer(block, f))
        # the neighbour files this layer as its ghost on the opposite side
        reqs.append(dist.isend(lay, plan.nbr[f], group=group, tag=f ^ 1))
        shape = list(block.shape)
        shape[2 - f // 2] = 1
        buf = torch.empty(shape, dtype=torch.float64)
        reqs.append(dist.irecv(buf, plan.nbr[f], group=group, tag=f))
        recv[f] = buf
    for r in reqs:
        r.wait()
    return [recv[f].numpy() if f in recv else None for f in range(6)]
