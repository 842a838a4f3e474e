"""Multi-rank (one process per GPU) decomposition of the hydro step.

Two ways to spread work over ranks, both as the reference does with MPI:

* AMR level: whole patches go to ranks (the reference's ProcessorNumber), balanced by
  cell count; each rank advances its patches with one batched launch per stage
  (ppm_b200_solve_level) and the level time step is the minimum over ranks
  (SetLevelTimeStep.C:66-69: CommunicationMinValue).  No data moves inside a step.

* Uniform grid: slabs along z, each with its own 3-cell ghost shell.  Before every step
  the z ghosts are exchanged with the neighbouring slabs (the reference's
  CopyZonesFromGrid between sibling grids), the x and y ghosts are filled locally.
  Every SolvePPM_DE sweep of a slab only reads cells of its own padded array and
  sweeps the transverse ghost pencils too (Grid_SolvePPM_DE.C:86-146), so after each
  step the slabs' active cells equal those of the undivided grid bit for bit.

torch.distributed carries the messages: NCCL between GPUs (device tensors), gloo for
the CPU tests; the code is the same.  Every rank takes the same collective steps in
the same order.
"""
from __future__ import annotations

import heapq

import numpy as np

from . import harness as H


# ---------------------------------------------------------------- AMR level partition
def partition_level(grids, nranks):
    """Patches -> ranks, largest first to the least loaded rank (cell counts incl.
    ghosts).  Returns a list of patch-index lists, one per rank."""
    heap = [(0, r) for r in range(nranks)]
    heapq.heapify(heap)
    parts = [[] for _ in range(nranks)]
    order = sorted(range(len(grids)), key=lambda k: -grids[k].size)
    for k in order:
        load, r = heapq.heappop(heap)
        parts[r].append(k)
        heapq.heappush(heap, (load + grids[k].size, r))
    return parts


def global_min(value, dist, device=None):
    """Minimum of a per-rank float over all ranks (the level time step)."""
    import torch
    t = value if isinstance(value, torch.Tensor) else torch.tensor(
        [float(value)], dtype=torch.float64, device=device)
    if dist is not None and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MIN)
    return t


# ---------------------------------------------------------------- z slabs of a grid
class Slabs:
    """A uniform 3-D grid of `active` cells split along z into `nranks` slabs.

    slab(rank) is the rank's Grid (3 ghost zones on every side, the global cell widths);
    z_range(rank) its global active z range.  bc: the global boundary per dimension
    ("periodic" or "outflow")."""

    def __init__(self, active, nranks, width=1.0, bc=("periodic",) * 3):
        assert len(active) == 3
        self.active = tuple(int(a) for a in active)
        self.nranks = int(nranks)
        nz = self.active[2]
        assert nz >= 3 * nranks, "every slab needs at least 3 active z layers"
        base, rem = divmod(nz, nranks)
        self.z0 = []
        z = 0
        for r in range(nranks):
            self.z0.append(z)
            z += base + (1 if r < rem else 0)
        self.z0.append(nz)
        self.width = width if isinstance(width, (tuple, list)) else (width,) * 3
        self.bc = tuple(bc)
        self.global_grid = H.Grid.uniform(self.active, width=self.width)

    def z_range(self, rank):
        return self.z0[rank], self.z0[rank + 1]

    def slab(self, rank):
        lo, hi = self.z_range(rank)
        nz = hi - lo
        dz = self.width[2] / self.active[2]
        shape = (self.active[0], self.active[1], nz)
        g = H.Grid.uniform(shape, width=(self.width[0], self.width[1], dz * nz))
        return g

    def scatter(self, global_fields, rank):
        """The rank's padded slab cut from a padded global field set (numpy)."""
        lo, hi = self.z_range(rank)
        ng = H.NGHOST
        return {k: np.ascontiguousarray(v[lo:hi + 2 * ng]) for k, v in global_fields.items()}

    def gather_active(self, slab_fields, rank, out):
        """Write the slab's active z layers into a padded global field set."""
        lo, hi = self.z_range(rank)
        ng = H.NGHOST
        for k, v in slab_fields.items():
            a = v.cpu().numpy() if hasattr(v, "cpu") else v
            out[k][ng + lo:ng + hi] = a[ng:ng + hi - lo]

    def neighbours(self, rank):
        """(below, above) ranks along z; None at an outflow edge."""
        r = self.nranks
        periodic = self.bc[2] == "periodic"
        below = rank - 1 if rank > 0 else (r - 1 if periodic else None)
        above = rank + 1 if rank < r - 1 else (0 if periodic else None)
        return below, above

    def local_bc(self):
        """Ghost fill of a slab by the device kernel: x, y from the global boundary,
        z left to the halo exchange."""
        return (self.bc[0], self.bc[1], "none")

    def exchange(self, fields, rank, dist):
        """Fill the z ghosts of the rank's slab from its neighbours (3 layers each way).

        fields: the slab's padded tensors (torch; device for NCCL, CPU for gloo).  At an
        outflow edge the ghosts copy the edge layer.  The send/recv pairs are posted
        together (batch_isend_irecv), so every rank takes part in the same exchange."""
        import torch

        ng = H.NGHOST
        names = sorted(fields)
        below, above = self.neighbours(rank)
        nz = fields[names[0]].shape[0] - 2 * ng
        # pack: lowest / highest 3 active layers of every field
        send_lo = torch.stack([fields[k][ng:2 * ng] for k in names]).contiguous()
        send_hi = torch.stack([fields[k][nz:nz + ng] for k in names]).contiguous()
        recv_lo = torch.empty_like(send_lo)
        recv_hi = torch.empty_like(send_hi)
        world = dist.get_world_size() if (dist is not None and dist.is_initialized()) else 1
        if world == 1:
            # one slab: the neighbours are this rank itself (periodic) or absent
            if below is not None:
                recv_lo.copy_(send_hi)
            if above is not None:
                recv_hi.copy_(send_lo)
        else:
            # upward flow (tag 0): my top layers go to the slab above, the slab below
            # sends me its top layers; then downward flow (tag 1).  Posting both flows
            # in the same order on every rank keeps the matching right also where the
            # neighbour below and above is the same rank (two slabs, periodic) and the
            # backend matches messages by order.
            ops = []
            if above is not None:
                ops.append(dist.P2POp(dist.isend, send_hi, above, tag=0))
            if below is not None:
                ops.append(dist.P2POp(dist.irecv, recv_lo, below, tag=0))
            if below is not None:
                ops.append(dist.P2POp(dist.isend, send_lo, below, tag=1))
            if above is not None:
                ops.append(dist.P2POp(dist.irecv, recv_hi, above, tag=1))
            if ops:
                for req in dist.batch_isend_irecv(ops):
                    req.wait()
        for i, k in enumerate(names):
            t = fields[k]
            if below is not None:
                t[0:ng] = recv_lo[i]
            else:
                t[0:ng] = t[ng:ng + 1].expand(ng, *t.shape[1:])
            if above is not None:
                t[nz + ng:nz + 2 * ng] = recv_hi[i]
            else:
                t[nz + ng:nz + 2 * ng] = t[nz + ng - 1:nz + ng].expand(ng, *t.shape[1:])
        return fields
