"""Spatial domain decomposition of one scene across ranks: x slabs of grid node
planes with ghost planes, a halo reduce after P2G, a halo broadcast before G2P
and particle migration.  The reference's CPU analogue splits one grid among
threads as per-thread proxy grids summed over z slabs
(MultiThreadForwardSimulation.cpp:179-202); here each rank holds only its slab.

Rank r owns node planes [lo_r, hi_r) along x and the particles whose cell
c = floor((x_0 - min_0) / dx) lies there (cells below the grid count as plane 0,
above it as the last plane).  A particle's stencil covers node planes
c - 1 .. c + 2, so a rank's local grid holds planes [lo_r - 1, hi_r + 2)
clipped to the grid: one ghost plane below its slab, two above.  A forward step
then runs, per rank:

  P2G of the rank's particles into its local grid (owned and ghost planes);
  halo_reduce: the ghost planes' partial sums go to the neighbour that owns
    them, which adds them to its own (ghost plane lo_r - 1 to rank r - 1,
    ghost planes hi_r, hi_r + 1 to rank r + 1);
  the grid update on owned planes;
  halo_broadcast: each owner's boundary planes overwrite the neighbours' ghost
    copies (planes lo_r, lo_r + 1 to rank r - 1, plane hi_r - 1 to rank r + 1);
  G2P and P_op_2 of the rank's particles;
  migrate: particles whose cell left the slab move to the neighbour owning it
    (a particle moves less than a cell per step under the CFL limit, so only
    neighbours exchange).

All traffic is point-to-point between neighbouring ranks with
torch.distributed isend / irecv (NCCL for device tensors over NVLink, gloo for
host tensors); no collective and no copy that reads another GPU's memory
from inside a kernel.  Each slab must be at
least two planes wide.  The grids are tensors of shape (planes, dim_y, dim_z,
channels) in the node order of the engine (plane-major), so a plane is one
contiguous block.
"""
from __future__ import annotations

from typing import Dict, List, Tuple

import torch
import torch.distributed as dist


class SlabDecomposition:
    def __init__(self, nx: int, world: int, rank: int):
        if world < 1 or not 0 <= rank < world:
            raise ValueError("bad rank / world size")
        if nx < 2 * world:
            raise ValueError("every slab needs at least two node planes")
        self.nx, self.world, self.rank = nx, world, rank
        self.bounds = [(r * nx // world, (r + 1) * nx // world) for r in range(world)]
        self.lo, self.hi = self.bounds[rank]
        # local planes [p0, p1): the slab, one ghost plane below, two above
        self.p0 = max(self.lo - 1, 0)
        self.p1 = min(self.hi + 2, nx)

    @property
    def local_planes(self) -> int:
        return self.p1 - self.p0

    def owner_of_cell(self, c: torch.Tensor) -> torch.Tensor:
        """Rank owning each cell index (clamped into the grid)."""
        c = torch.clamp(c, 0, self.nx - 1)
        owner = torch.zeros_like(c)
        for r, (lo, hi) in enumerate(self.bounds):
            owner = torch.where((c >= lo) & (c < hi), torch.full_like(c, r), owner)
        return owner

    # ------------------------------------------------------------ halos
    def _exchange(self, sends: List[Tuple[int, torch.Tensor]], recvs: List[Tuple[int, torch.Tensor]]):
        reqs = [dist.isend(t.contiguous(), peer) for peer, t in sends]
        reqs += [dist.irecv(t, peer) for peer, t in recvs]
        for q in reqs:
            q.wait()

    def halo_reduce(self, grid: torch.Tensor) -> None:
        """Add the neighbours' partial sums of this rank's boundary planes
        (their ghost planes) into it, in place.  grid: (local planes, ...)."""
        r, p0 = self.rank, self.p0
        sends, recvs, adds = [], [], []
        if r > 0:  # my lower ghost -> rank r-1; its upper ghosts -> my planes lo, lo+1
            sends.append((r - 1, grid[self.lo - 1 - p0:self.lo - p0]))
            buf = torch.empty_like(grid[self.lo - p0:self.lo + 2 - p0])
            recvs.append((r - 1, buf))
            adds.append((self.lo - p0, buf))
        if r < self.world - 1:  # my upper ghosts -> rank r+1; its lower ghost -> my plane hi-1
            sends.append((r + 1, grid[self.hi - p0:self.hi + 2 - p0]))
            buf = torch.empty_like(grid[self.hi - 1 - p0:self.hi - p0])
            recvs.append((r + 1, buf))
            adds.append((self.hi - 1 - p0, buf))
        self._exchange(sends, recvs)
        for at, buf in adds:
            grid[at:at + buf.shape[0]] += buf

    def halo_broadcast(self, grid: torch.Tensor) -> None:
        """Overwrite this rank's ghost planes with their owners' values, in place."""
        r, p0 = self.rank, self.p0
        sends, recvs = [], []
        if r > 0:  # my planes lo, lo+1 -> rank r-1's upper ghosts; its plane lo-1 -> my lower ghost
            sends.append((r - 1, grid[self.lo - p0:self.lo + 2 - p0]))
            recvs.append((r - 1, grid[self.lo - 1 - p0:self.lo - p0]))
        if r < self.world - 1:  # my plane hi-1 -> rank r+1's lower ghost; its lo, lo+1 -> my upper ghosts
            sends.append((r + 1, grid[self.hi - 1 - p0:self.hi - p0]))
            recvs.append((r + 1, grid[self.hi - p0:self.hi + 2 - p0]))
        # receive into temporaries, then copy: a view passed to irecv must be contiguous
        tmp = [(peer, torch.empty_like(view)) for peer, view in recvs]
        self._exchange(sends, tmp)
        for (_, view), (_, buf) in zip(recvs, tmp):
            view.copy_(buf)

    # ------------------------------------------------------------ particles
    def migrate(self, cell: torch.Tensor, fields: Dict[str, torch.Tensor]) -> Dict[str, torch.Tensor]:
        """Send the particles whose cell (x index, one per particle) left this
        rank's slab to the neighbour owning it and receive the neighbours'.
        fields: name -> tensor whose first axis is the particle; returns the
        particles kept (in their order), then those from rank - 1, then from
        rank + 1."""
        owner = self.owner_of_cell(cell)
        r = self.rank
        if torch.any((owner < r - 1) | (owner > r + 1)):
            raise RuntimeError("a particle moved past a neighbouring slab in one step")
        keep = owner == r
        names = sorted(fields)
        dev = cell.device
        out_parts: Dict[str, List[torch.Tensor]] = {k: [fields[k][keep]] for k in names}
        peers = [p for p in (r - 1, r + 1) if 0 <= p < self.world]
        # counts first
        send_n = {p: torch.tensor([int(torch.count_nonzero(owner == p))], dtype=torch.int64, device=dev)
                  for p in peers}
        recv_n = {p: torch.zeros(1, dtype=torch.int64, device=dev) for p in peers}
        self._exchange([(p, send_n[p]) for p in peers], [(p, recv_n[p]) for p in peers])
        for k in names:
            sends, recvs = [], []
            for p in peers:
                sends.append((p, fields[k][owner == p]))
                shape = (int(recv_n[p].item()),) + tuple(fields[k].shape[1:])
                recvs.append((p, torch.empty(shape, dtype=fields[k].dtype, device=dev)))
            sends = [(p, t) for p, t in sends if t.shape[0] > 0]
            recvs_nz = [(p, t) for p, t in recvs if t.shape[0] > 0]
            self._exchange(sends, recvs_nz)
            for p, t in recvs:
                out_parts[k].append(t)
        return {k: torch.cat(out_parts[k], 0) for k in names}
