"""Multi-GPU decomposition of the hot path: one process per GPU.

Two ways to shard (boxes are the unit of work):

* ``balance_boxes`` -- independent boxes (the benchmark's default, and a
  level's boxes): each rank takes a set of whole boxes, balanced by zone
  count with the longest-processing-time rule; no data-path collective.
* ``SlabHalo`` -- one periodic patch cut into z-slabs, one per rank, with
  the analogue of the driver's SYNC (AsterX/schedule.ccl:110-115,157-164):
  after the local periodic ghost fill, the ng ghost k-planes of every
  listed grid function are replaced by the neighbours' planes.  A k-plane
  of the engine's layout is contiguous (f[i + sy j + sz k]), so the halo of
  a field is two contiguous slices: no pack kernel.  The exchange is one
  batch of point-to-point operations (NCCL send/recv over NVLink on GPUs,
  gloo on CPU); with one rank it reduces to the periodic wrap.

Plane mapping (local indices, nz interior cells of the rank, v = 1 for a
field vertex-centred in z, else 0): the lower ghosts [0, ng) receive the
lower neighbour's planes [nz_b, nz_b + ng); the upper ghosts
[ng + nz + v, ng + nz + v + ng) receive the upper neighbour's planes
[ng + v, 2 ng + v).  For one rank this is exactly the periodic wrap
i -> ng + (i - ng) mod nz of the single-box ghost fill.
"""
from __future__ import annotations

from typing import Dict, Iterable, List, Sequence, Tuple

from .abi import CONS, Layout

EVOLVED = CONS + ["Avec_x", "Avec_y", "Avec_z", "Psi"]
PRIMS = ["rho", "velx", "vely", "velz", "eps", "press", "temperature", "Ye", "entropy",
         "Bvecx", "Bvecy", "Bvecz"]

# z-centring of the grid functions a substep exchanges (0: vertex in z)
_VERTEX_Z = {"Avec_x", "Avec_y", "Psi", "gxx", "gxy", "gxz", "gyy", "gyz", "gzz", "alp",
             "betax", "betay", "betaz", "kxx", "kxy", "kxz", "kyy", "kyz", "kzz",
             "dBz_stag"}


def vertex_in_z(name: str) -> bool:
    return name in _VERTEX_Z


def balance_boxes(zones: Sequence[int], world: int) -> List[List[int]]:
    """Box indices per rank, largest boxes first onto the least-loaded rank
    (ties to the lower rank): every box exactly once, and the largest load
    is at most 4/3 of the optimum."""
    loads = [0] * world
    out: List[List[int]] = [[] for _ in range(world)]
    for b in sorted(range(len(zones)), key=lambda q: (-zones[q], q)):
        r = min(range(world), key=lambda q: (loads[q], q))
        out[r].append(b)
        loads[r] += zones[b]
    for lst in out:
        lst.sort()
    return out


def slab_ranges(nz: int, world: int) -> List[Tuple[int, int]]:
    """(first global cell, cells) of each rank's z-slab, as even as possible."""
    base, extra = divmod(nz, world)
    out, k0 = [], 0
    for r in range(world):
        n = base + (1 if r < extra else 0)
        out.append((k0, n))
        k0 += n
    return out


class SlabHalo:
    """Ghost-plane exchange of a z-slab decomposition (see the module
    docstring).  `layout` is this rank's box (n[2] = its slab's cells)."""

    def __init__(self, layout: Layout, rank: int, world: int, group=None):
        if layout.n[2] < layout.ng:
            raise ValueError("a slab must be at least ng cells thick")
        self.L = layout
        self.rank = rank
        self.world = world
        self.group = group
        self.up = (rank + 1) % world
        self.down = (rank - 1) % world
        self.plane = layout.sz  # elements per k-plane

    def _slices(self, t, name):
        L, ng, nz, p = self.L, self.L.ng, self.L.n[2], self.plane
        v = 1 if vertex_in_z(name) else 0
        send_up = t[nz * p:(nz + ng) * p]
        send_down = t[(ng + v) * p:(2 * ng + v) * p]
        recv_low = t[0:ng * p]
        recv_high = t[(ng + nz + v) * p:(2 * ng + nz + v) * p]
        return send_up, send_down, recv_low, recv_high

    def exchange(self, tensors: Dict[str, "object"], names: Iterable[str]) -> None:
        names = list(names)
        if self.world == 1:
            for n in names:
                su, sd, rl, rh = self._slices(tensors[n], n)
                rl.copy_(su)
                rh.copy_(sd)
            return
        import torch.distributed as dist
        ops, bufs = [], []
        for n in names:
            su, sd, rl, rh = self._slices(tensors[n], n)
            # receive into separate buffers: a view being received into
            # must not overlap a view being sent
            bl, bh = rl.clone(), rh.clone()
            bufs.append((rl, bl, rh, bh))
            ops += [dist.P2POp(dist.isend, su.contiguous(), self.up, self.group),
                    dist.P2POp(dist.isend, sd.contiguous(), self.down, self.group),
                    dist.P2POp(dist.irecv, bl, self.down, self.group),
                    dist.P2POp(dist.irecv, bh, self.up, self.group)]
        for req in dist.batch_isend_irecv(ops):
            req.wait()
        for rl, bl, rh, bh in bufs:
            rl.copy_(bl)
            rh.copy_(bh)


def slab_layout(n_global: Tuple[int, int, int], ng: int, rank: int, world: int
                ) -> Tuple[Layout, int]:
    """This rank's box of a periodic patch on [0, 1]^3 cut into z-slabs, and
    the global index of its first interior cell."""
    k0, nz = slab_ranges(n_global[2], world)[rank]
    dx = tuple(1.0 / v for v in n_global)
    L = Layout((n_global[0], n_global[1], nz), ng, dx, (0.0, 0.0, k0 * dx[2]))
    return L, k0


def slab_substep(eng, L, f, fn, params, eos, alpha, beta, gamma, dt, halo: SlabHalo):
    """One RK substep of a rank's slab (axb_substep's sequence with the
    neighbours' ghost planes): RHS group, stage update, local periodic fill
    and halo exchange of the evolved variables, post-step group, local fill
    and exchange of the primitives."""
    eng.rhs_group(L, f, params, eos)
    eng.rk_stage(L, f, fn, f, f, alpha, beta, gamma, dt)
    eng.sync_periodic(L, f, EVOLVED)
    halo.exchange(f, EVOLVED)
    eng.con2prim_group(L, f, params, eos)
    eng.sync_periodic(L, f, PRIMS)
    halo.exchange(f, PRIMS)
