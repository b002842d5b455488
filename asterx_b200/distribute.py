"""Multi-GPU decomposition of the hot path: one process per GPU.

Two ways to shard (boxes are the unit of work):

* ``balance_boxes`` -- independent boxes (the benchmark's default, and a
  level's boxes): each rank takes a set of whole boxes, balanced by zone
  count with the longest-processing-time rule; no data-path collective.
* ``SlabHalo`` / ``NcclSlabHalo`` -- one periodic patch cut into z-slabs,
  one per rank (NcclSlabHalo: the same exchange in the engine, over NCCL), with
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

    def _buffers(self, like, nfields):
        """Persistent send and receive buffers for `nfields` fields (ng
        planes each, per neighbour), kept between exchanges."""
        import torch
        n = nfields * self.L.ng * self.plane
        key = (nfields, like.device, like.dtype)
        if getattr(self, "_key", None) != key:
            mk = lambda: torch.empty(n, dtype=like.dtype, device=like.device)
            self._bufs = (mk(), mk(), mk(), mk())  # send up, send down, recv low, recv high
            self._key = key
        return self._bufs

    def exchange(self, tensors: Dict[str, "object"], names: Iterable[str]) -> None:
        names = list(names)
        if self.world == 1:
            for n in names:
                su, sd, rl, rh = self._slices(tensors[n], n)
                rl.copy_(su)
                rh.copy_(sd)
            return
        import torch
        import torch.distributed as dist
        sl = [self._slices(tensors[n], n) for n in names]
        b_up, b_down, b_low, b_high = self._buffers(tensors[names[0]], len(names))
        # the ghost planes of all fields travel as one message per neighbour
        # and direction: pack, 4 point-to-point operations, unpack
        torch.cat([q[0] for q in sl], out=b_up)
        torch.cat([q[1] for q in sl], out=b_down)
        ops = [dist.P2POp(dist.isend, b_up, self.up, self.group),
               dist.P2POp(dist.isend, b_down, self.down, self.group),
               dist.P2POp(dist.irecv, b_low, self.down, self.group),
               dist.P2POp(dist.irecv, b_high, self.up, self.group)]
        for req in dist.batch_isend_irecv(ops):
            req.wait()
        seg = self.L.ng * self.plane
        for q, (_, _, rl, rh) in enumerate(sl):
            rl.copy_(b_low[q * seg:(q + 1) * seg])
            rh.copy_(b_high[q * seg:(q + 1) * seg])


class NcclSlabHalo:
    """The same exchange as SlabHalo behind the engine's C ABI: the packed
    ghost planes travel in one NCCL group per exchange (axb_halo_create /
    axb_halo_exchange; the pack and unpack are kernels of the engine).  One
    engine-side halo per list of grid functions, created on first use; rank
    0 makes the NCCL id and the process group hands it to the others."""

    def __init__(self, eng, layout: Layout, rank: int, world: int, group=None):
        if layout.n[2] < layout.ng:
            raise ValueError("a slab must be at least ng cells thick")
        self.eng, self.L, self.rank, self.world, self.group = eng, layout, rank, world, group
        self._halos = {}

    def _uid(self) -> bytes:
        uid = self.eng.halo_unique_id() if self.rank == 0 else None
        if self.world > 1:
            import torch.distributed as dist
            box = [uid]
            dist.broadcast_object_list(box, src=0, group=self.group)
            uid = box[0]
        return uid

    def exchange(self, tensors: Dict[str, "object"], names: Iterable[str]) -> None:
        key = tuple(names)
        if key not in self._halos:
            self._halos[key] = self.eng.halo_create(self.L, self.world, self.rank, self._uid(),
                                                    list(key))
        self.eng.halo_exchange(self._halos[key], tensors)

    def close(self) -> None:
        for h in self._halos.values():
            self.eng.halo_destroy(h)
        self._halos = {}


def allreduce_max(value: float, group=None, device=None) -> float:
    """The largest `value` over the ranks of `group` (one all-reduce of a
    double; the identity without an initialised process group)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def cfl_dt(max_speed: float, dx: Sequence[float], dtfac: float, cfl: float = 0.9) -> float:
    """Time step of the next substep: dtfac * dx[0] (the driver's fixed
    dtfac), capped so that dt * max_speed * sum(1/dx) <= cfl."""
    cap = cfl / (max(float(max_speed), 1e-300) * sum(1.0 / d for d in dx))
    return min(dtfac * dx[0], cap)


def slab_layout(n_global: Tuple[int, int, int], ng: int, rank: int, world: int
                ) -> Tuple[Layout, int]:
    """This rank's box of a periodic patch on [0, 1]^3 cut into z-slabs, and
    the global index of its first interior cell."""
    k0, nz = slab_ranges(n_global[2], world)[rank]
    dx = tuple(1.0 / v for v in n_global)
    L = Layout((n_global[0], n_global[1], nz), ng, dx, (0.0, 0.0, k0 * dx[2]))
    return L, k0


def prims_to_sync(params) -> List[str]:
    """The cell-centred primitives a substep fills and exchanges, plus zvec
    or svec when the fluxes reconstruct one of them (recon_type)."""
    extra = {1: ["zvec_x", "zvec_y", "zvec_z"], 2: ["svec_x", "svec_y", "svec_z"]}
    return PRIMS + extra.get(int(getattr(params, "recon_type", 0)), [])


def slab_substep(eng, L, f, fn, params, eos, alpha, beta, gamma, dt, halo,
                 cfl: bool = False):
    """One RK substep of a rank's slab (axb_substep's sequence with the
    neighbours' ghost planes): RHS group, stage update, local periodic fill
    and halo exchange of the evolved variables, post-step group, local fill
    and exchange of the primitives.  With `cfl`, returns the maximum
    characteristic speed of this substep's faces over all ranks (one
    all-reduce of a double after the RHS group; the engine's status is
    reset first), the input of the next substep's cfl_dt."""
    if cfl:
        eng.status_reset()
    eng.rhs_group(L, f, params, eos)
    smax = None
    if cfl:
        smax = allreduce_max(eng.status()["max_speed"], halo.group,
                             device=f["rho"].device)
    eng.rk_stage(L, f, fn, f, f, alpha, beta, gamma, dt)
    eng.sync_periodic(L, f, EVOLVED)
    halo.exchange(f, EVOLVED)
    eng.con2prim_group(L, f, params, eos)
    prims = prims_to_sync(params)
    eng.sync_periodic(L, f, prims)
    halo.exchange(f, prims)
    return smax
