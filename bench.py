#!/usr/bin/env python
"""Benchmark: zone-updates/s per RK3 substep of the GRMHD hot path.

Workload (one box per GPU): a periodic 256^3 patch with 3 ghost zones and a
static curved metric (gamma_ij = delta_ij + 0.05 * seeded sine modes, lapse
1 - 0.05 sin, shift amplitude 0.01), primitives from smooth seeded fields plus
three planar jumps, Lorentz factor up to 10, ideal gas Gamma = 4/3, WENO-Z
(or MP5) reconstruction, HLLE fluxes, flux-CT with generalised Lorenz gauge,
Palenzuela recovery (Noble backup), SSP-RK3 stages.  The inputs are seeded
synthetic fields of that shape; there is no dataset.  One "step" is one RK3
substep: RHS group + stage update + periodic ghost fill + post-step group
(curl A, dB, con2prim) + ghost fill of the primitives.

Prints one JSON line (rank 0).  ``--impl reference`` times the reference's
own CPU code for the same path (compiled from its sources through the
stand-in headers in oracle/) on the host cores instead.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

REPO = os.path.dirname(os.path.abspath(__file__))
if REPO not in sys.path:
    sys.path.insert(0, REPO)

METRIC = "Zone-updates/s per RK3 substep"
UNIT = "zone-updates/s"
SSPRK3 = [(0.0, 1.0, 1.0), (0.75, 0.25, 0.25), (1.0 / 3.0, 2.0 / 3.0, 2.0 / 3.0)]
GAMMA = 4.0 / 3.0
CFL_MAX = 0.9
# the tabulated-EOS substep: temperature reconstructed (the tabulated EOS has
# no eps(rho, p) for the fluxes), the recovery with the reference's default
# use_temperature = no (with it, the recovery floors eps at the atmosphere's
# eps, which the synthetic table's T^4 / rho makes ~1e5 at the 1e-13 density
# floor, and nearly every cell fails in both builds), atmosphere temperature
# inside the table
TAB_PARAMS = dict(reconstruct_with_temperature=1, t_atmo=0.011, use_temperature=0)
# the survey's algorithmic figure for one substep: 112 FP64 values per zone
# (RHS reads 34, stage 33, post-step reads 23 and writes 22)
SUBSTEP_BYTES = 112 * 8
EOS_KW = dict(rho=(1e-40, 1e10), eps=(0.0, 1e10))
# regions that run concurrently on two streams in the single-box substep
OVERLAPPED = {"sources", "aux", "flux_x", "flux_y"}
REGIONS = ["sources", "flux_x", "flux_y", "flux_z", "aux", "ct_psi", "rk_stage",
           "sync", "bstag", "c2p", "c2p_cells", "mlp"]
# Algorithmic FP64 values moved per interior zone by each kernel (each field
# read once, written once; ghost re-reads not counted).
ALG_DOUBLES = {
    "sources": 9 + 16 + 7,           # prims + vertex metric & curvature, 7 RHS
    "flux_x": 9 + 1 + 10 + 7 + 2,    # recon fields, dB_stag, metric; acc, B fluxes
    "flux_y": 9 + 1 + 10 + 14 + 2,   # + acc read-modify-write
    # z pass with the stage update fused (axb_substep): acc and the sources'
    # RHS read, U_n and U_k read, U_k written
    "flux_z": 9 + 1 + 10 + 7 + 7 + 14 + 7 + 2,
    "aux": 3 + 1 + 10 + 7,
    # CT + Psi with the fused stage: B fluxes, auxiliaries, lapse and shift,
    # U_n and U_k of A and Psi read, U_k written
    "ct_psi": 6 + 7 + 4 + 8 + 4,
    "rk_stage": 11 * 4,
    "bstag": 3 + 3,
    # ghost fill: the ghost shell of 11 + 12 fields, read and written, per
    # interior zone of a 256^3 box with 3 ghosts (262^3/256^3 - 1 = 7.3%)
    "sync": 2 * 23 * 0.073,
    "c2p": 7 + 3 + 7 + 7 + 12 + 7 + 3 + 6 + 1,
}


def parse_args():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=12)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=256, help="interior cells per axis")
    ap.add_argument("--recon", default="wenoz", choices=["wenoz", "mp5", "ppm"])
    ap.add_argument("--recvar", default="z", choices=["v", "z", "s"],
                    help="velocity variable the fluxes reconstruct (AsterX recon_type): "
                         "v = vel (v_vec), z = W vel (z_vec, default: the 256^3 state's "
                         "Lorentz factors up to 10 push a reconstructed v_vec past the "
                         "speed of light at some faces), s = rho h W^2 vel (s_vec)")
    ap.add_argument("--dtfac", type=float, default=0.25,
                    help="dt = dtfac * dx, capped by the CFL limit of the engine's "
                         "characteristic-speed maximum")
    ap.add_argument("--e2e-steps", type=int, default=6)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=12.0,
                    help="target CPU time of the reference baseline sample")
    ap.add_argument("--workload", default="substep", choices=["substep", "tab", "c2p", "amr"],
                    help="substep: the RK3 substep of one box (the headline); "
                         "tab: the same substep with the synthetic tabulated EOS at "
                         "192^3, MP5 (the tabulated-EOS configuration); "
                         "c2p: the independent-cell recovery microbenchmark, "
                         "plain seeds vs the learned guess; amr: a level of boxes of "
                         "uneven sizes, batched + CUDA graph vs one launch per box")
    ap.add_argument("--boxes", type=int, default=512, help="boxes of the amr workload")
    ap.add_argument("--amr-physics", default="config2", choices=["config2", "mild"],
                    help="amr workload state: config2 = the 256^3 workload's physics "
                         "(W <= 10, b^2/rho <= 10, 3 jumps) on every box; mild = W <= 2, "
                         "b^2/rho <= 0.1, no jumps")
    ap.add_argument("--decomp", default="boxes", choices=["boxes", "slab"],
                    help="with several GPUs: boxes = one independent periodic box per rank "
                         "(no data-path collective); slab = the ranks' boxes are z-slabs of "
                         "one periodic patch, with a ghost-plane exchange (NCCL send/recv) "
                         "after each ghost fill")
    ap.add_argument("--cells", type=int, default=1 << 26,
                    help="cells of the recovery microbenchmark")
    ap.add_argument("--train-pairs", type=int, default=1 << 24)
    ap.add_argument("--train-epochs", type=float, default=4.0)
    ap.add_argument("--mlp-act", default="relu", choices=["relu", "silu"],
                    help="hidden activation of the learned guess's network")
    return ap.parse_args()


def peak_hbm():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    try:
        with open(p) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def traffic_table():
    """Per-launch DRAM bytes from the committed ncu summaries (profiles/)."""
    p = os.path.join(REPO, "profiles", "traffic.json")
    try:
        with open(p) as fh:
            return json.load(fh)
    except Exception:
        return {}


class ClockSampler:
    """nvidia-smi clock / throttle-reason samples during the timed region:
    sampled every 50 ms from before the region (the first sample is awaited,
    so the sampler is running when the region starts), kept when their
    timestamp falls inside [begin(), stop()]."""

    FIELDS = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None
        self.t0 = None

    def start(self):
        try:
            import tempfile
            fd, self.path = tempfile.mkstemp(prefix="axb_clocks_", suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
            deadline = time.time() + 5.0
            while time.time() < deadline and os.path.getsize(self.path) == 0:
                time.sleep(0.02)
        except Exception:
            self.proc = None

    def begin(self):
        self.t0 = time.time()

    @staticmethod
    def _when(stamp):
        import datetime
        try:
            return datetime.datetime.strptime(stamp, "%Y/%m/%d %H:%M:%S.%f").timestamp()
        except Exception:
            return None

    def stop(self):
        t1 = time.time()
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        time.sleep(0.06)  # the sample that covers the region's end
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        with open(self.path) as fh:
            for line in fh:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 10 and parts[2].replace(".", "").isdigit():
                    rows.append(parts)
        os.unlink(self.path)
        inside = [r for r in rows if self.t0 is not None and self._when(r[0]) is not None
                  and self.t0 - 0.05 <= self._when(r[0]) <= t1 + 0.05]
        rows = inside or rows[-1:]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[2]) for r in rows]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[6 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": float(rows[0][3]),
                "reasons": reasons, "samples": len(rows),
                "power_w_max": max((float(r[4]) for r in rows
                                    if r[4].replace(".", "").isdigit()), default=None)}


# ---------------------------------------------------------------------------
# reference CPU code (the checker build of the reference sources)
# ---------------------------------------------------------------------------
class _StdoutToStderr:
    """Send file descriptor 1 to stderr while the reference code runs: its
    Palenzuela scheme prints from inside the solver when a bracket fails,
    and the benchmark's stdout must carry exactly one JSON line."""

    def __enter__(self):
        import ctypes
        sys.stdout.flush()
        self._libc = ctypes.CDLL(None)
        self._libc.fflush(None)
        self._saved = os.dup(1)
        os.dup2(2, 1)
        return self

    def __exit__(self, *exc):
        self._libc.fflush(None)
        sys.stdout.flush()
        os.dup2(self._saved, 1)
        os.close(self._saved)
        return False


def reference_substep_rate(seconds, recon, seed=2, start_n=24, recvar="z", tab=False):
    with _StdoutToStderr():
        return _reference_substep_rate(seconds, recon, seed, start_n, recvar, tab)


def _reference_substep_rate(seconds, recon, seed=2, start_n=24, recvar="z", tab=False):
    """Time the reference's scheduled routines (AsterX_Fluxes,
    AsterX_SourceTerms, AsterX_RHS, the stage update, AsterX_ComputedBstagFromA,
    AsterX_ComputedBFromdBstag, AsterX_Con2Prim) on one box of the workload,
    with the box edge chosen so that the sample takes about `seconds`.
    Returns (zone-updates/s, sample description, threads)."""
    import numpy as np
    from asterx_b200 import abi
    from asterx_b200 import workloads as W
    from oracle.oracle import reference
    ref = reference()
    if ref is None:
        raise RuntimeError("oracle/_ref/libaxref.so is not built")
    threads = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))

    table = W.synthetic_table() if tab else None

    def one(n, nsub):
        if tab:
            L, f = W.tabulated_box(n=n, ng=3, seed=seed + 3)
        else:
            L, f = W.curved_box(n=n, ng=3, seed=seed, wmax=10.0)
        W.cons_from_prims(L, f)
        W.saved_from_prims(f)
        for name in abi.GF_NAMES:
            f.setdefault(name, L.zeros())
        p = abi.default_params(reconstruction_method=recon, flux_type="hlle",
                               c2p_prime="palenzuela", c2p_second="noble",
                               recon_type={"v": 0, "z": 1, "s": 2}[recvar],
                               **(TAB_PARAMS if tab else {}))
        host = {k: v.copy() for k, v in f.items()}
        ref.setup(L, p, host)
        if tab:
            ref.eos_tabulated(*table)
        else:
            ref.eos_idealgas(GAMMA, **EOS_KW)
        dt = 0.25 * L.dx[0]
        evolved = abi.CONS + ["Avec_x", "Avec_y", "Avec_z", "Psi"]
        rhs = abi.HYDRO_RHS + abi.AVEC_RHS
        un = {k: host[k].copy() for k in evolved}
        t0 = time.perf_counter()
        for s in range(nsub):
            a_, b_, g_ = SSPRK3[s % 3]
            ref.run("fluxes")
            ref.run("sources")
            ref.run("rhs")
            for u, r in zip(evolved, rhs):
                host[u][:] = a_ * un[u] + b_ * host[u] + (g_ * dt) * host[r]
            ref.run("bstag")
            ref.run("dB")
            ref.run("c2p")
        return time.perf_counter() - t0, L

    n = start_n
    t, L = one(n, 1)
    rate = n ** 3 / t
    # box edge for ~seconds/3 per substep, then three substeps
    n = int(max(16, min(160, round((rate * seconds / 3.0) ** (1 / 3)))))
    t, L = one(n, 3)
    rate = 3 * n ** 3 / t
    return rate, f"{n}^3 box, 3 SSP-RK3 substeps, {t:.1f} s", threads, t


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    res_rate = []
    sample = None
    threads = None
    for _ in range(args.warmup):
        reference_substep_rate(2.0, args.recon, recvar=args.recvar)
    for _ in range(args.steps):
        rate, sample, threads, _t = reference_substep_rate(6.0, args.recon, recvar=args.recvar)
        res_rate.append(rate)
    value = statistics.median(res_rate)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"{args.n}^3 curved-metric patch (bounded CPU sample), "
                               f"{args.recon}+HLLE on {args.recvar}_vec, Palenzuela c2p, "
                               "flux-CT",
                   "parallelism": "OpenMP host threads"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads,
                         "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# the engine
# ---------------------------------------------------------------------------
def _mean_iters(hist):
    """Mean first-solver iteration count of a status histogram."""
    tot = sum(int(v) for v in hist)
    return sum(i * int(v) for i, v in enumerate(hist)) / tot if tot else None


def ours(args):
    import torch
    import torch.distributed as dist
    from datetime import timedelta

    from asterx_b200 import abi
    from asterx_b200 import workloads as W
    from asterx_b200.engine import Engine
    from asterx_b200.hostloop import HostStateLoop, substep_io

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        dist.init_process_group("nccl", timeout=timedelta(seconds=300),
                                device_id=dev)
    eng = Engine(local)
    xp = W._XP(torch, dev)
    tab = args.workload == "tab"
    if tab:
        L, f = W.tabulated_box(n=args.n, ng=3, seed=5 + rank, xp=xp)
    else:
        L, f = W.curved_box(n=args.n, ng=3, seed=2 + rank, wmax=10.0, xp=xp)
    W.cons_from_prims(L, f, xp=xp)
    W.saved_from_prims(f, xp=xp)
    # keep only the reconstructed velocity variable the fluxes use (the
    # recovery writes zvec / svec back only when they are given)
    for ax in "xyz":
        if args.recvar != "z":
            f.pop("zvec_" + ax, None)
        if args.recvar != "s":
            f.pop("svec_" + ax, None)
    skip = {"zvec_x", "zvec_y", "zvec_z", "svec_x", "svec_y", "svec_z", "dBx",
            "dBy", "dBz"}
    for name in abi.GF_NAMES:
        if name not in f and name not in skip:
            f[name] = torch.zeros(L.size, dtype=torch.float64, device=dev)
    evolved = abi.CONS + ["Avec_x", "Avec_y", "Avec_z", "Psi"]
    fn = {k: f[k].clone() for k in evolved}
    params = abi.default_params(reconstruction_method=args.recon, flux_type="hlle",
                                c2p_prime="palenzuela", c2p_second="noble",
                                recon_type={"v": 0, "z": 1, "s": 2}[args.recvar],
                                **(TAB_PARAMS if tab else {}))
    eos = eng.eos_tabulated(*W.synthetic_table()) if tab else eng.eos_idealgas(GAMMA, **EOS_KW)
    zones = args.n ** 3
    stream = torch.cuda.current_stream(dev)

    # time step: dtfac * dx, capped by the CFL limit of the characteristic
    # speeds of the initial state (the engine's max |lambda| over all faces
    # of one RHS evaluation): dt * smax * (1/dx + 1/dy + 1/dz) <= CFL_MAX
    eng.status_reset()
    eng.rhs_group(L, f, params, eos)
    smax0 = eng.status()["max_speed"]
    if world > 1:
        t = torch.tensor([smax0], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        smax0 = float(t.item())
    from asterx_b200.distribute import cfl_dt
    dt = cfl_dt(smax0, L.dx, args.dtfac, CFL_MAX)

    halo = None
    if world > 1 and args.decomp == "slab":
        from asterx_b200.distribute import SlabHalo
        halo = SlabHalo(L, rank, world)

    def substep(s):
        a_, b_, g_ = SSPRK3[s % 3]
        if s % 3 == 0:
            for k in evolved:
                fn[k].copy_(f[k])
        if halo is None:
            eng.substep(L, f, fn, params, eos, a_, b_, g_, dt, periodic=True)
        else:
            from asterx_b200.distribute import slab_substep
            slab_substep(eng, L, f, fn, params, eos, a_, b_, g_, dt, halo)

    # the FP64 peaks that bound the instruction-bound kernels
    fp64 = eng.probe_fp64()

    # warm-up, with the recovery failures and error word of every substep
    warm_fail = []
    warm_ew = 0
    for s in range(args.warmup):
        eng.status_reset()
        substep(s)
        st = eng.status()
        warm_fail.append(st["c2p_fail"])
        warm_ew |= st["error_word"]
    torch.cuda.synchronize()
    eng.status_reset()
    sampler = ClockSampler(local)
    sampler.start()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    eng.timing_begin()
    sampler.begin()
    e0.record(stream)
    for s in range(args.steps):
        substep(s)
    e1.record(stream)
    torch.cuda.synchronize()
    region_ms, region_n = eng.timing_end(len(REGIONS))
    if world > 1:
        dist.barrier()
    clocks = sampler.stop()
    ms = e0.elapsed_time(e1)
    st = eng.status()
    if world > 1:
        t = torch.tensor([ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    value = world * zones * args.steps / (ms / 1e3)
    launches = int(sum(region_n))
    healthy = (st["error_word"] & (abi.EW_NAN_FLUX | abi.EW_NAN_RHS)) == 0
    if not healthy:
        print(f"bench: the timed substeps raised error word {st['error_word']:#x} "
              "(non-finite face fluxes or RHS)", file=sys.stderr)

    # dominant kernel and its roofline: the kernel with the largest time of
    # its own; the sources and the vertex auxiliaries run on a second stream
    # beside the x and y flux passes, so those four regions' event times
    # include each other's and are no kernel's own time
    shares = {REGIONS[i]: region_ms[i] for i in range(len(REGIONS))
              if region_n[i] and REGIONS[i] in ALG_DOUBLES
              and REGIONS[i] not in OVERLAPPED}
    dom = max(shares, key=shares.get)
    idom = REGIONS.index(dom)
    avg_launch_s = region_ms[idom] / region_n[idom] / 1e3
    alg_bytes = ALG_DOUBLES[dom] * 8 * zones
    achieved = alg_bytes / avg_launch_s / 1e9
    peak, peak_kind = peak_hbm()
    traffic = traffic_table().get(f"{dom}:{args.recon}:{args.n}")
    substep_gbs = SUBSTEP_BYTES * zones / (ms / args.steps / 1e3) / 1e9

    # end to end through the C ABI from pinned host memory: every step copies
    # the fields the substep reads in and the fields it writes back out; the
    # copies of consecutive steps overlap (HostStateLoop: one field's copy in
    # waits for its copy out, the metric goes first)
    inputs, outputs = substep_io(params.recon_type)
    host = {k: torch.empty(L.size, dtype=torch.float64, pin_memory=True) for k in
            set(inputs) | set(outputs)}
    for k in host:
        host[k].copy_(f[k])
    torch.cuda.synchronize()
    h2d = 8 * L.size * len(inputs)
    d2h = 8 * L.size * len(outputs)
    ne = max(1, min(args.e2e_steps, args.steps))
    loop = HostStateLoop(torch, dev, f, host, inputs, outputs, compute_stream=stream)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e2 = torch.cuda.Event(enable_timing=True)
    e3 = torch.cuda.Event(enable_timing=True)
    e2.record(stream)
    for s in range(ne):
        loop.step(lambda s=s: substep(s))
    loop.finish()
    e3.record(stream)
    torch.cuda.synchronize()
    ms_e2e = e2.elapsed_time(e3)
    if world > 1:
        t = torch.tensor([ms_e2e], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_e2e = float(t.item())
    e2e_value = world * zones * ne / (ms_e2e / 1e3)

    cpu = None
    parity = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            rate, sample, threads, _t = reference_substep_rate(args.cpu_seconds, args.recon,
                                                               recvar=args.recvar, tab=tab)
            cpu = {"value": rate, "unit": UNIT, "cores": threads, "kind": "reference",
                   "sample": sample}
            parity = reference_parity(eng, L, f, params, eos, dt, tab=tab)
        except Exception as exc:  # the checker library may be absent
            cpu = {"value": None, "unit": UNIT, "cores": None, "kind": "reference",
                   "sample": f"unavailable: {exc}"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic (seeded fields of the configuration)",
            "config": {"workload": f"{args.n}^3 periodic patch, 3 ghosts, curved static "
                                   f"metric, W <= 10, b^2/rho <= 10, 3 planar jumps, "
                                   f"{args.recon}+HLLE on {args.recvar}_vec, flux-CT, "
                                   f"Palenzuela c2p (Noble backup), " +
                                   ("synthetic tabulated EOS 200x100x60 (P = rho T (1+Ye) "
                                    "+ T^4/3 + 100 rho^2), Ye in [0.05, 0.5], temperature "
                                    "reconstructed" if tab else "ideal gas Gamma=4/3") +
                                   ", SSP-RK3 substeps",
                       "eos": "tabulated3d" if tab else "idealgas",
                       "box": [args.n] * 3, "ghosts": 3, "recon": args.recon,
                       "recon_type": f"{args.recvar}_vec", "dt_over_dx": dt / L.dx[0],
                       "cfl": dt * smax0 * sum(1.0 / d for d in L.dx),
                       "parallelism": (f"one box per GPU x{world}" if halo is None else
                                       f"z-slabs of one patch, halo exchange x{world}"),
                       "l2": "inputs larger than L2 (146 MB per field)"},
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved,
                         "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "alg_bytes_per_launch": alg_bytes,
                         "avg_launch_ms": avg_launch_s * 1e3,
                         "substep": {"alg_bytes_per_zone": SUBSTEP_BYTES,
                                     "achieved": substep_gbs, "frac": substep_gbs / peak}},
            "kernels_ms_per_step": {REGIONS[i]: region_ms[i] / args.steps
                                    for i in range(len(REGIONS)) if region_n[i]},
            "kernels_note": "sources and aux run on a second stream beside flux_x and "
                            "flux_y, so their region times overlap those passes' (the "
                            "per-kernel shares are in the committed ncu launch list)",
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "steps": ne,
                    "copies": f"{len(inputs)} fields in, {len(outputs)} out per step from/to "
                              "pinned host arrays; a step's copies in overlap the previous "
                              "step's copies out"},
            "cpu_baseline": cpu,
            "parity": parity,
            "gpu_launches": launches,
            "clocks": clocks,
            "health": {"nan_free": healthy, "error_word": st["error_word"],
                       "c2p_fail_cells_timed": st["c2p_fail"],
                       "c2p_fail_per_substep_timed": st["c2p_fail"] / args.steps,
                       "c2p_fail_per_substep_warmup": warm_fail,
                       "warmup_error_word": warm_ew},
            "max_char_speed": st["max_speed"],
            "c2p_mean_iters": _mean_iters(st["iter_hist"]),
            "c2p_iter_hist": {int(i): int(v) for i, v in enumerate(st["iter_hist"]) if v},
            "fp64_probe": fp64,
        }
        print(json.dumps(line), flush=True)
    eng.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def reference_parity(eng, L, f, params, eos, dt, m=40, off=8, ng_ref=5, tab=False):
    """The checker half of the CPU-baseline leg: one substep (RHS group,
    stage U + dt RHS, post-step group; no ghost fill in between) of a
    m^3 sub-box cut from the timed state, on the engine (3 ghost zones) and
    on the reference build (ng_ref ghost zones, the same cells), with the
    maximum and L2 relative errors of the RHS and of the recovered
    primitives and conserved variables."""
    import numpy as np
    import torch

    from asterx_b200 import abi
    from asterx_b200 import workloads as W
    from asterx_b200.abi import Layout
    from oracle.oracle import reference
    ref = reference()
    if ref is None:
        return None
    o = L.ng + off
    lo = o - ng_ref
    L5 = Layout((m, m, m), ng_ref, L.dx,
                tuple(L.xmin[d] + (o - L.ng) * L.dx[d] for d in range(3)))
    L3 = Layout((m, m, m), 3, L5.dx, L5.xmin)
    npt = L5.npts[0]
    sub5 = {}
    for k, t in f.items():
        v = t.view(L.npts[2], L.npts[1], L.sy)[lo:lo + npt, lo:lo + npt, lo:lo + npt]
        a = L5.zeros()
        L5.view(a)[:, :, :npt] = v.cpu().numpy()
        sub5[k] = a
    d = ng_ref - 3
    n3 = L3.npts[0]

    def crop(a):
        out = L3.zeros()
        L3.view(out)[:, :, :n3] = L5.view(a)[d:d + n3, d:d + n3, d:d + n3]
        return out

    evolved = abi.CONS + ["Avec_x", "Avec_y", "Avec_z", "Psi"]
    rhs = abi.HYDRO_RHS + abi.AVEC_RHS
    cent = {"Avec_x": (1, 0, 0), "Avec_y": (0, 1, 0), "Avec_z": (0, 0, 1), "Psi": (0, 0, 0),
            "Avec_x_rhs": (1, 0, 0), "Avec_y_rhs": (0, 1, 0), "Avec_z_rhs": (0, 0, 1),
            "Psi_rhs": (0, 0, 0)}
    # engine
    dev = {k: torch.from_numpy(crop(a)).to(f["rho"].device) for k, a in sub5.items()}
    eng.rhs_group(L3, dev, params, eos)
    got_rhs = {k: dev[k].cpu().numpy() for k in rhs}
    eng.rk_stage(L3, dev, dev, dev, dev, 0.0, 1.0, 1.0, dt)
    eng.con2prim_group(L3, dev, params, eos)
    got = {k: dev[k].cpu().numpy() for k in dev}
    # reference build
    host = {k: a.copy() for k, a in sub5.items()}
    for name in abi.GF_NAMES:
        host.setdefault(name, L5.zeros())
    with _StdoutToStderr():
        ref.setup(L5, params, host)
        if tab:
            ref.eos_tabulated(*W.synthetic_table())
        else:
            ref.eos_idealgas(GAMMA, **EOS_KW)
        ref.rhs_group()
        want_rhs = {k: host[k].copy() for k in rhs}
        for u, r in zip(evolved, rhs):
            sl = L5.interior(cent.get(u, (1, 1, 1)))
            L5.view(host[u])[sl] = L5.view(host[u])[sl] + dt * L5.view(host[r])[sl]
        ref.con2prim_group()

    def errs(names, g, w):
        emax = el2 = ept = 0.0
        for k in names:
            c = cent.get(k, (1, 1, 1))
            gg = L3.view(g[k])[L3.interior(c)]
            ww = L3.view(crop(w[k]))[L3.interior(c)]
            scale = float(np.abs(ww).max()) or 1.0
            diff = np.abs(gg - ww)
            emax = max(emax, float(diff.max()) / scale)
            el2 = max(el2, float(np.linalg.norm(gg - ww) / (np.linalg.norm(ww) or 1.0)))
            ept = max(ept, float((diff / np.maximum(np.abs(ww), 1e-6 * scale)).max()))
        return {"max_rel": emax, "l2_rel": el2, "max_point_rel_floor_1e-6": ept}

    prims = ["rho", "eps", "press", "velx", "vely", "velz", "Bvecx", "Bvecy", "Bvecz"]
    fl_g = L3.view(got["con2prim_flag"])[L3.interior()]
    fl_w = L3.view(crop(host["con2prim_flag"]))[L3.interior()]
    diff = fl_g != fl_w
    ps = [abi.C2P_PRIME, abi.C2P_SECOND]
    # cells whose Palenzuela bracket ends within a few ulps of the iteration
    # cap may be recovered by the first scheme in one build and the second in
    # the other (both within the tolerance): counted apart from other
    # mismatches, and their primitives compared like every other cell's
    swaps = diff & np.isin(fl_g, ps) & np.isin(fl_w, ps)
    return {"sub_box": f"{m}^3 cells of the timed state (offset {off} from the interior "
                       f"corner), engine with 3 ghosts, reference build with {ng_ref}",
            "substep": "RHS group, U + dt RHS, post-step group",
            "rhs": errs(rhs, got_rhs, want_rhs),
            "prims_cons": errs(prims + abi.CONS, got, host),
            "flag_prime_second_swaps": int(swaps.sum()),
            "flag_other_mismatches": int((diff & ~swaps).sum()), "cells": int(diff.size),
            "c2p_fail_cells_reference": int((fl_w == abi.C2P_FAIL).sum())}


def c2p_bench(args):
    """Recovery microbenchmark: 2^26 independent cells (rho log-U[1e-12, 1e-2],
    eps log-U[1e-6, 10], W U[1, 50], b^2/rho log-U[1e-4, 100], isotropic
    directions, random metric), conserved variables from the exact FP64
    prim->cons map; Noble with Palenzuela backup at c2p_tol 1e-10.  The MLP
    guess is trained first on separately seeded pairs (not timed).  Reports
    cells/s of both, the Noble iteration histogram, the fallback rate and
    the maximum relative error of the recovered primitives against the truth."""
    import numpy as np
    import torch

    from asterx_b200 import abi
    from asterx_b200 import workloads as W
    from asterx_b200.engine import Engine

    if int(os.environ.get("RANK", "0")) != 0:
        return 0
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    eng = Engine(0)
    gamma = 5.0 / 3.0
    eos = eng.eos_idealgas(gamma, rho=(1e-40, 1e10), eps=(0.0, 1e10))
    # floors and ceilings set so that they do not alter the truth: W up to 50,
    # eps down to 1e-6 (temperature floor t_atmo below it), rho down to 1e-12
    params = abi.default_params(c2p_prime="noble", c2p_second="palenzuela", c2p_tol=1e-10,
                                max_iter=100, vw_lim=60.0, B_lim=1e8, rho_abs_min=1e-20,
                                t_atmo=1e-12)
    # training (separately seeded pairs)
    t_train = time.time()
    nt = args.train_pairs
    tr = W.c2p_cells(nt, seed=1001, gamma=gamma, device=dev)
    feats = torch.empty((nt, 8), dtype=torch.float32, device=dev)
    eng.mlp_features(eng.cells(nt, {k: tr[k] for k in abi.CELL_INPUTS}), 8, feats)
    tgt = torch.stack([tr["t_u"], tr["t_lnw"]], dim=1).float().contiguous()
    del tr
    mlp = eng.mlp_create(8, seed=7, bracket=0.02, act=args.mlp_act)
    loss = torch.zeros(1, dtype=torch.float32, device=dev)
    bs = 65536
    nsteps = max(1, int(args.train_epochs * nt / bs))
    gen = torch.Generator(device=dev)
    gen.manual_seed(3)
    for step in range(nsteps):
        idx = torch.randint(0, nt, (bs,), generator=gen, device=dev)
        lr = 3e-3 if step < 0.7 * nsteps else 5e-4
        eng.mlp_train_step(mlp, feats[idx], tgt[idx], lr=lr, loss=loss)
    torch.cuda.synchronize()
    train_s = time.time() - t_train
    train_loss = loss.item()
    del feats, tgt

    n = args.cells
    cells = W.c2p_cells(n, seed=2002, gamma=gamma, device=dev)
    truth = {k: cells[k] for k in ("rho", "eps", "press", "W")}
    t = {k: cells[k] for k in abi.CELL_INPUTS}
    outs = ["rho", "eps", "press", "w_lorentz", "iters", "flag", "fallback"]
    for k in outs:
        t[k] = torch.empty(n, dtype=torch.float64, device=dev)
    guess = torch.empty(2 * n, dtype=torch.float32, device=dev)
    cstruct = eng.cells(n, t)
    cstruct.guess = guess.data_ptr()
    stream = torch.cuda.current_stream(dev)
    res = {}
    for name, m in (("plain", None), ("learned", mlp)):
        for _ in range(args.warmup):
            eng.c2p_cells(cstruct, params, eos, mlp=m)
        torch.cuda.synchronize()
        eng.status_reset()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        eng.timing_begin()
        e0.record(stream)
        for _ in range(args.steps):
            eng.c2p_cells(cstruct, params, eos, mlp=m)
        e1.record(stream)
        torch.cuda.synchronize()
        region_ms, region_n = eng.timing_end(len(REGIONS))
        ms = e0.elapsed_time(e1) / args.steps
        st = eng.status()
        flag = t["flag"]
        ok = flag == abi.C2P_PRIME
        errs = {}
        for k, tk in (("rho", "rho"), ("eps", "eps"), ("press", "press"), ("w_lorentz", "W")):
            e = ((t[k] - truth[tk]).abs() / truth[tk].abs())[ok]
            errs[k] = float(e.max().item()) if e.numel() else None
        # cells that converged to a state away from the truth (a wrong root)
        bad = (((t["rho"] - truth["rho"]).abs() / truth["rho"]) > 1e-6) & ok
        errs["cells_rho_off_by_1e-6"] = int(bad.sum().item())
        hist = st["iter_hist"] / max(1, args.steps)
        it = np.arange(64)
        res[name] = {
            "cells_per_s": n / (ms / 1e3), "ms": ms,
            "mean_iters": float((hist * it).sum() / max(1, hist.sum())),
            "iter_hist": {int(i): int(v) for i, v in enumerate(hist) if v},
            # cells whose guessed first attempt failed and went to the plain
            # cold-start cascade (0 without a guess), and cells not recovered
            # by the first scheme
            "fallback_rate": float(t["fallback"].mean().item()),
            "second_scheme_or_worse_rate": float((~ok).double().mean().item()),
            "fail_rate": float((flag == abi.C2P_FAIL).double().mean().item()),
            "max_rel_err": errs,
            "recovery_kernel_ms": region_ms[REGIONS.index("c2p_cells")] / max(1, args.steps),
            "mlp_kernel_ms": region_ms[REGIONS.index("mlp")] / max(1, args.steps),
            "gpu_launches": int(sum(region_n)),
        }
    alg = 8 * (16 + 8)  # bytes per cell: 16 inputs read, 8 outputs written
    peak, peak_kind = peak_hbm()
    lr_ = res["learned"]
    rk = lr_["recovery_kernel_ms"]
    line = {
        "metric": "c2p cells/s (learned guess)", "value": lr_["cells_per_s"],
        "unit": "cells/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": lr_["ms"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64 (MLP bf16/f32)",
        "data": "synthetic (seeded cells of the configuration)",
        "config": {"workload": f"{n} independent cells, Noble (Palenzuela backup), "
                               "ideal gas Gamma=5/3, c2p_tol 1e-10, MLP 8-64-64-64-2 "
                               f"({args.mlp_act}) trained on {nt} pairs",
                   "cells": n, "l2": "inputs larger than L2"},
        "plain": res["plain"], "learned": res["learned"],
        "speedup_learned_vs_plain": lr_["cells_per_s"] / res["plain"]["cells_per_s"],
        "training": {"pairs": nt, "steps": nsteps, "batch": bs, "final_loss": train_loss,
                     "seconds": train_s},
        "roofline": {"bound": "hbm", "kernel": "c2p_cells",
                     "achieved": alg * n / (rk / 1e3) / 1e9, "peak": peak,
                     "peak_kind": peak_kind, "unit": "GB/s",
                     "frac": alg * n / (rk / 1e3) / 1e9 / peak, "traffic": None},
        "gpu_launches": lr_["gpu_launches"],
    }
    print(json.dumps(line), flush=True)
    eng.close()
    return 0


def amr_bench(args):
    """Batched AMR level: `boxes` boxes (512) with interior edges drawn
    log-uniformly from 16 to 64 per axis, 3 ghosts, the curved-metric physics
    of the 256^3 workload (WENO-Z + HLLE, Palenzuela with Noble backup,
    Gamma 4/3) in a milder state that a 16-cell box still resolves (Lorentz
    factor up to 2, magnetisation up to 0.1, no density jumps; the 256^3
    workload's W <= 10, sigma <= 10 and jumps run away on boxes this small),
    each box periodic on itself.  Times SSP-RK3 substeps done
    (a) as one axb_substep per box (each phase launched once per box, as the
    reference's driver does) and (b) as axb_batch_substep (one persistent
    launch per phase over all boxes, tuned by the autotuner) replayed from a
    CUDA graph holding one full RK3 step.  U_n of the evolved variables lives
    in one arena, so its copy at the start of each RK3 step is one copy."""
    import math

    import numpy as np
    import torch

    from asterx_b200 import abi
    from asterx_b200 import workloads as W
    from asterx_b200.engine import Engine

    if int(os.environ.get("RANK", "0")) != 0:
        return 0
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    eng = Engine(0)
    xp = W._XP(torch, dev)
    rng = np.random.default_rng(33)
    shapes = [tuple(int(round(math.exp(rng.uniform(math.log(16), math.log(64)))))
                    for _ in range(3)) for _ in range(args.boxes)]
    evolved = abi.CONS + ["Avec_x", "Avec_y", "Avec_z", "Psi"]
    skip = {"zvec_x", "zvec_y", "zvec_z", "svec_x", "svec_y", "svec_z", "dBx", "dBy", "dBz"}
    layouts, fields = [], []
    for b, n in enumerate(shapes):
        if args.amr_physics == "config2":
            L, f = W.curved_box(n=n, ng=3, seed=1000 + b, wmax=10.0, xp=xp)
        else:
            L, f = W.curved_box(n=n, ng=3, seed=1000 + b, wmax=2.0, njumps=0,
                                sigma=(1e-3, 0.1), xp=xp)
        W.cons_from_prims(L, f, xp=xp)
        W.saved_from_prims(f, xp=xp)
        for ax in "xyz":
            if args.recvar != "z":
                f.pop("zvec_" + ax, None)
            if args.recvar != "s":
                f.pop("svec_" + ax, None)
        for name in abi.GF_NAMES:
            if name not in f and name not in skip:
                f[name] = torch.zeros(L.size, dtype=torch.float64, device=dev)
        layouts.append(L)
        fields.append(f)
    # evolved variables and their U_n copies as views of two arenas
    sizes = [L.size for L in layouts]
    total = sum(sizes) * len(evolved)
    arena = torch.empty(total, dtype=torch.float64, device=dev)
    arena_n = torch.empty(total, dtype=torch.float64, device=dev)
    fields_n = []
    off = 0
    for L, f in zip(layouts, fields):
        fn = {}
        for k in evolved:
            v = arena[off:off + L.size]
            v.copy_(f[k])
            f[k] = v
            fn[k] = arena_n[off:off + L.size]
            off += L.size
        fields_n.append(fn)
    zones = sum(n[0] * n[1] * n[2] for n in shapes)
    params = abi.default_params(reconstruction_method=args.recon, flux_type="hlle",
                                c2p_prime="palenzuela", c2p_second="noble",
                                recon_type={"v": 0, "z": 1, "s": 2}[args.recvar])
    eos = eng.eos_idealgas(GAMMA, **EOS_KW)
    # one time step for the level: dtfac times the finest spacing, capped by
    # the CFL limit of the largest characteristic speed over all boxes
    from asterx_b200.distribute import cfl_dt
    eng.status_reset()
    smax = 0.0
    dxmin = min(min(L.dx) for L in layouts)
    for L, f in zip(layouts, fields):
        eng.rhs_group(L, f, params, eos)
    smax = eng.status()["max_speed"]
    dt = cfl_dt(smax, (dxmin,) * 3, args.dtfac, CFL_MAX)
    stream = torch.cuda.current_stream(dev)
    # keep a pristine copy so both modes start from the same state
    pristine = arena.clone()

    def per_box_step():
        arena_n.copy_(arena)
        for a_, b_, g_ in SSPRK3:
            for L, f, fn in zip(layouts, fields, fields_n):
                eng.substep(L, f, fn, params, eos, a_, b_, g_, dt, periodic=True)

    batch = eng.batch_create(layouts, fields, fields_n, params, eos)

    def batched_step():
        arena_n.copy_(arena)
        for a_, b_, g_ in SSPRK3:
            eng.batch_substep(batch, a_, b_, g_, dt, periodic=True)

    def timed(fn, nsteps):
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(nsteps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    nrk = max(1, args.steps // 3)  # timed RK3 steps (3 substeps each)
    # (a) one launch per box and phase
    for _ in range(max(1, args.warmup // 3)):
        per_box_step()
    t0 = time.perf_counter()
    ms_a = timed(per_box_step, nrk)
    wall_a = time.perf_counter() - t0
    # (b) batched, tuned, replayed from a CUDA graph
    arena.copy_(pristine)
    tuning = eng.batch_autotune(batch)
    for _ in range(max(1, args.warmup // 3)):
        batched_step()
    ms_b_nograph = timed(batched_step, nrk)
    graph = torch.cuda.CUDAGraph()
    torch.cuda.synchronize()
    with torch.cuda.graph(graph):
        batched_step()
    graph.replay()
    torch.cuda.synchronize()
    eng.status_reset()
    sampler = ClockSampler(0)
    sampler.start()
    sampler.begin()
    ms_b = timed(graph.replay, nrk)
    clocks = sampler.stop()
    st = eng.status()
    # one substep traced per kernel region (outside the graph)
    eng.timing_begin()
    eng.batch_substep(batch, *SSPRK3[1], dt, periodic=True)
    region_ms, region_n = eng.timing_end(len(REGIONS))
    sub = 3 * nrk
    v_b = zones * sub / (ms_b / 1e3)
    v_a = zones * sub / (ms_a / 1e3)
    line = {
        "metric": "Zone-updates/s per RK3 substep (batched AMR level)", "value": v_b,
        "unit": UNIT, "n_gpus": 1, "steps": sub, "warmup": args.warmup,
        "ms_per_step": ms_b / sub, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded boxes of the level)",
        "config": {"workload": f"{args.boxes} boxes, edges log-uniform in [16, 64] per axis, "
                               f"3 ghosts, curved metric, " +
                               ("W <= 10, sigma <= 10, 3 jumps, " if args.amr_physics ==
                                "config2" else "W <= 2, sigma <= 0.1, no jumps, ") +
                               f"{args.recon}+HLLE on {args.recvar}_vec, Palenzuela c2p, "
                               "Gamma=4/3, SSP-RK3; batched persistent launches in a CUDA "
                               "graph vs one launch per box",
                   "boxes": args.boxes, "zones": zones, "recon": args.recon,
                   "dt": dt, "max_char_speed_initial": smax,
                   "l2": "level data far larger than L2"},
        "per_box_launch": {"value": v_a, "ms_per_step": ms_a / sub,
                           "host_wall_s": wall_a, "launches_per_substep": 11 * args.boxes},
        "batched_no_graph": {"value": zones * sub / (ms_b_nograph / 1e3),
                             "ms_per_step": ms_b_nograph / sub},
        "speedup_batched_graph_vs_per_box": v_b / v_a,
        "autotune": tuning,
        "kernels_ms_per_substep": {REGIONS[i]: region_ms[i] for i in range(len(REGIONS))
                                   if region_n[i]},
        "gpu_launches": int(sum(region_n)) * sub,
        "clocks": clocks,
        "error_word": st["error_word"], "c2p_fail_cells": st["c2p_fail"],
    }
    print(json.dumps(line), flush=True)
    del graph
    eng.close()
    return 0


def main():
    args = parse_args()
    if args.impl == "reference":
        return reference_arm(args)
    if args.workload == "c2p":
        return c2p_bench(args)
    if args.workload == "amr":
        return amr_bench(args)
    if args.workload == "tab" and "--n" not in sys.argv:
        args.n = 192
    if args.workload == "tab" and "--recon" not in sys.argv:
        args.recon = "mp5"
    return ours(args)


if __name__ == "__main__":
    sys.exit(main())
