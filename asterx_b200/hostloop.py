"""Substeps of a box whose state lives in pinned host memory.

A caller that keeps the grid functions on the host (the reference's CPU
build keeps them there between scheduled groups) copies, every substep, the
fields the substep reads to the device and the fields it writes back.  The
copies dominate such a loop, so `HostStateLoop` pipelines them over two copy
streams: the host-to-device copies of substep s + 1 run while the
device-to-host copies of substep s drain (PCIe carries both directions at
once), each field's copy in waiting only for that field's copy out (the
host array is the state both copies touch); fields that are only read (the
metric) go first.  Every substep still moves every input in and every output
out; only their order and overlap change.
"""
from typing import Callable, Dict, Sequence

from asterx_b200.abi import CONS, SAVED

METRIC = ["gxx", "gxy", "gxz", "gyy", "gyz", "gzz", "alp", "betax", "betay", "betaz",
          "kxx", "kxy", "kxz", "kyy", "kyz", "kzz"]
PRIMS = ["rho", "velx", "vely", "velz", "eps", "press", "temperature", "Ye", "entropy",
         "Bvecx", "Bvecy", "Bvecz"]
EVOLVED = CONS + ["Avec_x", "Avec_y", "Avec_z", "Psi"]
STAG = ["dBx_stag", "dBy_stag", "dBz_stag"]


def substep_io(recon_type: int):
    """(inputs, outputs) of one periodic substep (`axb_substep`): it reads the
    metric, the primitives (and zvec / svec when they are reconstructed), the
    evolved variables, dB_stag and the recovery seeds (saved_*); it writes the
    evolved variables, dB_stag (curl A), the primitives, the seeds and the
    recovery flag."""
    rec = {1: ["zvec_x", "zvec_y", "zvec_z"], 2: ["svec_x", "svec_y", "svec_z"]}
    prims = PRIMS + rec.get(int(recon_type), [])
    inputs = METRIC + prims + EVOLVED + STAG + list(SAVED)
    outputs = EVOLVED + STAG + prims + list(SAVED) + ["con2prim_flag"]
    return inputs, outputs


class HostStateLoop:
    """Pipelined host<->device copies around a substep on the device.

    `dev` and `host` map field names to device tensors and pinned host
    tensors of the same size.  `step(run)` issues one substep: the inputs'
    copies in (each output field after its previous copy out), `run()` on
    the compute stream once they have landed, then the outputs' copies out
    once it has finished.  The next substep's copies in start when this
    substep's kernels have finished (they overwrite what the kernels read);
    its kernels also wait for the copies out of the fields they only write.
    Nothing blocks the host; `finish()` makes the compute stream wait for
    the last copies out."""

    def __init__(self, torch, device, dev: Dict, host: Dict, inputs: Sequence[str],
                 outputs: Sequence[str], compute_stream=None):
        self.torch = torch
        self.dev = dev
        self.host = host
        both = [k for k in inputs if k in outputs]
        # copies in: read-only inputs first (they wait for nothing), then the
        # state in the order it is copied out; copies out: write-only fields
        # first (the next substep's kernels wait for them), then the state
        self.inputs = [k for k in inputs if k not in outputs] + both
        self.write_only = [k for k in outputs if k not in inputs]
        self.outputs = self.write_only + both
        self.compute = compute_stream or torch.cuda.current_stream(device)
        self.s_in = torch.cuda.Stream(device)
        self.s_out = torch.cuda.Stream(device)
        self.ev_out = {k: None for k in self.outputs}
        self.ev_in = torch.cuda.Event()
        self.ev_done = torch.cuda.Event()

    def step(self, run: Callable[[], None]):
        torch = self.torch
        start = torch.cuda.Event()
        start.record(self.compute)
        self.s_in.wait_event(start)
        with torch.cuda.stream(self.s_in):
            for k in self.inputs:
                ev = self.ev_out.get(k)
                if ev is not None:
                    self.s_in.wait_event(ev)
                self.dev[k].copy_(self.host[k], non_blocking=True)
            self.ev_in.record(self.s_in)
        self.compute.wait_event(self.ev_in)
        for k in self.write_only:  # the previous copy out of what run() overwrites
            if self.ev_out[k] is not None:
                self.compute.wait_event(self.ev_out[k])
        with torch.cuda.stream(self.compute):
            run()
        self.ev_done.record(self.compute)
        self.s_out.wait_event(self.ev_done)
        with torch.cuda.stream(self.s_out):
            for k in self.outputs:
                self.host[k].copy_(self.dev[k], non_blocking=True)
                ev = torch.cuda.Event()
                ev.record(self.s_out)
                self.ev_out[k] = ev

    def finish(self):
        for ev in self.ev_out.values():
            if ev is not None:
                self.compute.wait_event(ev)
