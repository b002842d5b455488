"""The ordering of HostStateLoop's copies and kernels, on the CPU: a stand-in
for torch's streams and events queues every copy, record, wait and kernel
per stream, and a scheduler runs the queues in random interleavings that
respect only the event waits (as a GPU may).  Every interleaving must leave
the host state that running the substeps one after another gives; a copy in
that overtook its field's copy out, or a kernel that overtook a copy, would
show as a different state."""
import random

from asterx_b200.hostloop import HostStateLoop


class _Event:
    def __init__(self):
        self.op = None  # the record operation it stands for

    def record(self, stream):
        op = {"kind": "record", "done": False}
        stream.ops.append(op)
        self.op = op


class _Stream:
    def __init__(self, *a, **k):
        self.ops = []

    def wait_event(self, ev):
        self.ops.append({"kind": "wait", "on": ev.op, "done": False})


class _Tensor:
    def __init__(self, owner, name):
        self.owner, self.name = owner, name

    def copy_(self, src, non_blocking=False):
        self.owner.current.ops.append({"kind": "copy", "dst": self, "src": src,
                                       "done": False})


class _FakeTorch:
    """torch.cuda as HostStateLoop uses it."""

    def __init__(self):
        self.default = _Stream()
        self.current = self.default
        fake = self

        class cuda:  # noqa: N801 - mirrors torch.cuda
            Stream = _Stream
            Event = _Event

            @staticmethod
            def current_stream(device=None):
                return fake.default

            class stream:  # noqa: N801
                def __init__(self, s):
                    self.s = s

                def __enter__(self):
                    self.prev = fake.current
                    fake.current = self.s

                def __exit__(self, *exc):
                    fake.current = self.prev

        self.cuda = cuda


def _execute(streams, values, rng):
    """Run the queued operations in a random order that honours the waits."""
    heads = {id(s): 0 for s in streams}
    while True:
        ready = []
        for s in streams:
            i = heads[id(s)]
            if i < len(s.ops):
                op = s.ops[i]
                if op["kind"] != "wait" or op["on"] is None or op["on"]["done"]:
                    ready.append(s)
        if not ready:
            break
        s = rng.choice(ready)
        op = s.ops[heads[id(s)]]
        if op["kind"] == "copy":
            values[op["dst"]] = values[op["src"]]
        elif op["kind"] == "run":
            op["fn"](values)
        op["done"] = True
        heads[id(s)] += 1
    assert all(heads[id(s)] == len(s.ops) for s in streams), "a wait never ended"


def _substep(inputs, outputs, dev, step):
    def fn(values):
        total = sum(hash((k, values[dev[k]])) for k in inputs) % 1000003
        for k in outputs:
            values[dev[k]] = (k, step, total)
    return fn


def test_host_state_loop_orders_copies_and_kernels():
    inputs = ["g1", "g2", "rho", "tau", "seed"]      # g*: read only
    outputs = ["rho", "tau", "seed", "flag"]         # flag: write only
    nsteps = 5
    # the reference: the substeps one after another on host values
    ref = {k: ("init", k) for k in set(inputs) | set(outputs)}
    for s in range(nsteps):
        total = sum(hash((k, ref[k])) for k in inputs) % 1000003
        for k in outputs:
            ref[k] = (k, s, total)
    for trial in range(200):
        fake = _FakeTorch()
        dev = {k: _Tensor(fake, "dev:" + k) for k in set(inputs) | set(outputs)}
        host = {k: _Tensor(fake, "host:" + k) for k in dev}
        values = {host[k]: ("init", k) for k in host}
        values.update({dev[k]: ("stale", k) for k in dev})
        loop = HostStateLoop(fake, None, dev, host, inputs, outputs)
        streams = [fake.default, loop.s_in, loop.s_out]
        for s in range(nsteps):
            fn = _substep(inputs, outputs, dev, s)
            loop.step(lambda fn=fn: fake.current.ops.append(
                {"kind": "run", "fn": fn, "done": False}))
        loop.finish()
        _execute(streams, values, random.Random(trial))
        got = {k: values[host[k]] for k in host}
        assert got == ref, trial
