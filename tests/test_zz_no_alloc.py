"""axb_rhs_group_noalloc: the RHS group for callers that cannot allocate
device memory.  It must give the same RHS as axb_rhs_group (to the 1e-12
tolerance of the RHS parity tests) on two calls in a row, taking its scratch
from the library's static device array, and reject boxes beyond its limit.
This file is collected last so a failing run has already run everything
else; it creates its own engine, so it also passes alone."""
import ctypes as C

import pytest

from asterx_b200 import abi
from asterx_b200 import workloads as W
from tests.helpers import errors, full_fields, interior

OUT = abi.HYDRO_RHS + abi.AVEC_RHS
SCRATCH = abi.ACC + abi.BFLUX + abi.AUX


@pytest.mark.gpu
def test_rhs_group_noalloc_matches_rhs_group():
    import torch

    from asterx_b200.engine import Engine

    eng = Engine(0)
    try:
        lib = eng.lib
        lib.axb_rhs_group_noalloc.argtypes = [C.POINTER(abi.Box), C.POINTER(abi.Fields),
                                              C.POINTER(abi.Params), C.c_void_p,
                                              C.c_void_p]
        lib.axb_rhs_group_noalloc.restype = C.c_int
        L, f = W.curved_box(n=16, ng=3, seed=17, wmax=2.0, sigma=(1e-3, 0.3),
                            theta=(0.1, 1.0))
        f = full_fields(L, f)
        p = abi.default_params(reconstruction_method="wenoz", flux_type="hlle")
        eos = eng.eos_idealgas(4.0 / 3.0, rho=(1e-40, 1e10), eps=(0.0, 1e10))
        dev = eng.upload(L, f)
        eng.rhs_group(L, dev, p, eos)
        torch.cuda.synchronize()
        want = {n: dev[n].cpu().numpy() for n in OUT}

        # first a call on a box of another size, seed and layout, so that the
        # static array holds values the 16^3 calls below do not write: a
        # kernel that read a scratch entry its group never writes would see
        # them
        L2, f2 = W.curved_box(n=20, ng=3, seed=23, wmax=2.0, sigma=(1e-3, 0.3),
                              theta=(0.1, 1.0))
        f2 = full_fields(L2, f2)
        dev2 = eng.upload(L2, f2)
        io2 = {n: t for n, t in dev2.items() if n not in SCRATCH}
        box2 = L2.box()
        fields2 = eng.fields_struct(io2)
        rc = lib.axb_rhs_group_noalloc(C.byref(box2), C.byref(fields2), C.byref(p),
                                       eos, eng.stream_ptr())
        assert rc == 0
        torch.cuda.synchronize()
        del dev2, io2

        # inputs and outputs only: no scratch pointers at all
        io = {n: t for n, t in dev.items() if n not in SCRATCH}
        box = L.box()
        fields = eng.fields_struct(io)
        for call in range(2):
            for n in OUT:
                io[n].fill_(float("nan"))
            rc = lib.axb_rhs_group_noalloc(C.byref(box), C.byref(fields), C.byref(p),
                                           eos, eng.stream_ptr())
            assert rc == 0
            torch.cuda.synchronize()
            for n in OUT:
                got = io[n].cpu().numpy()
                emax, _ = errors(interior(L, n, got), interior(L, n, want[n]))
                assert emax <= 1e-12, (call, n, emax)

        # a box beyond the static array is refused, not run
        Lbig = abi.Layout((48, 48, 48), 3, (1 / 48,) * 3, (0, 0, 0))
        bigbox = Lbig.box()
        rc = lib.axb_rhs_group_noalloc(C.byref(bigbox), C.byref(fields), C.byref(p),
                                       eos, eng.stream_ptr())
        assert rc == 5  # AXB_ERR_TOO_LARGE
        # sizes out of range are refused before any arithmetic on them
        huge = L.box()
        huge.ng = 1 << 30
        rc = lib.axb_rhs_group_noalloc(C.byref(huge), C.byref(fields), C.byref(p),
                                       eos, eng.stream_ptr())
        assert rc == 1  # AXB_ERR_ARG
    finally:
        eng.close()
