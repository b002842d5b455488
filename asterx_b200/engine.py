"""Python handle on the engine's C ABI (``include/asterx_b200.h``).

This is the host-side driver used by the tests, ``bench.py`` and
``__graft_entry__``: it loads the in-tree ``libasterx_b200.so``, keeps device
buffers as torch CUDA tensors (torch is used only for memory and streams) and
passes raw pointers to the C entry points.  There is no fallback: if the
library or a B200 is missing, construction raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import abi
from .abi import GF, GF_NAMES, NUM_GF, Box, Fields, Layout, Params

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libasterx_b200.so")

_vp = C.c_void_p
_dp = C.POINTER(C.c_double)


class AxbError(RuntimeError):
    STATUS = {1: "AXB_ERR_ARG", 2: "AXB_ERR_GHOSTS", 3: "AXB_ERR_CUDA",
              4: "AXB_ERR_UNSUPPORTED", 5: "AXB_ERR_TOO_LARGE",
              6: "AXB_ERR_NO_DEVICE"}

    def __init__(self, rc, what):
        super().__init__(f"{what} failed: {self.STATUS.get(rc, rc)}")
        self.rc = rc


def load_library(path=LIB_PATH):
    if not os.path.exists(path):
        raise FileNotFoundError(
            f"{path} is missing: build it with `python -m asterx_b200.build`")
    lib = C.CDLL(path)
    lib.axb_params_default.argtypes = [C.POINTER(Params)]
    lib.axb_gf_name.restype = C.c_char_p
    lib.axb_gf_name.argtypes = [C.c_int]
    lib.axb_ctx_create.argtypes = [C.c_int, C.POINTER(_vp)]
    lib.axb_ctx_destroy.argtypes = [_vp]
    lib.axb_status_reset.argtypes = [_vp, _vp]
    lib.axb_status_read.argtypes = [_vp, _vp, C.POINTER(C.c_uint32),
                                    C.POINTER(C.c_double), C.POINTER(C.c_uint32),
                                    C.POINTER(C.c_uint64)]
    lib.axb_eos_create_idealgas.argtypes = [C.c_double, C.c_double, _dp, _dp, _dp,
                                            C.c_double, C.c_double, C.POINTER(_vp)]
    lib.axb_eos_create_tabulated3d.argtypes = [C.c_int, C.c_int, C.c_int, _dp, _dp, _dp,
                                               _dp, C.c_double, C.c_double, C.c_double,
                                               C.POINTER(_vp)]
    lib.axb_eos_destroy.argtypes = [_vp]
    lib.axb_rhs_group.argtypes = [_vp, C.POINTER(Box), C.POINTER(Fields),
                                  C.POINTER(Params), _vp, _vp]
    lib.axb_con2prim_group.argtypes = [_vp, C.POINTER(Box), C.POINTER(Fields),
                                       C.POINTER(Params), _vp, _vp]
    lib.axb_con2prim_group_guess.argtypes = [_vp, C.POINTER(Box), C.POINTER(Fields),
                                             C.POINTER(Params), _vp, _vp, _vp]
    lib.axb_rk_stage.argtypes = [_vp, C.POINTER(Box)] + [C.POINTER(Fields)] * 4 + \
        [C.c_double] * 4 + [_vp]
    lib.axb_sync_periodic.argtypes = [_vp, C.POINTER(Box), C.POINTER(Fields),
                                      C.POINTER(C.c_int), C.c_int, _vp]
    lib.axb_substep.argtypes = [_vp, C.POINTER(Box), C.POINTER(Fields),
                                C.POINTER(Fields), C.POINTER(Params), _vp,
                                C.c_double, C.c_double, C.c_double, C.c_double,
                                C.c_int, _vp]
    _fp = C.POINTER(C.c_float)
    lib.axb_mlp_param_count.argtypes = [C.c_int]
    lib.axb_mlp_param_count.restype = C.c_int64
    lib.axb_mlp_create.argtypes = [C.c_int, _vp, C.c_uint64, C.c_double, C.POINTER(_vp)]
    lib.axb_mlp_create_act.argtypes = [C.c_int, C.c_int, _vp, C.c_uint64, C.c_double,
                                       C.POINTER(_vp)]
    lib.axb_mlp_create_act.restype = C.c_int
    lib.axb_mlp_destroy.argtypes = [_vp]
    lib.axb_mlp_get_params.argtypes = [_vp, _vp]
    lib.axb_mlp_features.argtypes = [_vp, C.POINTER(abi.Cells), C.c_int, _vp, _vp]
    lib.axb_mlp_forward.argtypes = [_vp, _vp, _vp, C.c_int64, _vp, _vp]
    lib.axb_mlp_train_step.argtypes = [_vp, _vp, _vp, _vp, C.c_int64, C.c_float, C.c_float,
                                       C.c_float, C.c_float, _vp, _vp, _vp]
    lib.axb_c2p_cells.argtypes = [_vp, C.POINTER(abi.Cells), C.POINTER(Params), _vp, _vp,
                                  _vp]
    lib.axb_batch_create.argtypes = [_vp, C.c_int, C.POINTER(Box), C.POINTER(Fields),
                                     C.POINTER(Fields), C.POINTER(Params), _vp, C.POINTER(_vp)]
    lib.axb_batch_destroy.argtypes = [_vp]
    lib.axb_batch_substep.argtypes = [_vp, _vp, C.c_double, C.c_double, C.c_double,
                                      C.c_double, C.c_int, _vp]
    lib.axb_batch_autotune.argtypes = [_vp, _vp, C.POINTER(C.c_int), _vp]
    lib.axb_import_fields.argtypes = [_vp, C.POINTER(Box), C.POINTER(abi.FieldsStrided),
                                      C.POINTER(C.c_int), C.c_int, C.POINTER(Fields), _vp]
    lib.axb_import_fields.restype = C.c_int
    lib.axb_export_fields.argtypes = [_vp, C.POINTER(Box), C.POINTER(Fields),
                                      C.POINTER(C.c_int), C.c_int,
                                      C.POINTER(abi.FieldsStrided), _vp]
    lib.axb_export_fields.restype = C.c_int
    lib.axb_fill_boundary.argtypes = [_vp, C.POINTER(Box), C.POINTER(Fields),
                                      C.POINTER(C.c_int), C.c_int, C.POINTER(C.c_int), _vp]
    lib.axb_fill_boundary.restype = C.c_int
    lib.axb_rhs_group_bc.argtypes = [_vp, C.POINTER(Box), C.POINTER(Fields),
                                     C.POINTER(Params), _vp, C.POINTER(C.c_int), _vp]
    lib.axb_rhs_group_bc.restype = C.c_int
    lib.axb_rk_lincomb.argtypes = [_vp, C.POINTER(Box), C.POINTER(Fields), C.c_int,
                                   _dp, C.POINTER(C.POINTER(Fields)), C.c_double,
                                   C.POINTER(Fields), _vp]
    lib.axb_rk_lincomb.restype = C.c_int
    lib.axb_tmunu.argtypes = [_vp, C.POINTER(Box), C.POINTER(Fields), C.POINTER(Params),
                              C.c_int, C.POINTER(_dp), _vp]
    lib.axb_tmunu.restype = C.c_int
    lib.axb_estimate_error.argtypes = [_vp, C.POINTER(Box), C.POINTER(_dp), C.c_int, C.c_int,
                                       C.c_double, _dp, _vp]
    lib.axb_estimate_error.restype = C.c_int
    lib.axb_probe_fp64.argtypes = [_dp]
    lib.axb_probe_fp64.restype = C.c_int
    lib.axb_timing_begin.argtypes = [_vp]
    lib.axb_timing_end.argtypes = [_vp, C.POINTER(C.c_double), C.POINTER(C.c_int), C.c_int]
    for name in ("axb_con2prim_group", "axb_substep", "axb_rk_stage",
                 "axb_sync_periodic", "axb_c2p_cells", "axb_eos_create_tabulated3d",
                 "axb_mlp_create", "axb_mlp_destroy", "axb_mlp_get_params",
                 "axb_mlp_features", "axb_mlp_forward", "axb_mlp_train_step",
                 "axb_batch_create", "axb_batch_destroy", "axb_batch_substep",
                 "axb_batch_autotune"):
        if hasattr(lib, name):
            getattr(lib, name).restype = C.c_int
    return lib


class Engine:
    """One device context of the engine."""

    def __init__(self, device=0, path=LIB_PATH):
        import torch
        if not torch.cuda.is_available():
            raise RuntimeError("the engine needs a CUDA device (sm_100)")
        self.torch = torch
        self.device = torch.device("cuda", device)
        torch.cuda.set_device(self.device)
        self.lib = load_library(path)
        self.ctx = _vp()
        self._check(self.lib.axb_ctx_create(device, C.byref(self.ctx)), "axb_ctx_create")
        self._eos = []
        self._mlp = []
        self._batches = []

    def _check(self, rc, what):
        if rc != 0:
            raise AxbError(rc, what)

    def stream_ptr(self, stream=None):
        s = stream if stream is not None else self.torch.cuda.current_stream(self.device)
        return _vp(s.cuda_stream)

    # -- equations of state ---------------------------------------------------
    def eos_idealgas(self, gamma, umass=1.0, rho=(1e-40, 1.0), eps=(0.0, 2.0),
                     ye=(0.0, 1.0), poly_gamma=2.0, poly_k=100.0):
        h = _vp()
        r = (C.c_double * 2)(*rho)
        e = (C.c_double * 2)(*eps)
        y = (C.c_double * 2)(*ye)
        self._check(self.lib.axb_eos_create_idealgas(
            gamma, umass, C.cast(r, _dp), C.cast(e, _dp), C.cast(y, _dp),
            poly_gamma, poly_k, C.byref(h)), "axb_eos_create_idealgas")
        self._eos.append(h)
        return h

    def eos_tabulated(self, logrho, logtemp, ye, table, energy_shift=0.0,
                      poly_gamma=2.0, poly_k=100.0):
        """Tabulated3d EOS from arrays in the layout of
        ``workloads.synthetic_table`` (19 variables per node, variable
        fastest)."""
        arrs = [np.ascontiguousarray(a, dtype=np.float64)
                for a in (logrho, logtemp, ye, table)]
        lr, lt, y, t = arrs
        if t.size != 19 * lr.size * lt.size * y.size:
            raise ValueError("table size does not match the axes")
        h = _vp()
        ptr = [a.ctypes.data_as(_dp) for a in arrs]
        self._check(self.lib.axb_eos_create_tabulated3d(
            len(lr), len(lt), len(y), *ptr, energy_shift, poly_gamma, poly_k,
            C.byref(h)), "axb_eos_create_tabulated3d")
        self._eos.append(h)
        return h

    def eos_stellarcollapse(self, datasets, poly_gamma=2.0, poly_k=100.0):
        """Tabulated3d EOS from a StellarCollapse table's datasets as the
        file holds them (eos_tables.read_stellarcollapse), converted as the
        reference's reader converts them."""
        from . import eos_tables as T
        T.bind(self.lib)
        (nrho, ntemp, nye), axes, sets, ptrs, shift = T._args(datasets)
        h = _vp()
        self._check(self.lib.axb_eos_create_stellarcollapse(
            nrho, ntemp, nye, *[a.ctypes.data_as(_dp) for a in axes], ptrs, shift,
            poly_gamma, poly_k, C.byref(h)), "axb_eos_create_stellarcollapse")
        self._eos.append(h)
        return h

    # -- memory ---------------------------------------------------------------
    def upload(self, layout: Layout, fields: dict, names=None):
        """Device copies (torch float64 tensors) of the given host arrays, plus
        zero-filled buffers for every other grid function in ``names``."""
        t = self.torch
        out = {}
        for n, a in fields.items():
            out[n] = t.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).to(self.device)
        for n in (names or GF_NAMES):
            if n not in out:
                out[n] = t.zeros(layout.size, dtype=t.float64, device=self.device)
        return out

    @staticmethod
    def fields_struct(tensors: dict) -> Fields:
        f = Fields()
        for n, ten in tensors.items():
            if n in GF:
                f.gf[GF[n]] = ten.data_ptr()
        return f

    # -- routines ---------------------------------------------------------------
    def rhs_group(self, layout: Layout, tensors: dict, params: Params, eos, stream=None):
        box = layout.box()
        f = self.fields_struct(tensors)
        self._check(self.lib.axb_rhs_group(self.ctx, C.byref(box), C.byref(f),
                                           C.byref(params), eos,
                                           self.stream_ptr(stream)), "axb_rhs_group")

    def con2prim_group(self, layout: Layout, tensors: dict, params: Params, eos,
                       stream=None, mlp=None):
        """axb_con2prim_group, or axb_con2prim_group_guess with a network."""
        box = layout.box()
        f = self.fields_struct(tensors)
        if mlp is None:
            self._check(self.lib.axb_con2prim_group(self.ctx, C.byref(box), C.byref(f),
                                                    C.byref(params), eos,
                                                    self.stream_ptr(stream)),
                        "axb_con2prim_group")
        else:
            self._check(self.lib.axb_con2prim_group_guess(self.ctx, C.byref(box), C.byref(f),
                                                          C.byref(params), eos, mlp,
                                                          self.stream_ptr(stream)),
                        "axb_con2prim_group_guess")

    @staticmethod
    def strided_struct(arrays: dict):
        """axb_fields_strided from {name: (tensor, sy, sz)}."""
        fs = abi.FieldsStrided()
        for n, (t, sy, sz) in arrays.items():
            fs.gf[GF[n]] = t.data_ptr()
            fs.sy[GF[n]] = int(sy)
            fs.sz[GF[n]] = int(sz)
        return fs

    def import_fields(self, layout, strided, names, tensors, stream=None):
        """axb_import_fields: `strided` {name: (tensor, sy, sz)} into the
        engine-layout `tensors`."""
        box = layout.box()
        fs = self.strided_struct(strided)
        f = self.fields_struct(tensors)
        ids = (C.c_int * len(names))(*[GF[n] for n in names])
        self._check(self.lib.axb_import_fields(self.ctx, C.byref(box), C.byref(fs), ids,
                                               len(names), C.byref(f), self.stream_ptr(stream)),
                    "axb_import_fields")

    def export_fields(self, layout, tensors, names, strided, stream=None):
        box = layout.box()
        fs = self.strided_struct(strided)
        f = self.fields_struct(tensors)
        ids = (C.c_int * len(names))(*[GF[n] for n in names])
        self._check(self.lib.axb_export_fields(self.ctx, C.byref(box), C.byref(f), ids,
                                               len(names), C.byref(fs), self.stream_ptr(stream)),
                    "axb_export_fields")

    def fill_boundary(self, layout, tensors, names, bc, stream=None):
        """axb_fill_boundary: the ghost layers of `names` by the face rules
        bc = (x-lower, x-upper, y-lower, y-upper, z-lower, z-upper), each an
        abi.BC_* code."""
        box = layout.box()
        f = self.fields_struct(tensors)
        ids = (C.c_int * len(names))(*[GF[n] for n in names])
        b = (C.c_int * 6)(*bc)
        self._check(self.lib.axb_fill_boundary(self.ctx, C.byref(box), C.byref(f), ids,
                                               len(names), b, self.stream_ptr(stream)),
                    "axb_fill_boundary")

    def tmunu(self, layout, tensors, params, eT, interp_order=2, stream=None):
        """axb_tmunu: add T_{mu nu} at the interior vertices to the ten
        tensors eT = [eTtt, eTtx, eTty, eTtz, eTxx, eTxy, eTxz, eTyy, eTyz,
        eTzz] (the box's layout)."""
        box = layout.box()
        f = self.fields_struct(tensors)
        ptrs = (_dp * 10)(*[C.cast(t.data_ptr(), _dp) for t in eT])
        self._check(self.lib.axb_tmunu(self.ctx, C.byref(box), C.byref(f), C.byref(params),
                                       interp_order, ptrs, self.stream_ptr(stream)),
                    "axb_tmunu")

    def estimate_error(self, layout, vars, method, out, epsilon_err=0.0, stream=None):
        """axb_estimate_error: the regrid indicator `method` (an abi.REGRID
        code) of the tensors `vars` at the interior cells, written to `out`."""
        box = layout.box()
        ptrs = (_dp * len(vars))(*[C.cast(t.data_ptr(), _dp) for t in vars])
        self._check(self.lib.axb_estimate_error(self.ctx, C.byref(box), ptrs, len(vars),
                                                method, epsilon_err,
                                                C.cast(out.data_ptr(), _dp),
                                                self.stream_ptr(stream)),
                    "axb_estimate_error")

    def rhs_group_bc(self, layout, tensors, params, eos, bc, stream=None):
        """axb_rhs_group_bc: the RHS group with physical outer boundaries."""
        box = layout.box()
        f = self.fields_struct(tensors)
        b = (C.c_int * 6)(*bc)
        self._check(self.lib.axb_rhs_group_bc(self.ctx, C.byref(box), C.byref(f),
                                              C.byref(params), eos, b,
                                              self.stream_ptr(stream)), "axb_rhs_group_bc")

    def rk_lincomb(self, layout, out, states, coef, gdt, rhs, stream=None):
        """axb_rk_lincomb: out = sum coef[q] * states[q] + gdt * RHS (rhs: a
        dict with the RHS grid functions' names)."""
        box = layout.box()
        fo = self.fields_struct(out)
        fs = [self.fields_struct(t) for t in states]
        fr = self.fields_struct(rhs)
        arr = (C.POINTER(Fields) * len(fs))(*[C.pointer(x) for x in fs])
        cf = (C.c_double * len(coef))(*coef)
        self._check(self.lib.axb_rk_lincomb(self.ctx, C.byref(box), C.byref(fo), len(fs),
                                            cf, arr, gdt, C.byref(fr),
                                            self.stream_ptr(stream)), "axb_rk_lincomb")

    def rk_stage(self, layout, out, un, uk, rhs, alpha, beta, gamma, dt, stream=None):
        box = layout.box()
        fs = [self.fields_struct(t) for t in (out, un, uk, rhs)]
        self._check(self.lib.axb_rk_stage(self.ctx, C.byref(box), *[C.byref(x) for x in fs],
                                          alpha, beta, gamma, dt,
                                          self.stream_ptr(stream)), "axb_rk_stage")

    def sync_periodic(self, layout, tensors, names, stream=None):
        box = layout.box()
        f = self.fields_struct(tensors)
        ids = (C.c_int * len(names))(*[GF[n] for n in names])
        self._check(self.lib.axb_sync_periodic(self.ctx, C.byref(box), C.byref(f), ids,
                                               len(names), self.stream_ptr(stream)),
                    "axb_sync_periodic")

    # -- multi-GPU halo exchange (z-slabs over NCCL) ------------------------------
    def _bind_halo(self):
        L = self.lib
        L.axb_halo_unique_id.argtypes = [C.c_char_p]
        L.axb_halo_create.argtypes = [_vp, C.POINTER(Box), C.c_int, C.c_int, C.c_char_p,
                                      C.POINTER(C.c_int), C.c_int, C.POINTER(_vp)]
        L.axb_halo_exchange.argtypes = [_vp, C.POINTER(Fields), _vp]
        L.axb_halo_destroy.argtypes = [_vp]

    def halo_unique_id(self) -> bytes:
        self._bind_halo()
        buf = C.create_string_buffer(128)
        self._check(self.lib.axb_halo_unique_id(buf), "axb_halo_unique_id")
        return buf.raw

    def halo_create(self, layout, nranks, rank, uid: bytes, names):
        self._bind_halo()
        h = _vp()
        box = layout.box()
        ids = (C.c_int * len(names))(*[GF[n] for n in names])
        self._check(self.lib.axb_halo_create(self.ctx, C.byref(box), nranks, rank, uid, ids,
                                             len(names), C.byref(h)), "axb_halo_create")
        return h

    def halo_exchange(self, halo, tensors, stream=None):
        f = self.fields_struct(tensors)
        self._check(self.lib.axb_halo_exchange(halo, C.byref(f), self.stream_ptr(stream)),
                    "axb_halo_exchange")

    def halo_destroy(self, halo):
        self._check(self.lib.axb_halo_destroy(halo), "axb_halo_destroy")

    def substep(self, layout, tensors, tensors_n, params, eos, alpha, beta, gamma, dt,
                periodic=True, stream=None):
        box = layout.box()
        f = self.fields_struct(tensors)
        fn = self.fields_struct(tensors_n)
        self._check(self.lib.axb_substep(self.ctx, C.byref(box), C.byref(f), C.byref(fn),
                                         C.byref(params), eos, alpha, beta, gamma, dt,
                                         int(periodic), self.stream_ptr(stream)),
                    "axb_substep")

    def probe_fp64(self):
        """FP64 rates of this device: FMA TFLOP/s, divisions, square roots and
        reciprocal square roots in G/s (axb_probe_fp64)."""
        out = (C.c_double * 4)()
        self._check(self.lib.axb_probe_fp64(out), "axb_probe_fp64")
        return dict(fma_tflops=out[0], div_gops=out[1], sqrt_gops=out[2],
                    rsqrt_gops=out[3])

    def timing_begin(self):
        self._check(self.lib.axb_timing_begin(self.ctx), "axb_timing_begin")

    def timing_end(self, nregions=14):
        ms = (C.c_double * nregions)()
        cnt = (C.c_int * nregions)()
        self._check(self.lib.axb_timing_end(self.ctx, ms, cnt, nregions), "axb_timing_end")
        return list(ms), list(cnt)

    def status_reset(self, stream=None):
        self._check(self.lib.axb_status_reset(self.ctx, self.stream_ptr(stream)),
                    "axb_status_reset")

    def status(self, stream=None):
        ew = C.c_uint32()
        ms = C.c_double()
        nf = C.c_uint32()
        hist = (C.c_uint64 * 64)()
        self._check(self.lib.axb_status_read(self.ctx, self.stream_ptr(stream),
                                             C.byref(ew), C.byref(ms), C.byref(nf),
                                             hist), "axb_status_read")
        return dict(error_word=ew.value, max_speed=ms.value, c2p_fail=nf.value,
                    iter_hist=np.array(hist[:], dtype=np.int64))

    # -- independent cells and the learned guess -----------------------------
    def cells(self, n, tensors: dict):
        """axb_cells over torch device tensors (float64, length n) keyed by
        abi.CELL_INPUTS / CELL_SEEDS / CELL_OUTPUTS names."""
        ptrs = {}
        for k, t in tensors.items():
            if t is None:
                continue
            assert t.dtype == self.torch.float64 and t.is_cuda and t.numel() >= n, k
            ptrs[k] = t.data_ptr()
        return abi.cells_struct(n, ptrs)

    def c2p_cells(self, cells, params: Params, eos, mlp=None, stream=None):
        if mlp is not None and not cells.guess:
            # scratch for the learned guess, kept for later calls of this size
            n = int(cells.n)
            buf = getattr(self, "_guess_buf", None)
            if buf is None or buf.numel() < 2 * n:
                buf = self.torch.empty(2 * n, dtype=self.torch.float32, device=self.device)
                self._guess_buf = buf
            cells.guess = buf.data_ptr()
        self._check(self.lib.axb_c2p_cells(self.ctx, C.byref(cells), C.byref(params), eos,
                                           mlp, self.stream_ptr(stream)), "axb_c2p_cells")

    def mlp_create(self, nf=8, params=None, seed=1, bracket=0.05, act="silu"):
        h = _vp()
        arr = None
        if params is not None:
            arr = np.ascontiguousarray(params, dtype=np.float32)
            assert arr.size == self.lib.axb_mlp_param_count(nf)
        a = {"silu": 0, "relu": 1}[act]
        self._check(self.lib.axb_mlp_create_act(nf, a, None if arr is None else arr.ctypes.data,
                                                seed, bracket, C.byref(h)),
                    "axb_mlp_create_act")
        self._mlp.append(h)
        return h

    def mlp_params(self, mlp, nf):
        out = np.zeros(self.lib.axb_mlp_param_count(nf), dtype=np.float32)
        self._check(self.lib.axb_mlp_get_params(mlp, out.ctypes.data), "axb_mlp_get_params")
        return out

    def mlp_features(self, cells, nf, out, stream=None):
        self._check(self.lib.axb_mlp_features(self.ctx, C.byref(cells), nf, out.data_ptr(),
                                              self.stream_ptr(stream)), "axb_mlp_features")

    def mlp_forward(self, mlp, features, out, stream=None):
        n = features.shape[0]
        self._check(self.lib.axb_mlp_forward(self.ctx, mlp, features.data_ptr(), n,
                                             out.data_ptr(), self.stream_ptr(stream)),
                    "axb_mlp_forward")

    def mlp_train_step(self, mlp, features, targets, lr=1e-3, betas=(0.9, 0.999),
                       eps=1e-8, loss=None, grad=None, stream=None):
        n = features.shape[0]
        self._check(self.lib.axb_mlp_train_step(
            self.ctx, mlp, features.data_ptr(), targets.data_ptr(), n, lr, betas[0],
            betas[1], eps, None if loss is None else loss.data_ptr(),
            None if grad is None else grad.data_ptr(), self.stream_ptr(stream)),
            "axb_mlp_train_step")

    # -- batched level --------------------------------------------------------
    def batch_create(self, layouts, tensors, tensors_n, params: Params, eos):
        """A batch over boxes (Layouts) with their device tensors (U_k) and the
        U_n tensors of the evolved variables."""
        n = len(layouts)
        boxes = (Box * n)(*[L.box() for L in layouts])
        fs = (Fields * n)(*[self.fields_struct(t) for t in tensors])
        fns = (Fields * n)(*[self.fields_struct(t) for t in tensors_n])
        h = _vp()
        self._check(self.lib.axb_batch_create(self.ctx, n, boxes, fs, fns, C.byref(params),
                                              eos, C.byref(h)), "axb_batch_create")
        self._batches.append(h)
        return h

    def batch_substep(self, batch, alpha, beta, gamma, dt, periodic=True, stream=None):
        self._check(self.lib.axb_batch_substep(self.ctx, batch, alpha, beta, gamma, dt,
                                               int(periodic), self.stream_ptr(stream)),
                    "axb_batch_substep")

    def batch_autotune(self, batch, stream=None):
        out = (C.c_int * 3)()
        self._check(self.lib.axb_batch_autotune(self.ctx, batch, out, self.stream_ptr(stream)),
                    "axb_batch_autotune")
        return dict(seg_y=out[0], seg_z=out[1], ctas_per_sm=out[2])

    def batch_destroy(self, batch):
        self.lib.axb_batch_destroy(batch)
        self._batches = [b for b in self._batches if b.value != batch.value]

    def close(self):
        for h in self._batches:
            self.lib.axb_batch_destroy(h)
        self._batches = []
        for h in self._mlp:
            self.lib.axb_mlp_destroy(h)
        self._mlp = []
        for h in self._eos:
            self.lib.axb_eos_destroy(h)
        self._eos = []
        if self.ctx:
            self.lib.axb_ctx_destroy(self.ctx)
            self.ctx = _vp()
