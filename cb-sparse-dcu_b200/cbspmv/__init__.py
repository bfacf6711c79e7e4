"""Python binding of the CB-SpMV C ABI (include/cbspmv.h).

A thin ctypes layer over ``libcbspmv.so`` (built in-tree by
``cb-sparse-dcu_b200/Makefile``).  It mirrors the reference's operator surface
-- ``coo2block_gather`` (cb-spmv-dcu/src/coo2block.h:628) and ``cb_spmv``
(cb-spmv-dcu/src/cb-spmv-dcu.hpp:1088) -- and adds the split upload/execute
calls, the adjoint, and a ``torch.autograd.Function`` used as a test harness.

There is no fallback: if the library is missing, importing this package
raises.  Device arguments are torch CUDA tensors; streams default to torch's
current stream.
"""
from __future__ import annotations

import ctypes
import os
import pathlib

import numpy as np

_HERE = pathlib.Path(__file__).resolve().parent
LIB_PATH = pathlib.Path(os.environ.get("CBSPMV_LIB", _HERE / "libcbspmv.so"))

F64, F32 = 0, 1
STATUS = {0: "OK", 1: "INVALID", 2: "UNSORTED", 3: "BOUNDS", 4: "ALLOC",
          5: "CUDA", 6: "STATE", 7: "UNSUPPORTED", 8: "DEVICE"}


class CBSpMVError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"cbspmv {STATUS.get(code, code)}: {message}")
        self.code = code
        self.status = STATUS.get(code, str(code))


class Opts(ctypes.Structure):
    _fields_ = [("block_size", ctypes.c_int), ("row_owned", ctypes.c_int),
                ("waves_per_block", ctypes.c_int),
                ("dense_sixteenths", ctypes.c_int),
                ("force_coo64", ctypes.c_int), ("value_type", ctypes.c_int),
                ("want_transpose", ctypes.c_int),
                ("tile_entries", ctypes.c_int), ("kernel", ctypes.c_int),
                ("keep_values", ctypes.c_int)]


class CooDesc(ctypes.Structure):
    _fields_ = [("m", ctypes.c_int32), ("n", ctypes.c_int32),
                ("nnz", ctypes.c_int64), ("row", ctypes.c_void_p),
                ("col", ctypes.c_void_p), ("val", ctypes.c_void_p)]


class Metrics(ctypes.Structure):
    _fields_ = [("runtime_ms", ctypes.c_double), ("gflops", ctypes.c_double)]


_INFO_FIELDS = [
    ("m", "q"), ("n", "q"), ("nnz", "q"), ("gb_m", "q"), ("gb_n", "q"),
    ("gb_nnzb", "q"), ("gather_flag", "i"), ("direct_coo_columns", "i"),
    ("compact_coo_indices", "i"), ("load_balanced", "i"), ("unit_values", "i"),
    ("super_sparse_blocks", "q"), ("analyzed_blocks", "q"),
    ("super_sparse_ratio", "d"), ("load_stddev_before", "d"),
    ("load_stddev_after", "d"), ("coo_blocks", "q"), ("csr_blocks", "q"),
    ("dense_blocks", "q"), ("uniform_blocks", "q"), ("segments", "q"),
    ("patterns", "q"), ("stored_values", "q"), ("tiles", "q"),
    ("split_rows", "q"), ("device_bytes", "q"), ("algorithmic_bytes", "q"),
    ("scratch_bytes", "q"), ("rowseg_bytes", "q")]
_CT = {"q": ctypes.c_int64, "i": ctypes.c_int32, "d": ctypes.c_double}


class TuneReport(ctypes.Structure):
    _fields_ = [("block_size", ctypes.c_int), ("tile_entries", ctypes.c_int),
                ("kernel", ctypes.c_int), ("rhs_lanes", ctypes.c_int),
                ("ms", ctypes.c_double), ("tried", ctypes.c_int)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class Info(ctypes.Structure):
    _fields_ = [(k, _CT[t]) for k, t in _INFO_FIELDS]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in _INFO_FIELDS}


_P = ctypes.c_void_p
_I64 = ctypes.c_int64


def _load():
    if not LIB_PATH.exists():
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `make -C "
            f"{_HERE.parent}` (or __graft_entry__.build())")
    lib = ctypes.CDLL(str(LIB_PATH))
    sig = {
        "cbspmv_default_opts": (None, [ctypes.POINTER(Opts)]),
        "cbspmv_coo2block_gather": (ctypes.c_int, [ctypes.POINTER(CooDesc),
                                                   ctypes.POINTER(Opts),
                                                   ctypes.POINTER(_P)]),
        "cbspmv_cb_spmv": (ctypes.c_int, [_P, _P, _P, ctypes.POINTER(Metrics)]),
        "cbspmv_upload": (ctypes.c_int, [_P, _P]),
        "cbspmv_plan_save": (ctypes.c_int, [_P, ctypes.c_char_p]),
        "cbspmv_plan_save_ex": (ctypes.c_int, [_P, ctypes.c_char_p, ctypes.c_int]),
        "cbspmv_plan_load": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(_P)]),
        "cbspmv_plan_opts": (ctypes.c_int, [_P, ctypes.POINTER(Opts)]),
        "cbspmv_spmv": (ctypes.c_int, [_P, _P, _P, ctypes.c_int, _I64, _I64, _P]),
        "cbspmv_spmv_host": (ctypes.c_int, [_P, _P, _P, ctypes.c_int, _P]),
        "cbspmv_spmv_host_async": (ctypes.c_int, [_P, _P, _P, ctypes.c_int, _P]),
        "cbspmv_spmv_t": (ctypes.c_int, [_P, _P, _P, ctypes.c_int, _I64, _I64, _P]),
        "cbspmv_grad_vals": (ctypes.c_int, [_P, _P, _P, _P, ctypes.c_int, _I64,
                                            _I64, _P]),
        "cbspmv_adjoint": (ctypes.c_int, [_P, _P, _P, _P, _P, ctypes.c_int, _I64, _I64,
                                          _I64, _P]),
        "cbspmv_num_values": (_I64, [_P]),
        "cbspmv_adjoint_fused": (ctypes.c_int, [_P, _P, _P, _P, _P, ctypes.c_int, _I64, _I64,
                                                _I64, _P]),
        "cbspmv_grad_size_t": (_I64, [_P]),
        "cbspmv_grad_positions_t": (ctypes.c_int, [_P, _P]),
        "cbspmv_set_values": (ctypes.c_int, [_P, _P, _P]),
        "cbspmv_value_coords": (ctypes.c_int, [_P, _P, _P, _P]),
        "cbspmv_input_slots": (ctypes.c_int, [_P, _P]),
        "cbspmv_info_get": (ctypes.c_int, [_P, ctypes.POINTER(Info)]),
        "cbspmv_export": (_I64, [_P, ctypes.c_char_p, _P]),
        "cbspmv_export_t": (_I64, [_P, ctypes.c_char_p, _P]),
        "cbspmv_export_scalars": (None, [_P, ctypes.c_int, _P, _P]),
        "cbspmv_destroy": (ctypes.c_int, [_P]),
        "cbspmv_last_error": (ctypes.c_size_t, [ctypes.c_char_p, ctypes.c_size_t]),
        "cbspmv_launch_count": (_I64, []),
        "cbspmv_autotune": (ctypes.c_int, [_P, ctypes.c_int, _P, _P, _P]),
        "cbspmv_check": (ctypes.c_int, [_P, _P]),
        "cbspmv_autotune_ex": (ctypes.c_int, [_P, ctypes.c_int, _P, _P, _P, _P]),
        "cbspmv_set_rhs_lanes": (ctypes.c_int, [_P, ctypes.c_int]),
        "cbspmv_tune": (ctypes.c_int, [ctypes.POINTER(CooDesc), ctypes.POINTER(Opts), ctypes.c_int,
                                       _P, ctypes.POINTER(_P), _P]),
        "cbspmv_debug_wait_polls": (None, [_I64]),
        "cbspmv_batch_create": (ctypes.c_int, [_P, ctypes.c_int, _P, ctypes.POINTER(_P)]),
        "cbspmv_batch_bind": (ctypes.c_int, [_P, _P, _P, _P]),
        "cbspmv_batch_run": (ctypes.c_int, [_P, _P]),
        "cbspmv_batch_run_each": (ctypes.c_int, [_P, _P]),
        "cbspmv_batch_graph_launch": (ctypes.c_int, [_P, ctypes.c_int, _P]),
        "cbspmv_batch_destroy": (ctypes.c_int, [_P]),
        "cbspmv_batch_check": (ctypes.c_int, [_P, _P]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


_lib = _load()


def lib():
    return _lib


def last_error() -> str:
    buf = ctypes.create_string_buffer(4096)
    _lib.cbspmv_last_error(buf, len(buf))
    return buf.value.decode()


def _check(code: int) -> None:
    if code != 0:
        raise CBSpMVError(code, last_error())


def launch_count() -> int:
    return int(_lib.cbspmv_launch_count())


def debug_wait_polls(polls: int) -> None:
    """Polls each device wait makes before giving up (0: at once); -1
    restores the default.  For tests of the give-up path."""
    _lib.cbspmv_debug_wait_polls(int(polls))


def default_opts(**kw) -> Opts:
    o = Opts()
    _lib.cbspmv_default_opts(ctypes.byref(o))
    for k, v in kw.items():
        if not hasattr(o, k):
            raise TypeError(f"unknown option {k}")
        setattr(o, k, int(v))
    return o


def _np_ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def _stream(stream):
    if stream is None:
        import torch
        return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    if isinstance(stream, int):
        return ctypes.c_void_p(stream)
    return ctypes.c_void_p(stream.cuda_stream)


def _dptr(t):
    return ctypes.c_void_p(t.data_ptr())


INT_EXPORTS = [
    "gb_row_idx", "gb_col_idx", "gb_row_ptr", "nnz_per_blk", "type_per_blk",
    "segment_rows", "segment_begin", "segment_end", "segment_direct",
    "segment_uniform", "block_row_uniform", "flat_row_ptr", "flat_col_idx",
    "pattern_row_ptr", "pattern_col_idx", "pattern_output_ptr",
    "pattern_output_rows", "block_cols_offset", "block_cols", "bidx_origin",
    "bidx_end", "bidx_nnz"]
EXPORT_DTYPES = {k: np.int32 for k in INT_EXPORTS}
EXPORT_DTYPES.update({"pay_u32": np.uint32, "pay_f64": np.float64,
                      "pay_u32_off": np.int64, "pay_f64_off": np.int64})
SCALARS = ["m", "n", "nnz", "gb_m", "gb_n", "gb_nnzb", "gather_flag",
           "direct_coo_columns", "compact_coo_indices", "super_sparse_blocks",
           "analyzed_blocks", "load_balanced"]
FSCALARS = ["super_sparse_ratio", "load_stddev_before", "load_stddev_after"]


class Plan:
    """A built CB structure (the reference's GLOBAL_BLOCK) plus its device
    layout.  ``Plan(coo)`` is ``coo2block_gather``; ``cb_spmv`` is the
    reference's one-call SpMV; ``spmv`` / ``spmv_t`` / ``grad_vals`` run on
    torch CUDA tensors."""

    def __init__(self, coo=None, *, m=None, n=None, row=None, col=None,
                 val=None, **opts):
        if coo is not None:
            m, n, row, col, val = coo.m, coo.n, coo.row, coo.col, coo.val
        self._row = np.ascontiguousarray(row, np.int32)
        self._col = np.ascontiguousarray(col, np.int32)
        self._val = np.ascontiguousarray(val, np.float64)
        self.m, self.n = int(m), int(n)
        self.nnz = int(self._row.shape[0])
        if self._col.shape[0] != self.nnz or self._val.shape[0] != self.nnz:
            raise CBSpMVError(1, "row, col and val lengths differ")
        self.opts = default_opts(**opts)
        desc = CooDesc(self.m, self.n, self.nnz, _np_ptr(self._row),
                       _np_ptr(self._col), _np_ptr(self._val))
        h = ctypes.c_void_p()
        _check(_lib.cbspmv_coo2block_gather(ctypes.byref(desc),
                                            ctypes.byref(self.opts),
                                            ctypes.byref(h)))
        self._h = h
        self.f32 = self.opts.value_type == F32
        self.bs = self.opts.block_size
        self.has_transpose = bool(self.opts.want_transpose)
        self._uploaded = False

    # ---- plan files
    def save(self, path, spmv_only: bool = False) -> None:
        """Writes the built plan to a .cbplan file (cbspmv_plan_save_ex);
        spmv_only: without the host block arrays and the per-value arrays
        (a plan loaded from it multiplies but cannot take new values or give
        value gradients)."""
        _check(_lib.cbspmv_plan_save_ex(self._h, str(path).encode(), 1 if spmv_only else 0))

    @classmethod
    def load(cls, path) -> "Plan":
        """A plan read from a .cbplan file, without the COO input or the CB
        build (cbspmv_plan_load)."""
        h = ctypes.c_void_p()
        _check(_lib.cbspmv_plan_load(str(path).encode(), ctypes.byref(h)))
        self = cls.__new__(cls)
        self._h = h
        self.opts = Opts()
        _check(_lib.cbspmv_plan_opts(h, ctypes.byref(self.opts)))
        i = self.info()
        self.m, self.n, self.nnz = int(i["m"]), int(i["n"]), int(i["nnz"])
        self.f32 = self.opts.value_type == F32
        self.bs = self.opts.block_size
        self.has_transpose = bool(self.opts.want_transpose)
        self._uploaded = False
        return self

    # ---- lifetime
    def close(self):
        if getattr(self, "_h", None):
            _lib.cbspmv_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- structure
    def info(self) -> dict:
        i = Info()
        _check(_lib.cbspmv_info_get(self._h, ctypes.byref(i)))
        return i.as_dict()

    def export(self, transpose: bool = False) -> dict:
        """All GLOBAL_BLOCK arrays and scalars under the oracle's dump
        names."""
        fn = _lib.cbspmv_export_t if transpose else _lib.cbspmv_export
        s = np.zeros(12, np.int64)
        f = np.zeros(3, np.float64)
        _lib.cbspmv_export_scalars(self._h, int(transpose), _np_ptr(s), _np_ptr(f))
        out = {k: int(v) for k, v in zip(SCALARS, s)}
        out.update({k: float(v) for k, v in zip(FSCALARS, f)})
        for name, dt in EXPORT_DTYPES.items():
            cnt = fn(self._h, name.encode(), None)
            if cnt < 0:
                raise CBSpMVError(1, f"unknown export {name}")
            a = np.zeros(cnt, dt)
            if cnt:
                fn(self._h, name.encode(), _np_ptr(a))
            out[name] = a
        return out

    def num_values(self) -> int:
        return int(_lib.cbspmv_num_values(self._h))

    def value_coords(self):
        k = self.num_values()
        r = np.zeros(k, np.int32)
        c = np.zeros(k, np.int32)
        f = np.zeros(k, np.int64)
        _check(_lib.cbspmv_value_coords(self._h, _np_ptr(r), _np_ptr(c), _np_ptr(f)))
        return r, c, f

    def input_slots(self) -> np.ndarray:
        s = np.zeros(self.nnz, np.int64)
        _check(_lib.cbspmv_input_slots(self._h, _np_ptr(s)))
        return s

    # ---- device
    def upload(self, stream=None):
        if not self._uploaded:
            _check(_lib.cbspmv_upload(self._h, _stream(stream)))
            self._uploaded = True
        return self

    def _check_dev(self, *ts):
        import torch
        want = torch.float32 if self.f32 else torch.float64
        for t in ts:
            if not t.is_cuda or t.dtype != want or not t.is_contiguous():
                raise CBSpMVError(1, f"expected a contiguous CUDA {want} tensor")

    def spmv(self, x, y=None, stream=None):
        """y = A x.  x: (n,) or (n, k) CUDA tensor of the plan's dtype."""
        import torch
        self.upload(stream)
        self._check_dev(x)
        k = 1 if x.dim() == 1 else x.shape[1]
        if y is None:
            y = torch.empty((self.m,) if x.dim() == 1 else (self.m, k),
                            dtype=x.dtype, device=x.device)
        self._check_dev(y)
        _check(_lib.cbspmv_spmv(self._h, _dptr(x), _dptr(y), k, k, k,
                                _stream(stream)))
        return y

    def check(self, stream=None) -> None:
        """Synchronizes and raises CBSpMVError (status DEVICE) if a launch on
        this plan gave up a bounded device wait since the last report."""
        _check(_lib.cbspmv_check(self._h, _stream(stream)))

    def autotune(self, nrhs: int = 1, stream=None):
        """Times the kernels (and, for nrhs > 1, the lanes per entry) that can
        run this plan for nrhs right-hand sides and keeps the fastest;
        returns (kernel, ms)."""
        self.upload(stream)
        k = ctypes.c_int()
        rl = ctypes.c_int()
        ms = ctypes.c_double()
        _check(_lib.cbspmv_autotune_ex(self._h, int(nrhs), _stream(stream), ctypes.byref(k),
                                       ctypes.byref(rl), ctypes.byref(ms)))
        self.opts.kernel = k.value
        self.rhs_lanes = rl.value
        return k.value, ms.value

    def set_rhs_lanes(self, lanes: int) -> None:
        _check(_lib.cbspmv_set_rhs_lanes(self._h, int(lanes)))

    def spmv_t(self, g, gx=None, stream=None):
        """gx = A^T g (needs want_transpose=1)."""
        import torch
        self.upload(stream)
        self._check_dev(g)
        k = 1 if g.dim() == 1 else g.shape[1]
        if gx is None:
            gx = torch.empty((self.n,) if g.dim() == 1 else (self.n, k),
                             dtype=g.dtype, device=g.device)
        self._check_dev(gx)
        _check(_lib.cbspmv_spmv_t(self._h, _dptr(g), _dptr(gx), k, k, k,
                                  _stream(stream)))
        return gx

    def grad_vals(self, g, x, out=None, stream=None):
        """Gradient of <g, A x> w.r.t. the stored value slots."""
        import torch
        self.upload(stream)
        self._check_dev(g, x)
        k = 1 if g.dim() == 1 else g.shape[1]
        if out is None:
            out = torch.empty(self.num_values(), dtype=g.dtype, device=g.device)
        _check(_lib.cbspmv_grad_vals(self._h, _dptr(g), _dptr(x), _dptr(out), k,
                                     k, k, _stream(stream)))
        return out

    def adjoint(self, g, x, gx=None, gvals=None, want_gx=True, want_gvals=True,
                stream=None):
        """(A^T g, value gradient) in one call, the value gradient on a
        second stream of the plan's (needs want_transpose=1 for A^T g);
        returns (gx, gvals), None for an output not wanted."""
        import torch
        self.upload(stream)
        self._check_dev(g, x)
        k = 1 if g.dim() == 1 else g.shape[1]
        if want_gx and gx is None:
            gx = torch.empty((self.n,) if g.dim() == 1 else (self.n, k),
                             dtype=g.dtype, device=g.device)
        if want_gvals and gvals is None:
            gvals = torch.empty(self.num_values(), dtype=g.dtype, device=g.device)
        gx = gx if want_gx else None
        gvals = gvals if want_gvals else None
        for t in (gx, gvals):
            if t is not None:
                self._check_dev(t)
        _check(_lib.cbspmv_adjoint(self._h, _dptr(g), _dptr(x),
                                   _dptr(gx) if gx is not None else None,
                                   _dptr(gvals) if gvals is not None else None,
                                   k, k, k, k, _stream(stream)))
        return gx, gvals

    def adjoint_fused(self, g, x, gx=None, gvals_t=None, stream=None):
        """(A^T g, value gradient) in one kernel launch on the transposed
        layout (its row-segment stream when it has one, else its tiles); the
        value gradient is in that layout's order (see ``grad_positions_t``).
        Returns (gx, gvals_t)."""
        import torch
        self.upload(stream)
        self._check_dev(g, x)
        k = 1 if g.dim() == 1 else g.shape[1]
        if gx is None:
            gx = torch.empty((self.n,) if g.dim() == 1 else (self.n, k),
                             dtype=g.dtype, device=g.device)
        if gvals_t is None:
            gvals_t = torch.zeros(int(_lib.cbspmv_grad_size_t(self._h)), dtype=g.dtype,
                                  device=g.device)
        self._check_dev(gx, gvals_t)
        _check(_lib.cbspmv_adjoint_fused(self._h, _dptr(g), _dptr(x), _dptr(gx),
                                         _dptr(gvals_t), k, k, k, k, _stream(stream)))
        return gx, gvals_t

    def grad_positions_t(self) -> np.ndarray:
        """For each input nonzero, its position in ``adjoint_fused``'s value
        gradient (the order depends on the uploaded layout: uploads first)."""
        self.upload()
        pos = np.zeros(self.nnz, np.int64)
        _check(_lib.cbspmv_grad_positions_t(self._h, _np_ptr(pos)))
        return pos

    def set_values(self, vals, stream=None):
        """Re-pack A (and A^T) from new input values (nnz, caller order)."""
        self.upload(stream)
        self._check_dev(vals)
        if vals.numel() != self.nnz:
            raise CBSpMVError(1, "expected one value per input nonzero")
        _check(_lib.cbspmv_set_values(self._h, _dptr(vals), _stream(stream)))

    def spmv_host(self, x: np.ndarray, nrhs: int = 1) -> np.ndarray:
        """y = A x through host buffers (copies inside)."""
        dt = np.float32 if self.f32 else np.float64
        x = np.ascontiguousarray(x, dt)
        y = np.zeros((self.m, nrhs) if nrhs > 1 else self.m, dt)
        _check(_lib.cbspmv_spmv_host(self._h, _np_ptr(x), _np_ptr(y), nrhs, None))
        self._uploaded = True
        return y

    def cb_spmv(self, x: np.ndarray, y: np.ndarray | None = None):
        """The reference's cb_spmv: host FP64 x and y, one checked launch,
        100 warm-up and 1000 timed launches; returns (y, {runtime, gflops})."""
        x = np.ascontiguousarray(x, np.float64)
        if y is None:
            y = np.zeros(self.m, np.float64)
        met = Metrics()
        _check(_lib.cbspmv_cb_spmv(self._h, _np_ptr(x), _np_ptr(y),
                                   ctypes.byref(met)))
        self._uploaded = True
        return y, {"runtime": met.runtime_ms, "gflops": met.gflops}


class Batch:
    """Several uploaded plans run together (cbspmv_batch_*): Y_k = A_k X_k,
    X_k (n_k, nrhs[k]) and Y_k (m_k, nrhs[k]) contiguous CUDA tensors.
    ``run`` is one persistent kernel launch over all matrices, ``run_each``
    one launch per matrix, ``graph_launch`` replays a CUDA graph of either."""

    def __init__(self, plans, nrhs, stream=None):
        self.plans = list(plans)
        for p in self.plans:
            p.upload(stream)
        self.nrhs = [int(k) for k in nrhs]
        if len(self.nrhs) != len(self.plans):
            raise CBSpMVError(1, "one nrhs value per plan")
        arr = (_P * len(self.plans))(*[p._h for p in self.plans])
        k = np.ascontiguousarray(self.nrhs, np.int32)
        h = ctypes.c_void_p()
        _check(_lib.cbspmv_batch_create(ctypes.cast(arr, _P), len(self.plans),
                                        _np_ptr(k), ctypes.byref(h)))
        self._h = h
        self._io = None

    def bind(self, xs, ys, stream=None):
        """Binds lists of CUDA tensors (kept referenced by the batch)."""
        for p, x, y in zip(self.plans, xs, ys):
            p._check_dev(x, y)
        xa = (_P * len(xs))(*[t.data_ptr() for t in xs])
        ya = (_P * len(ys))(*[t.data_ptr() for t in ys])
        _check(_lib.cbspmv_batch_bind(self._h, ctypes.cast(xa, _P), ctypes.cast(ya, _P),
                                      _stream(stream)))
        self._io = (list(xs), list(ys))
        return self

    def run(self, stream=None):
        _check(_lib.cbspmv_batch_run(self._h, _stream(stream)))

    def run_each(self, stream=None):
        _check(_lib.cbspmv_batch_run_each(self._h, _stream(stream)))

    def graph_launch(self, per_matrix: bool = False, stream=None):
        _check(_lib.cbspmv_batch_graph_launch(self._h, int(per_matrix), _stream(stream)))

    def check(self, stream=None) -> None:
        """Synchronizes and raises CBSpMVError (status DEVICE) if a batch
        launch gave up a bounded device wait since the last report."""
        _check(_lib.cbspmv_batch_check(self._h, _stream(stream)))

    def close(self):
        if getattr(self, "_h", None):
            _lib.cbspmv_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def tune(coo, nrhs: int = 1, stream=None, **opts):
    """cbspmv_tune: the fastest plan over block size (16, 32), tile size
    (auto, 128 entries), kernel and lanes per entry, built from `coo`;
    returns (plan, report dict)."""
    row = np.ascontiguousarray(coo.row, np.int32)
    col = np.ascontiguousarray(coo.col, np.int32)
    val = np.ascontiguousarray(coo.val, np.float64)
    desc = CooDesc(coo.m, coo.n, row.shape[0], _np_ptr(row), _np_ptr(col), _np_ptr(val))
    o = default_opts(**opts)
    h = ctypes.c_void_p()
    rep = TuneReport()
    _check(_lib.cbspmv_tune(ctypes.byref(desc), ctypes.byref(o), int(nrhs), _stream(stream),
                            ctypes.byref(h), ctypes.byref(rep)))
    plan = Plan.__new__(Plan)
    plan._h = h
    plan._row, plan._col, plan._val = row, col, val
    plan.opts = Opts()
    _check(_lib.cbspmv_plan_opts(h, ctypes.byref(plan.opts)))
    plan.m, plan.n, plan.nnz = int(coo.m), int(coo.n), int(row.shape[0])
    plan.f32 = plan.opts.value_type == F32
    plan.bs = plan.opts.block_size
    plan.has_transpose = bool(plan.opts.want_transpose)
    plan._uploaded = True
    plan.rhs_lanes = rep.rhs_lanes
    return plan, rep.as_dict()


def coo2block_gather(row, col, val, m, n, **opts) -> Plan:
    """The reference's coo2block_gather: returns the built Plan."""
    return Plan(m=m, n=n, row=row, col=col, val=val, **opts)


def cb_spmv(plan: Plan, x, y=None):
    """The reference's cb_spmv on a built Plan."""
    return plan.cb_spmv(x, y)


from .autograd import CBSpMVFunction, cbspmv_apply  # noqa: E402,F401
