"""Loads CB builders that share the ``cbdump_*`` ABI and returns their output
as numpy arrays, so the reference (oracle/_ref), the oracle restatement
(oracle/liboracle.so) and the product builder can be compared array by array.

Test infrastructure only.
"""
from __future__ import annotations

import ctypes
import os
import pathlib

import numpy as np

REPO = pathlib.Path(__file__).resolve().parent.parent
ORACLE_DIR = REPO / "oracle"
REF_DIR = ORACLE_DIR / "_ref"

INT_ARRAYS = [
    "gb_row_idx", "gb_col_idx", "gb_row_ptr", "nnz_per_blk", "type_per_blk",
    "segment_rows", "segment_begin", "segment_end", "segment_direct",
    "segment_uniform", "block_row_uniform", "flat_row_ptr", "flat_col_idx",
    "pattern_row_ptr", "pattern_col_idx", "pattern_output_ptr",
    "pattern_output_rows", "block_cols_offset", "block_cols", "bidx_origin",
    "bidx_end", "bidx_nnz",
]
DTYPES = {name: np.int32 for name in INT_ARRAYS}
DTYPES.update({"pay_u32": np.uint32, "pay_f64": np.float64,
               "pay_u32_off": np.int64, "pay_f64_off": np.int64})
SCALARS = ["m", "n", "nnz", "gb_m", "gb_n", "gb_nnzb", "gather_flag",
           "direct_coo_columns", "compact_coo_indices", "super_sparse_blocks",
           "analyzed_blocks", "load_balanced"]
FSCALARS = ["super_sparse_ratio", "load_stddev_before", "load_stddev_after"]

_P = ctypes.c_void_p


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def _setup(lib):
    lib.cbdump_free.argtypes = [_P]
    lib.cbdump_scalars.argtypes = [_P, _P, _P]
    lib.cbdump_array.argtypes = [_P, ctypes.c_char_p, _P]
    lib.cbdump_array.restype = ctypes.c_int64
    return lib


def dump(lib, handle) -> dict:
    """All scalars and arrays of a built handle, then frees it."""
    s = np.zeros(12, np.int64)
    f = np.zeros(3, np.float64)
    lib.cbdump_scalars(handle, _ptr(s), _ptr(f))
    out = {k: int(v) for k, v in zip(SCALARS, s)}
    out.update({k: float(v) for k, v in zip(FSCALARS, f)})
    for name, dt in DTYPES.items():
        n = lib.cbdump_array(handle, name.encode(), None)
        assert n >= 0, name
        a = np.zeros(n, dt)
        lib.cbdump_array(handle, name.encode(), _ptr(a) if n else None)
        out[name] = a
    lib.cbdump_free(handle)
    return out


_ORACLE = None


def oracle_lib():
    global _ORACLE
    if _ORACLE is None:
        path = ORACLE_DIR / "liboracle.so"
        if not path.exists():
            raise RuntimeError(f"{path} missing: run `make -C oracle`")
        lib = _setup(ctypes.CDLL(str(path)))
        lib.oracle_build.restype = _P
        lib.oracle_build.argtypes = [ctypes.c_int] * 7 + [ctypes.c_int64, _P, _P, _P]
        lib.oracle_spmv_coo.argtypes = [ctypes.c_int, ctypes.c_int64, _P, _P, _P, _P, _P]
        lib.oracle_spmm_coo_ld.argtypes = [ctypes.c_int, ctypes.c_int64, _P, _P, _P,
                                           ctypes.c_int, _P, ctypes.c_int64, _P,
                                           ctypes.c_int64, _P]
        lib.oracle_spmm_t_coo_ld.argtypes = lib.oracle_spmm_coo_ld.argtypes
        lib.oracle_grad_vals.argtypes = [ctypes.c_int64, _P, _P, ctypes.c_int, _P,
                                         ctypes.c_int64, _P, ctypes.c_int64, _P]
        lib.oracle_cb_decode_spmv.restype = ctypes.c_int
        lib.oracle_cb_decode_spmv.argtypes = [ctypes.c_int, ctypes.c_int64,
                                              ctypes.c_int64] + [ctypes.c_int] * 3 + [_P] * 11
        _ORACLE = lib
    return _ORACLE


_REF = {}


def ref_lib(bs: int, row_owned: int):
    """The reference's own host code for one compile-time configuration, or
    None when oracle/_ref has not been built (no reference sources here)."""
    key = (bs, row_owned)
    if key not in _REF:
        path = REF_DIR / f"libcbref_bs{bs}_ro{row_owned}.so"
        if not path.exists():
            _REF[key] = None
        else:
            lib = _setup(ctypes.CDLL(str(path)))
            lib.cbdump_build.restype = _P
            lib.cbdump_build.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                         _P, _P, _P]
            lib.cbref_spmv_prepare.restype = _P
            lib.cbref_spmv_prepare.argtypes = [ctypes.c_int, ctypes.c_int,
                                               ctypes.c_int64, _P, _P, _P, _P]
            lib.cbref_spmv_set_y.argtypes = [_P, _P]
            lib.cbref_spmv_check.argtypes = [_P]
            lib.cbref_spmv_check.restype = ctypes.c_int
            lib.cbref_spmv_free.argtypes = [_P]
            _REF[key] = lib
    return _REF[key]


def _coo_arrays(coo):
    row = np.ascontiguousarray(coo.row, np.int32)
    col = np.ascontiguousarray(coo.col, np.int32)
    val = np.ascontiguousarray(coo.val, np.float64)
    return row, col, val


def ref_build(coo, bs=16, row_owned=1) -> dict | None:
    lib = ref_lib(bs, row_owned)
    if lib is None:
        return None
    row, col, val = _coo_arrays(coo)
    h = lib.cbdump_build(coo.m, coo.n, coo.nnz, _ptr(row), _ptr(col), _ptr(val))
    return dump(lib, h)


def oracle_build(coo, bs=16, row_owned=1, waves=4, dense_sixteenths=15,
                 force_coo64=0) -> dict:
    lib = oracle_lib()
    row, col, val = _coo_arrays(coo)
    h = lib.oracle_build(bs, row_owned, waves, dense_sixteenths, force_coo64,
                         coo.m, coo.n, coo.nnz, _ptr(row), _ptr(col), _ptr(val))
    assert h, "oracle_build rejected the options"
    return dump(lib, h)


def compare_dumps(a: dict, b: dict, what: str = "") -> None:
    """Asserts two dumps are identical: integers and payload bit for bit;
    the two load-stddev statistics to 1e-12 relative (the reference computes
    them with -ffast-math sums)."""
    for k in SCALARS:
        assert a[k] == b[k], f"{what}: scalar {k}: {a[k]} != {b[k]}"
    assert a["super_sparse_ratio"] == b["super_sparse_ratio"], what
    for k in ("load_stddev_before", "load_stddev_after"):
        assert np.isclose(a[k], b[k], rtol=1e-12, atol=0), f"{what}: {k}"
    for k in DTYPES:
        x, y = a[k], b[k]
        assert x.shape == y.shape, f"{what}: {k} length {x.shape} != {y.shape}"
        if k == "pay_f64":
            ok = np.array_equal(x.view(np.uint64), y.view(np.uint64))
        else:
            ok = np.array_equal(x, y)
        if not ok:
            bad = np.flatnonzero(x != y)[:5] if x.dtype != np.float64 else \
                np.flatnonzero(x.view(np.uint64) != y.view(np.uint64))[:5]
            raise AssertionError(f"{what}: {k} differs at {bad}: "
                                 f"{x[bad]} vs {y[bad]}")


def oracle_spmv(coo, x) -> np.ndarray:
    """The reference's serial COO loop (utils.h:98-111), FP64, input order."""
    lib = oracle_lib()
    row, col, val = _coo_arrays(coo)
    x = np.ascontiguousarray(x, np.float64)
    y = np.zeros(coo.m, np.float64)
    lib.oracle_spmv_coo(coo.m, coo.nnz, _ptr(row), _ptr(col), _ptr(val),
                        _ptr(x), _ptr(y))
    return y


def oracle_spmm_ld(coo, x, transpose=False):
    """(Y, absrow) in long double; x is (nrhs, n) row-major == column-major
    n x nrhs.  With transpose=True computes A^T g for g of shape (nrhs, m)."""
    lib = oracle_lib()
    row, col, val = _coo_arrays(coo)
    x = np.ascontiguousarray(np.atleast_2d(x), np.float64)
    nrhs = x.shape[0]
    out_dim = coo.n if transpose else coo.m
    y = np.zeros((nrhs, out_dim), np.float64)
    ab = np.zeros((nrhs, out_dim), np.float64)
    fn = lib.oracle_spmm_t_coo_ld if transpose else lib.oracle_spmm_coo_ld
    fn(out_dim, coo.nnz, _ptr(row), _ptr(col), _ptr(val), nrhs, _ptr(x),
       x.shape[1], _ptr(y), out_dim, _ptr(ab))
    return y, ab


def oracle_grad_vals(coo, g, x) -> np.ndarray:
    lib = oracle_lib()
    row, col, _ = _coo_arrays(coo)
    g = np.ascontiguousarray(np.atleast_2d(g), np.float64)
    x = np.ascontiguousarray(np.atleast_2d(x), np.float64)
    out = np.zeros(coo.nnz, np.float64)
    lib.oracle_grad_vals(coo.nnz, _ptr(row), _ptr(col), g.shape[0], _ptr(g),
                         g.shape[1], _ptr(x), x.shape[1], _ptr(out))
    return out


def decode_spmv(d: dict, bs: int, x) -> np.ndarray:
    """y from a CB dump, reading every encoding as the device kernels do."""
    lib = oracle_lib()
    x = np.ascontiguousarray(x, np.float64)
    y = np.zeros(d["m"], np.float64)
    arrs = [d[k] for k in ("gb_row_idx", "gb_col_idx", "nnz_per_blk",
                           "type_per_blk", "block_cols_offset", "block_cols",
                           "pay_u32", "pay_u32_off", "pay_f64", "pay_f64_off")]
    rc = lib.oracle_cb_decode_spmv(bs, d["m"], d["gb_nnzb"], d["gather_flag"],
                                   d["direct_coo_columns"],
                                   d["compact_coo_indices"],
                                   *[_ptr(a) for a in arrs], _ptr(x), _ptr(y))
    assert rc == 0
    return y


def ref_check(coo, x, y, bs=16) -> bool | None:
    """The reference's own check_results_consistency (utils.h:85-136) on y."""
    lib = ref_lib(bs, 1)
    if lib is None:
        return None
    row, col, val = _coo_arrays(coo)
    x = np.ascontiguousarray(x, np.float64)
    y = np.ascontiguousarray(y, np.float64)
    ctx = lib.cbref_spmv_prepare(coo.m, coo.n, coo.nnz, _ptr(row), _ptr(col),
                                 _ptr(val), _ptr(x))
    lib.cbref_spmv_set_y(ctx, _ptr(y))
    ok = lib.cbref_spmv_check(ctx)
    lib.cbref_spmv_free(ctx)
    return bool(ok)


def have_ref() -> bool:
    return ref_lib(16, 1) is not None and os.environ.get("CB_NO_REF") != "1"
