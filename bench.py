"""CB-SpMV benchmark (one JSON line on rank 0).

Workload (the configuration the headline metric is quoted on): plain
CB-SpMV, FP64, on the power-law matrix n = 2^20 (row lengths power-law with
exponent 2.1 in [1, 20000], mean 16 nnz/row; 70% of columns within +-4096 of
the diagonal, 30% uniform; values N(0,1); seed 1), 16x16 blocks.  Synthetic
and seeded.  A step is one y = A x over the whole matrix.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

value       algorithmic GB/s of the whole job: the bytes of the packed CB
            matrix the kernel must read (descriptors + payload, no padding),
            x read once and y written once, divided by the device time of a
            step (CUDA events, max over ranks); inputs resident in HBM.
e2e         the same metric through the C ABI with host buffers
            (cbspmv_spmv_host_async: pinned x copied in, y copied out every
            step; consecutive steps overlap copy in, kernel and copy out).
roofline    the kernel of the one launch of a step (the row-segment stream
            kernel: every block of this matrix is a COO block) against the
            measured HBM copy bandwidth; traffic = its DRAM bytes per launch
            from the committed ncu summary (profiles/).
cpu_baseline  the reference's own CPU SpMV (utils.h:98-111, compiled from its
            headers into oracle/_ref) on a bounded sample, 1 thread as written.
configs     the other workloads (LAP, PL FP32, PL unit values, PL built with
            row_owned = 0 (balanced schedule beside row-owned), ST FP64/FP32,
            DIFF forward and adjoint with 8 right-hand sides, BAT 512-matrix
            batch), each timed on the device with its roofline fraction and
            checked against the oracle (--configs none skips).
comparator  cuSPARSE CSR SpMV (and BSR, block sizes 2-16, the analogue of
            the reference's hipSPARSE BSR baseline) on the same matrix.
--impl reference   times that CPU SpMV as the reference arm (rank 0 only).

Multi-GPU: every rank runs its own copy of the workload (replicas; SpMV of
one matrix needs no exchange), weak scaling, timed as the max over ranks.
--mode shard instead splits the one matrix over the ranks by block rows
(cbspmv.shard.RowShard, x all-gathered over NCCL inside every step), strong
scaling: the whole matrix's algorithmic bytes over the slowest rank's time.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import pathlib
import re
import statistics
import subprocess
import sys
import tempfile
import time

REPO = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(REPO / "cb-sparse-dcu_b200"))

METRIC = "SpMV GB/s (algorithmic CB bytes / t), plain CB-SpMV FP64, power-law n=2^20"
# Algorithmic bytes of one SpMV of the headline workload in this library's
# layout (cbspmv_info.algorithmic_bytes: tile descriptors, COO indices and
# values without padding, x once, y once).  The reference arm divides by the
# same count without loading the product library; a CPU test checks that the
# library reports this number.
PL_FP64_ALG_BYTES = 221776532
UNIT = "GB/s"
WORKLOAD = ("power-law n=2^20, alpha 2.1, lengths [1,20000], mean 16 nnz/row, "
            "70% within +-4096 of diagonal, N(0,1) values, seed 1; FP64; 16x16 blocks")


def _peaks():
    try:
        d = json.loads((REPO / "MEASURED_PEAKS.json").read_text())
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def _ncu_traffic(kernel: str):
    """DRAM bytes per launch of `kernel` on the PL FP64 workload from the
    committed ncu summaries (profiles/), or None."""
    pat = r"dram_bytes_per_launch_pl_fp64\[" + re.escape(kernel) + r"\]\s*=\s*([0-9.eE+]+)"
    for p in sorted((REPO / "profiles").glob("*.md")):
        m = re.search(pat, p.read_text())
        if m:
            return float(m.group(1))
    return None


class Clocks:
    """Samples SM clocks and throttle reasons with nvidia-smi while running."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        tmp = pathlib.Path(tempfile.mkdtemp(prefix="cbspmv_clocks_"))
        self.path = tmp / f"clocks_rank{index}.csv"
        self.err = tmp / f"clocks_rank{index}.err"
        self.gpu = str(index)
        try:  # the device as nvidia-smi names it (CUDA_VISIBLE_DEVICES may remap)
            import torch
            uuid = str(torch.cuda.get_device_properties(index).uuid)
            if uuid:
                self.gpu = uuid if uuid.startswith("GPU-") else "GPU-" + uuid
        except Exception:
            pass

    def __enter__(self):
        try:
            self.path.parent.mkdir(exist_ok=True)
            self.f = open(self.path, "w")
            self.ferr = open(self.err, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}",
                 "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,"
                 "clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
                 "clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,"
                 "clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=self.f, stderr=self.ferr)
            # start timing only once sampling runs (nvidia-smi needs ~1 s)
            t0 = time.time()
            while time.time() - t0 < 10 and self.proc.poll() is None:
                if self.path.stat().st_size > 0:
                    break
                time.sleep(0.05)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()
            self.ferr.close()

    def summary(self):
        if not self.path.exists():
            return None
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                 "sw_power_cap"]
        for line in self.path.read_text().splitlines():
            f = [v.strip() for v in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def _timed(fn, reps: int, warmup: int, flush=None):
    """Mean device time (ms) of fn over reps runs after warmup runs, CUDA
    events on the current stream around each run; flush(), when given, runs
    before each timed run outside the events (an L2 flush for workloads that
    fit in L2)."""
    import torch
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    total = 0.0
    for _ in range(reps):
        if flush is not None:
            flush()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        e1.synchronize()
        total += e0.elapsed_time(e1)
    return total / reps


def _oracle():
    """The CPU oracle (test infrastructure: the checker of every result the
    bench reports, never the thing timed)."""
    sys.path.insert(0, str(REPO / "tests"))
    import cbdump as cd
    return cd


def _parity(y, yref, ab, f32) -> dict:
    """Error of a result against the long-double oracle.  y, yref, ab:
    (nrhs, rows); ab = sum_k |a_ik x_kj| per row.  max_err_rowscaled =
    max |y - yref| / ab (the tests' bound: <= 1e-12 FP64, <= 1e-5 FP32);
    for FP32 the plain errors against the FP64 oracle are stated too."""
    import numpy as np
    y = np.asarray(y, np.float64)
    d = np.abs(y - yref)
    tol = 1e-5 if f32 else 1e-12
    err = float(np.max(d / (ab + 1e-300))) if d.size else 0.0
    out = {"max_err_rowscaled": float(f"{err:.3g}"), "tol": tol, "pass": bool(err <= tol)}
    if f32:
        ymax = float(np.max(np.abs(yref))) if yref.size else 0.0
        dmax = float(np.max(d)) if d.size else 0.0
        out["fp32_vs_fp64_oracle"] = {
            "max_abs_err": float(f"{dmax:.3g}"),
            "max_abs_err_over_max_abs_y": float(f"{(dmax / ymax) if ymax else 0.0:.3g}")}
    return out


def secondary_configs(dev, peak: float, want=("lap", "pl32", "st", "diff", "bat"),
                      bat_count: int = 512) -> dict:
    """The other workloads of the benchmark suite, each timed on the device
    and each result checked against the oracle at its full size (outside the
    timed region): LAP (5-point Laplacian 256^2, FP64), PL in FP32, PL with
    unit values (the value-free payload the reference uses for its
    unit-valued inputs), ST (27-point x 3 dof stencil on 64^3, FP64 and FP32),
    DIFF (power-law n = 2^18, 8 right-hand sides, FP32: forward, adjoint A^T G
    and the value gradient) and BAT (512 uneven FP32 matrices with 1-16
    right-hand sides: the batched launch, its CUDA graph, one launch per
    matrix, and a graph of those).  Every plan is autotuned first
    (cbspmv_autotune).  Algorithmic bytes: the packed matrix the kernel must
    read, x and y once per right-hand side."""
    import numpy as np
    import torch
    import cbspmv
    from cbspmv import gen
    cd = _oracle()

    l2_flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    flush = lambda: l2_flush.zero_()  # noqa: E731
    out = {}

    def single(name, coo, f32, reps=50, bsr=False):
        plan = cbspmv.Plan(coo, value_type=int(f32))
        kernel, _ = plan.autotune(1)
        dt = torch.float32 if f32 else torch.float64
        xh = gen.uniform_x(coo.n, 0)
        if f32:
            xh = xh.astype(np.float32).astype(np.float64)  # the x the GPU sees
        x = torch.from_numpy(xh).to(dev, dt)
        y = torch.empty(coo.m, dtype=dt, device=dev)
        info = plan.info()
        small = info["device_bytes"] < (200 << 20)
        ms = _timed(lambda: plan.spmv(x, y), reps, 5, flush if small else None)
        plan.check()
        yref, ab = cd.oracle_spmm_ld(coo, xh[None, :])
        alg = info["algorithmic_bytes"]
        out[name] = {"nnz": coo.nnz, "kernel": kernel, "ms": round(ms, 4),
                     "gbs": round(alg / ms / 1e6, 1), "gflops": round(2 * coo.nnz / ms / 1e6, 1),
                     "frac": round(alg / ms / 1e6 / peak, 4),
                     "parity": _parity(y.cpu().numpy()[None, :], yref, ab, f32),
                     "l2": "flushed before each step" if small else "inputs larger than L2"}
        del plan
        if bsr and not f32:
            try:
                c = bsr_comparator(coo, xh, dev)
                if c["ms"]:
                    c["this_library_speedup"] = round(c["ms"] / ms, 2)
                out[name]["comparator_bsr"] = c
            except Exception as exc:  # the comparator is informative only
                out[name]["comparator_bsr"] = {"unavailable": str(exc)[:200]}

    if "lap" in want:
        single("LAP fp64 (256^2 5-point)", gen.laplacian_2d(), False)
    if "pl32" in want:
        single("PL fp32 (n=2^20)", gen.power_law(), True)
    if "unit" in want:  # the reference's own matrices are unit-valued (its reader sets 1.0)
        pl = gen.power_law()
        single("PL fp64 unit values (value-free payload)",
               gen.Coo(pl.m, pl.n, pl.row, pl.col, np.ones(pl.nnz)), False)
        del pl
    if "bal" in want:  # the balanced schedule (the reference's load-balance ablation)
        try:
            balanced_config(dev, peak, out)
        except Exception as exc:  # informative only: never breaks the bench line
            out["PL fp64 balanced (row_owned = 0)"] = {"unavailable": str(exc)[:200]}
    if "st" in want:
        st = gen.stencil_27pt()
        single("ST fp64 (64^3 x 3 dof 27-point)", st, False, reps=20, bsr=True)
        single("ST fp32 (64^3 x 3 dof 27-point)", st, True, reps=20)
        del st
    if "diff" in want:
        diff_config(dev, peak, flush, out)
    if "bat" in want:
        bat_config(dev, peak, bat_count, out)
    return out


def balanced_config(dev, peak, out):
    """PL FP64 built with row_owned = 0: the balanced schedule (kernel 6:
    the entries in the reference's balanced block order, added into y with
    atomics, as its non-row-owned mode) beside the same plan's row-owned
    kernel (kernel 5), each checked against the oracle."""
    import numpy as np
    import torch
    import cbspmv
    from cbspmv import gen
    cd = _oracle()
    coo = gen.power_law()
    xh = gen.uniform_x(coo.n, 0)
    x = torch.from_numpy(xh).to(dev)
    yref, ab = cd.oracle_spmm_ld(coo, xh[None, :])
    r = {"nnz": coo.nnz, "l2": "inputs larger than L2", "parity": {}}
    for kernel, name in ((6, "balanced"), (5, "row_owned_stream")):
        plan = cbspmv.Plan(coo, row_owned=0, kernel=kernel)
        y = torch.empty(coo.m, dtype=torch.float64, device=dev)
        alg = plan.info()["algorithmic_bytes"]
        ms = _timed(lambda: plan.spmv(x, y), 100, 5)
        plan.check()
        r[name + "_ms"] = round(ms, 4)
        r[name + "_gbs"] = round(alg / ms / 1e6, 1)
        r[name + "_frac"] = round(alg / ms / 1e6 / peak, 4)
        r["parity"][name] = _parity(y.cpu().numpy()[None, :], yref, ab, False)
        r["load_stddev_before_after"] = [round(plan.info()["load_stddev_before"], 2),
                                         round(plan.info()["load_stddev_after"], 2)]
        del plan
    out["PL fp64 balanced (row_owned = 0)"] = r


def _cusparse():
    """The cuSPARSE library torch loads (a comparator only)."""
    import torch
    here = pathlib.Path(torch.__file__).parent.parent / "nvidia" / "cusparse" / "lib"
    for cand in (here / "libcusparse.so.12", "libcusparse.so.12"):
        try:
            return ctypes.CDLL(str(cand))
        except OSError:
            continue
    raise OSError("libcusparse.so.12 not found")


def bsr_comparator(coo, xh, dev, sizes=(2, 4, 8, 16)):
    """cuSPARSE BSR SpMV on the same matrix, FP64: the analogue of the
    reference's hipSPARSE BSR baseline (cb-spmv-dcu/benchmark/hipSparse-bsr/
    main.hip.cpp:99-187): CSR converted to BSR on the device (csr2bsr,
    row-major blocks) for block sizes 2, 4, 8 and 16, each timed with bsrmv,
    the fastest reported.  Its y is checked against the oracle's."""
    import numpy as np
    import torch
    cd = _oracle()
    lib = _cusparse()
    P, I = ctypes.c_void_p, ctypes.c_int
    lib.cusparseCreate.argtypes = [ctypes.POINTER(P)]
    lib.cusparseSetStream.argtypes = [P, P]
    lib.cusparseCreateMatDescr.argtypes = [ctypes.POINTER(P)]
    lib.cusparseDestroyMatDescr.argtypes = [P]
    lib.cusparseDestroy.argtypes = [P]
    lib.cusparseXcsr2bsrNnz.argtypes = [P, I, I, I, P, P, P, I, P, P, ctypes.POINTER(I)]
    lib.cusparseDcsr2bsr.argtypes = [P, I, I, I, P, P, P, P, I, P, P, P, P]
    lib.cusparseDbsrmv.argtypes = [P, I, I, I, I, I, ctypes.POINTER(ctypes.c_double), P, P, P,
                                   P, I, P, ctypes.POINTER(ctypes.c_double), P]
    m, n = coo.m, coo.n
    crow = np.zeros(m + 1, np.int64)
    np.add.at(crow, coo.row.astype(np.int64) + 1, 1)
    crow_d = torch.from_numpy(np.cumsum(crow).astype(np.int32)).to(dev)
    col_d = torch.from_numpy(coo.col.astype(np.int32)).to(dev)
    val_d = torch.from_numpy(coo.val.astype(np.float64)).to(dev)
    yref, ab = cd.oracle_spmm_ld(coo, xh[None, :])
    h, dA, dC = P(), P(), P()
    ok = lambda rc, what: None if rc == 0 else (_ for _ in ()).throw(  # noqa: E731
        RuntimeError(f"{what}: cusparse status {rc}"))
    ok(lib.cusparseCreate(ctypes.byref(h)), "create")
    ok(lib.cusparseSetStream(h, P(torch.cuda.current_stream().cuda_stream)), "stream")
    ok(lib.cusparseCreateMatDescr(ctypes.byref(dA)), "descr")
    ok(lib.cusparseCreateMatDescr(ctypes.byref(dC)), "descr")
    alpha, beta = ctypes.c_double(1.0), ctypes.c_double(0.0)
    per = {}
    try:
        for bd in sizes:
            mb, nb = (m + bd - 1) // bd, (n + bd - 1) // bd
            xp = torch.zeros(nb * bd, dtype=torch.float64, device=dev)
            xp[:n] = torch.from_numpy(xh).to(dev)
            yp = torch.empty(mb * bd, dtype=torch.float64, device=dev)
            rowp = torch.empty(mb + 1, dtype=torch.int32, device=dev)
            nnzb = I(0)
            ok(lib.cusparseXcsr2bsrNnz(h, 0, m, n, dA, P(crow_d.data_ptr()), P(col_d.data_ptr()),
                                       bd, dC, P(rowp.data_ptr()), ctypes.byref(nnzb)), "nnz")
            torch.cuda.synchronize()
            nbytes = nnzb.value * bd * bd * 8
            if nnzb.value * bd * bd >= 2**31 - 1 or nbytes > (48 << 30):
                # the legacy BSR routines index values with 32-bit ints
                per[bd] = {"skipped": f"{nnzb.value} blocks: {nnzb.value * bd * bd} values, "
                                      "beyond the library's 32-bit value index"}
                continue
            colb = torch.empty(max(nnzb.value, 1), dtype=torch.int32, device=dev)
            valb = torch.empty(max(nnzb.value * bd * bd, 1), dtype=torch.float64, device=dev)
            ok(lib.cusparseDcsr2bsr(h, 0, m, n, dA, P(val_d.data_ptr()), P(crow_d.data_ptr()),
                                    P(col_d.data_ptr()), bd, dC, P(valb.data_ptr()),
                                    P(rowp.data_ptr()), P(colb.data_ptr())), "csr2bsr")

            def mv():
                ok(lib.cusparseDbsrmv(h, 0, 0, mb, nb, nnzb.value, ctypes.byref(alpha), dC,
                                      P(valb.data_ptr()), P(rowp.data_ptr()),
                                      P(colb.data_ptr()), bd, P(xp.data_ptr()),
                                      ctypes.byref(beta), P(yp.data_ptr())), "bsrmv")
            ms = _timed(mv, 50, 5)
            torch.cuda.synchronize()
            err = float(np.max(np.abs(yp[:m].cpu().numpy() - yref[0]) / (ab[0] + 1e-300)))
            per[bd] = {"ms": round(ms, 4), "blocks": nnzb.value,
                       "block_bytes": nbytes, "max_err_rowscaled": float(f"{err:.3g}")}
            del colb, valb, xp, yp, rowp
            torch.cuda.empty_cache()
    finally:
        lib.cusparseDestroyMatDescr(dA)
        lib.cusparseDestroyMatDescr(dC)
        lib.cusparseDestroy(h)
    timed = {k: v for k, v in per.items() if "ms" in v}
    best = min(timed, key=lambda k: timed[k]["ms"]) if timed else None
    return {"library": "cuSPARSE BSR SpMV (csr2bsr + bsrmv, FP64, row-major blocks)",
            "block_sizes": per, "best_block": best,
            "ms": timed[best]["ms"] if best else None}


def diff_config(dev, peak, flush, out):
    """DIFF: Y = A X, then G -> A^T G and the value gradient; every output
    checked against the oracle at full size."""
    import numpy as np
    import torch
    import cbspmv
    from cbspmv import gen
    cd = _oracle()

    coo = gen.power_law(1 << 18, seed=3, mean=24)
    k = 8
    plan = cbspmv.Plan(coo, value_type=1, want_transpose=1)
    kernel, _ = plan.autotune(k)
    Xh = gen.uniform_x(coo.n, 1, nrhs=k).astype(np.float32).astype(np.float64)
    Gh = gen.uniform_x(coo.m, 2, nrhs=k).astype(np.float32).astype(np.float64)
    X = torch.from_numpy(np.ascontiguousarray(Xh.T)).to(dev, torch.float32)
    G = torch.from_numpy(np.ascontiguousarray(Gh.T)).to(dev, torch.float32)
    Y = torch.empty(coo.m, k, device=dev)
    GX = torch.empty(coo.n, k, device=dev)
    GV = torch.empty(plan.num_values(), device=dev)
    GX2 = torch.empty(coo.n, k, device=dev)
    GP = torch.zeros(cbspmv.lib().cbspmv_grad_size_t(plan._h), device=dev)
    info = plan.info()
    xy = 4 * (coo.n + coo.m) * (k - 1)
    fwd_bytes = info["algorithmic_bytes"] + xy
    adj_bytes = fwd_bytes + plan.num_values() * 4 + 4 * (coo.n + coo.m) * k
    t_f = _timed(lambda: plan.spmv(X, Y), 30, 5, flush)
    # the adjoint the autograd backward runs: A^T G and the value gradient
    # per slot of A on a second stream (cbspmv_adjoint); beside it the
    # one-launch form on the transposed layout (cbspmv_adjoint_fused)
    t_a = _timed(lambda: plan.adjoint_fused(G, X, GX2, GP), 30, 5, flush)
    t_a2 = _timed(lambda: plan.adjoint(G, X, GX, GV), 30, 5, flush)
    plan.check()
    yref, ab = cd.oracle_spmm_ld(coo, Xh)
    gref, gab = cd.oracle_spmm_ld(coo, Gh, transpose=True)
    vref = cd.oracle_grad_vals(coo, Gh, Xh)
    vscale = np.sum(np.abs(Gh[:, coo.row] * Xh[:, coo.col]), axis=0)[None, :]
    gv = GV.cpu().numpy().astype(np.float64)[plan.input_slots()][None, :]
    gp = GP.cpu().numpy().astype(np.float64)[plan.grad_positions_t()][None, :]
    out["DIFF fp32 (n=2^18, 8 rhs)"] = {
        "nnz": coo.nnz, "kernel": kernel, "fwd_ms": round(t_f, 4), "adj_ms": round(t_a2, 4),
        "fwd_plus_adj_over_fwd": round((t_f + t_a2) / t_f, 3),
        "adj": "the autograd backward's adjoint: A^T G and the value gradient on two "
               "streams (cbspmv_adjoint)",
        "adj_fused_ms": round(t_a, 4),
        "fwd_plus_adj_fused_over_fwd": round((t_f + t_a) / t_f, 3),
        "fwd_gbs": round(fwd_bytes / t_f / 1e6, 1), "fwd_frac": round(fwd_bytes / t_f / 1e6 / peak, 4),
        "adj_gbs": round(adj_bytes / t_a2 / 1e6, 1),
        "gflops_fwd": round(2 * coo.nnz * k / t_f / 1e6, 1), "l2": "flushed before each step",
        "parity": {"forward": _parity(Y.cpu().numpy().T, yref, ab, True),
                   "adjoint_gx": _parity(GX.cpu().numpy().T, gref, gab, True),
                   "value_gradient": _parity(gv, vref[None, :], vscale, True),
                   "adjoint_gx_fused": _parity(GX2.cpu().numpy().T, gref, gab, True),
                   "value_gradient_fused": _parity(gp, vref[None, :], vscale, True)}}
    del plan
    # library comparator for the forward: cuSPARSE SpMM (CSR, int32 indices)
    try:
        import warnings
        with warnings.catch_warnings():
            warnings.simplefilter("ignore")
            idx = torch.from_numpy(np.stack([coo.row, coo.col]).astype(np.int64))
            A = torch.sparse_coo_tensor(idx, torch.from_numpy(coo.val.astype(np.float32)),
                                        (coo.m, coo.n)).coalesce().to_sparse_csr()
            A = torch.sparse_csr_tensor(A.crow_indices().to(torch.int32),
                                        A.col_indices().to(torch.int32), A.values(),
                                        A.shape).to(dev)
            t_c = _timed(lambda: torch.mm(A, X), 30, 5, flush)
        out["DIFF fp32 (n=2^18, 8 rhs)"]["comparator"] = {
            "library": "cuSPARSE SpMM via torch.mm (CSR, FP32, int32 indices)",
            "fwd_ms": round(t_c, 4), "this_library_speedup": round(t_c / t_f, 2)}
        del A
    except Exception as exc:  # informative only
        out["DIFF fp32 (n=2^18, 8 rhs)"]["comparator"] = {"unavailable": str(exc)[:200]}


def _check_batch(cd, items, xs_h, ys, threads=16) -> dict:
    """Every matrix of a batch against the oracle, on host threads (the
    oracle's C calls release the GIL); the worst matrix's figures."""
    from concurrent.futures import ThreadPoolExecutor
    yh = [y.cpu().numpy() for y in ys]

    def one(k):
        it = items[k]
        yref, ab = cd.oracle_spmm_ld(it.coo, xs_h[k].T)
        return _parity(yh[k].reshape(it.coo.m, it.nrhs).T, yref, ab, True)

    with ThreadPoolExecutor(max_workers=max(1, min(threads, os.cpu_count() or 1))) as ex:
        res = list(ex.map(one, range(len(items))))
    worst = max(range(len(res)), key=lambda k: res[k]["max_err_rowscaled"])
    out = dict(res[worst])
    out["checked_matrices"] = len(res)
    out["pass"] = all(r["pass"] for r in res)
    out["worst_matrix"] = worst
    return out


def bat_config(dev, peak, count, out):
    """BAT: `count` uneven FP32 matrices (512 is the workload); each mode's
    results checked against the oracle, every matrix."""
    import numpy as np
    import torch
    import cbspmv
    from cbspmv import gen
    cd = _oracle()
    items = gen.batch_uneven(count=count)
    plans = [cbspmv.Plan(it.coo, value_type=1) for it in items]
    rng = np.random.default_rng(40)
    xs_h = [rng.uniform(-1, 1, (it.coo.n, it.nrhs)).astype(np.float32).astype(np.float64)
            for it in items]
    xs = [torch.from_numpy(x).to(dev, torch.float32) for x in xs_h]
    ys = [torch.empty(it.coo.m, it.nrhs, device=dev) for it in items]
    b = cbspmv.Batch(plans, [it.nrhs for it in items]).bind(xs, ys)
    alg = sum(p.info()["algorithmic_bytes"] + 4 * (it.coo.n + it.coo.m) * (it.nrhs - 1)
              for p, it in zip(plans, items))
    r = {"matrices": len(items), "nnz": sum(it.coo.nnz for it in items), "algorithmic_bytes": alg,
         "parity": {}}
    for name, fn in (("batched", b.run), ("batched_graph", lambda: b.graph_launch(False)),
                     ("per_matrix", b.run_each), ("per_matrix_graph", lambda: b.graph_launch(True))):
        for y in ys:
            y.fill_(float("nan"))
        ms = _timed(fn, 5, 3)
        torch.cuda.synchronize()
        r[name + "_ms"] = round(ms, 3)
        r[name + "_gbs"] = round(alg / ms / 1e6, 1)
        r["parity"][name] = _check_batch(cd, items, xs_h, ys)
    r["batched_frac"] = round(r["batched_gbs"] / peak, 4)
    r["batched_over_per_matrix"] = round(r["per_matrix_ms"] / r["batched_ms"], 2)
    r["batched_graph_over_per_matrix"] = round(r["per_matrix_ms"] / r["batched_graph_ms"], 2)
    r["l2"] = "inputs larger than L2"
    out[f"BAT fp32 ({len(items)} matrices, 1-16 rhs)"] = r
    b.close()


def _dist():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def _ref_cpu(coo, x, seconds: float, max_reps: int):
    """Times the reference's check_results_consistency (its whole CPU SpMV)
    on the full matrix; returns (seconds per SpMV, kind, reps)."""
    import numpy as np
    sys.path.insert(0, str(REPO / "tests"))
    import cbdump as cd  # the oracle/_ref loader (checker only)
    lib = cd.ref_lib(16, 1)
    row, col, val = (np.ascontiguousarray(a) for a in (coo.row, coo.col, coo.val))
    xv = np.ascontiguousarray(x, np.float64)
    if lib is not None:
        P = ctypes.c_void_p
        ctx = lib.cbref_spmv_prepare(coo.m, coo.n, coo.nnz, row.ctypes.data_as(P),
                                     col.ctypes.data_as(P), val.ctypes.data_as(P),
                                     xv.ctypes.data_as(P))
        y = cd.oracle_spmv(coo, xv)
        lib.cbref_spmv_set_y(ctx, y.ctypes.data_as(P))
        run = lambda: lib.cbref_spmv_check(ctx)  # noqa: E731
        kind = "reference"
    else:
        run = lambda: cd.oracle_spmv(coo, xv)  # noqa: E731
        kind = "port"
    run()
    reps, t0 = 0, time.perf_counter()
    while reps < max_reps and (time.perf_counter() - t0 < seconds or reps < 2):
        run()
        reps += 1
    dt = (time.perf_counter() - t0) / reps
    if lib is not None:
        lib.cbref_spmv_free(ctx)
    return dt, kind, reps


def _row_prefix(coo, nnz_target: int):
    """The first rows of coo holding about nnz_target nonzeros (a bounded
    sample with the workload's row distribution)."""
    import numpy as np
    k = int(min(coo.nnz, max(1, nnz_target)))
    rows = int(coo.row[k - 1]) + 1
    k = int(np.searchsorted(coo.row, rows))
    return type(coo)(rows, coo.n, coo.row[:k], coo.col[:k], coo.val[:k])


def reference_arm(args, budget_s: float = 150.0):
    world, rank, _ = _dist()
    if rank != 0:
        return
    sys.path.insert(0, str(REPO / "cb-sparse-dcu_b200" / "cbspmv"))
    import gen  # the workload generator alone (numpy), not the product library
    coo = gen.power_law()
    x = gen.uniform_x(coo.n, 0)
    alg = PL_FP64_ALG_BYTES  # the same metric's byte count as the GPU arm
    # size each step so that warm-up + timed steps fit the time budget
    t_full, kind, _ = _ref_cpu(coo, x, 0.0, 1)
    frac = min(1.0, budget_s / max(1, args.steps + args.warmup) / t_full)
    sample = _row_prefix(coo, int(frac * coo.nnz)) if frac < 1.0 else coo
    share = sample.nnz / coo.nnz
    _ref_cpu(sample, x, 0.0, max(1, args.warmup))
    dt, kind, reps = _ref_cpu(sample, x, 1e9, max(1, args.steps))
    value = alg * share / dt / 1e9
    desc = (f"{reps} steps, each the reference's CPU SpMV (check_results_consistency, "
            f"utils.h:85-136, serial as written) over the first {sample.m} rows "
            f"({sample.nnz} nnz, {share:.4f} of the workload); a full SpMV takes "
            f"{t_full * 1e3:.1f} ms")
    line = {
        "impl": "reference", "metric": METRIC, "value": round(value, 3), "unit": UNIT,
        "n_gpus": world, "steps": reps, "warmup": args.warmup,
        "ms_per_step": round(dt * 1e3, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded)",
        "config": {"workload": WORKLOAD, "nnz": coo.nnz, "algorithmic_bytes": alg,
                   "parallelism": "rank 0 only (CPU)"},
        "cpu_baseline": {"value": round(value, 3), "unit": UNIT, "cores": 1, "kind": kind,
                         "sample": desc},
        "e2e": {"value": round(value, 3), "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def shard_arm(args):
    """--mode shard: the headline matrix split over the N ranks by block rows
    (cbspmv.shard.RowShard: each rank its rows' plan, x all-gathered over
    NCCL inside every step), strong scaling: value = the whole matrix's
    algorithmic bytes / the slowest rank's step time."""
    import numpy as np
    import torch
    import torch.distributed as dist
    import cbspmv
    from cbspmv import gen, shard
    from cbspmv.dist import Group
    world, rank, local = _dist()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pg = Group("nccl", dev)
    coo = gen.power_law()
    x_host = gen.uniform_x(coo.n, 0)
    sh = shard.RowShard(coo, world, rank)
    plans = [p for p in (sh.full, sh.own, sh.halo) if p is not None]
    alg_rank = sum(p.info()["algorithmic_bytes"] for p in plans)
    x_own = torch.from_numpy(x_host[sh.c0:sh.c1].copy()).to(dev)
    y = torch.empty(sh.r1 - sh.r0, dtype=torch.float64, device=dev)
    sh.spmv(x_own, y)  # correctness gate: this rank's rows
    torch.cuda.synchronize()
    sys.path.insert(0, str(REPO / "tests"))
    import cbdump as cd
    yref, ab = cd.oracle_spmm_ld(coo, x_host[None, :])
    err = float(np.max(np.abs(y.cpu().numpy() - yref[0][sh.r0:sh.r1]) /
                       (ab[0][sh.r0:sh.r1] + 1e-300))) if sh.r1 > sh.r0 else 0.0
    if pg.max(err) > 1e-12:
        raise SystemExit(f"bench: sharded SpMV error {err:.3g} above 1e-12")
    alg = alg_rank
    if world > 1:
        t = torch.tensor([float(alg_rank)], dtype=torch.float64, device=dev)
        dist.all_reduce(t)
        alg = int(t.item())
    for _ in range(args.warmup):
        sh.spmv(x_own, y)
    launches0 = cbspmv.launch_count()
    pg.barrier()
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        sh.spmv(x_own, y)
    ev1.record(stream)
    torch.cuda.synchronize()
    launches = cbspmv.launch_count() - launches0
    ms = pg.max(ev0.elapsed_time(ev1) / args.steps)
    if rank == 0:
        line = {
            "metric": METRIC, "value": round(alg / (ms * 1e-3) / 1e9, 2), "unit": UNIT,
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(ms, 5), "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            "mode": "shard",
            "config": {"workload": WORKLOAD, "nnz": coo.nnz, "algorithmic_bytes": alg,
                       "parallelism": f"block-row shards x{world}, x all-gathered (NCCL)",
                       "x_piece_bytes": sh.L * 8, "l2": "inputs larger than L2 at N=1"},
            "gpu_launches": launches,
        }
        print(json.dumps(line), flush=True)
    pg.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10000)
    ap.add_argument("--warmup", type=int, default=50)
    ap.add_argument("--impl", default="cbspmv", choices=["cbspmv", "reference"])
    ap.add_argument("--mode", default="replicas", choices=["replicas", "shard"],
                    help="N > 1: every rank its own copy of the headline SpMV (replicas, "
                         "weak scaling; the default) or one matrix split by block rows "
                         "(shard, strong scaling)")
    ap.add_argument("--e2e-steps", type=int, default=300)
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--configs", default="all",
                    help="other workloads to time (rank 0, N=1 only): all, none, or a "
                         "comma list of lap,pl32,unit,bal,st,diff,bat")
    ap.add_argument("--bat-count", type=int, default=512,
                    help="matrices in the BAT batch (512 is the workload; fewer for "
                         "profiling captures)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        reference_arm(args)
        return
    if args.mode == "shard":
        shard_arm(args)
        return

    import numpy as np
    import torch
    import cbspmv
    from cbspmv import gen

    from cbspmv.dist import Group
    world, rank, local = _dist()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pg = Group("nccl", dev)

    coo = gen.power_law()
    x_host = gen.uniform_x(coo.n, 0)
    plan = cbspmv.Plan(coo)
    info = plan.info()
    alg = info["algorithmic_bytes"]
    x = torch.from_numpy(x_host).to(dev)
    y = torch.empty(coo.m, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream()

    # correctness gate: the bench does not report a wrong kernel
    plan.spmv(x, y)
    torch.cuda.synchronize()
    sys.path.insert(0, str(REPO / "tests"))
    import cbdump as cd
    yref, ab = cd.oracle_spmm_ld(coo, x_host[None, :])
    err = float(np.max(np.abs(y.cpu().numpy() - yref[0]) / (ab[0] + 1e-300)))
    if err > 1e-12:
        raise SystemExit(f"bench: SpMV error {err:.3g} above 1e-12")

    for _ in range(args.warmup):
        plan.spmv(x, y)
    launches0 = cbspmv.launch_count()
    pg.barrier()
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    with Clocks(local) as clk:
        ev0.record(stream)
        for _ in range(args.steps):
            plan.spmv(x, y)
        ev1.record(stream)
        torch.cuda.synchronize()
    pg.barrier()
    launches = cbspmv.launch_count() - launches0
    ms = pg.max(ev0.elapsed_time(ev1) / args.steps)
    value = world * alg / (ms * 1e-3) / 1e9
    gflops = world * 2.0 * coo.nnz / (ms * 1e-3) / 1e9

    # end to end through the C ABI with host buffers (pinned)
    xp = torch.from_numpy(x_host).pin_memory()
    yp = torch.empty(coo.m, dtype=torch.float64).pin_memory()
    lib = cbspmv.lib()
    P = ctypes.c_void_p
    sptr = P(stream.cuda_stream)
    for _ in range(3):
        lib.cbspmv_spmv_host_async(plan._h, P(xp.data_ptr()), P(yp.data_ptr()), 1, sptr)
    pg.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.e2e_steps):
        rc = lib.cbspmv_spmv_host_async(plan._h, P(xp.data_ptr()), P(yp.data_ptr()), 1, sptr)
        if rc:
            raise SystemExit(f"spmv_host_async failed: {cbspmv.last_error()}")
    e1.record(stream)  # after every step's copy out (the stream waits for each)
    torch.cuda.synchronize()
    # the last step's y, read back through the pipeline, is the oracle's
    err_e2e = float(np.max(np.abs(yp.numpy() - yref[0]) / (ab[0] + 1e-300)))
    if err_e2e > 1e-12:
        raise SystemExit(f"bench: pipelined host SpMV error {err_e2e:.3g} above 1e-12")
    ms_e2e = pg.max(e0.elapsed_time(e1) / args.e2e_steps)
    e2e_value = world * alg / (ms_e2e * 1e-3) / 1e9

    peak, peak_kind = _peaks()
    kname = "cb_rowseg_kernel" if plan.info()["rowseg_bytes"] > 0 else "cb_spmv_stream_kernel"
    achieved = alg / (ms * 1e-3) / 1e9
    roof = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
            "frac": round(achieved / peak, 4), "peak_source": peak_kind,
            "traffic": _ncu_traffic(kname),
            "kernel": f"{kname} (the one launch of each SpMV)"}

    # library comparator: cuSPARSE CSR SpMV (through torch) on the same matrix
    comparator = None
    if rank == 0:
        try:
            import warnings
            crow = np.zeros(coo.m + 1, np.int64)
            np.add.at(crow, coo.row.astype(np.int64) + 1, 1)
            with warnings.catch_warnings():
                warnings.simplefilter("ignore")
                A = torch.sparse_csr_tensor(
                    torch.from_numpy(np.cumsum(crow).astype(np.int32)).to(dev),
                    torch.from_numpy(coo.col.astype(np.int32)).to(dev),
                    torch.from_numpy(coo.val).to(dev), (coo.m, coo.n))
            xs = x.view(-1, 1)
            ms_cs = _timed(lambda: torch.sparse.mm(A, xs), 200, 10)
            csr_bytes = coo.nnz * (4 + 8) + (coo.m + 1) * 4 + (coo.n + coo.m) * 8
            comparator = {"library": "cuSPARSE CSR SpMV via torch.sparse.mm (FP64, int32 indices)",
                          "ms": round(ms_cs, 4), "csr_bytes": csr_bytes,
                          "csr_gbs": round(csr_bytes / ms_cs / 1e6, 1),
                          "this_library_speedup": round(ms_cs / ms, 2)}
            del A
        except Exception as exc:  # the comparator is informative only
            comparator = {"unavailable": str(exc)[:200]}
    # and cuSPARSE BSR (the reference's own library baseline is hipSPARSE BSR)
    if rank == 0 and world == 1 and args.configs != "none":
        try:
            cb = bsr_comparator(coo, x_host, dev)
            if cb["ms"]:
                cb["this_library_speedup"] = round(cb["ms"] / ms, 2)
            comparator = {"csr": comparator, "bsr": cb}
        except Exception as exc:
            comparator = {"csr": comparator, "bsr": {"unavailable": str(exc)[:200]}}

    line = None
    configs = None
    if rank == 0 and world == 1 and args.configs != "none":
        want = {"lap", "pl32", "unit", "bal", "st", "diff", "bat"} if args.configs == "all" \
            else set(args.configs.split(","))
        configs = secondary_configs(dev, peak, want, args.bat_count)
    if rank == 0:
        cpu_dt, kind, reps = _ref_cpu(coo, x_host, args.cpu_seconds, 400)
        cpu = {"value": round(alg / cpu_dt / 1e9, 3), "unit": UNIT, "cores": 1, "kind": kind,
               "host_cores": os.cpu_count(),
               "sample": f"{reps} full SpMVs of the workload on 1 host thread "
                         "(check_results_consistency, utils.h:85-136, serial as written) "
                         f"on a host with {os.cpu_count()} cores",
               "ms_per_spmv": round(cpu_dt * 1e3, 3)}
        line = {
            "metric": METRIC, "value": round(value, 2), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 5),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic (seeded power-law matrix, x ~ U[-1,1])",
            "config": {"workload": WORKLOAD, "nnz": coo.nnz, "m": coo.m,
                       "algorithmic_bytes": alg, "device_bytes": info["device_bytes"],
                       "tiles": info["tiles"], "coo_blocks": info["coo_blocks"],
                       "gather": info["gather_flag"],
                       "l2": "inputs larger than L2 (packed matrix > 126 MB)",
                       "parallelism": f"replicas x{world}"},
            "gflops": round(gflops, 2),
            "e2e": {"value": round(e2e_value, 3), "unit": UNIT,
                    "h2d_bytes_per_step": coo.n * 8, "d2h_bytes_per_step": coo.m * 8,
                    "ms_per_step": round(ms_e2e, 4)},
            "roofline": roof,
            "cpu_baseline": cpu,
            "gpu_launches": launches,
            "comparator": comparator,
            "clocks": clk.summary(),
        }
        if configs is not None:
            line["configs"] = configs
            flags = []

            def collect(d):
                if isinstance(d, dict):
                    if "pass" in d and "max_err_rowscaled" in d:
                        flags.append(bool(d["pass"]))
                    for v in d.values():
                        collect(v)
            collect(configs)
            line["parity"] = {"headline_max_err_rowscaled": float(f"{err:.3g}"),
                              "configs_checked": len(flags), "all_pass": all(flags)}
    pg.close()
    if line:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
