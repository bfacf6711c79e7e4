"""GPU parity of the row-segment stream (kernel 5, the automatic choice for
one right-hand side when every block is a COO block) against the oracle.

Tolerance as in test_gpu_spmv: per row, |y - y_ref| <= tol * sum |a x|,
tol = 1e-12 FP64, 1e-5 FP32 (against the FP64 oracle).  The cases cover the
layout's edges: rows that cross many segments (spans of several parts),
empty rows (ordinals mapped back to rows), entry counts that fill the last
chunk exactly or leave one entry, a single entry, duplicates summed by the
builder, rectangular shapes and a power-law matrix.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = {False: 1e-12, True: 1e-5}


def _coo(m, n, rows, cols, rng, unit=False):
    from cbspmv import gen
    key = np.unique(np.asarray(rows, np.int64) * n + np.asarray(cols, np.int64))
    r, c = key // n, key % n
    v = np.ones(r.size) if unit else rng.standard_normal(r.size)
    return gen.Coo(m, n, r.astype(np.int32), c.astype(np.int32), v)


def _cases():
    from cbspmv import gen
    rng = np.random.default_rng(17)
    out = [("random", gen.random_small(rng, 3000, 2500, 40000)),
           ("dups", gen.random_small(rng, 1200, 1000, 9000, dup=True)),
           ("wide", gen.random_small(rng, 300, 200000, 30000)),
           ("tall", gen.random_small(rng, 200000, 300, 30000)),
           ("power-law", gen.power_law(1 << 15, seed=3)),
           ("unit", gen.random_small(rng, 3000, 2500, 40000, unit=True))]
    # one row of 60000 entries (one per 16x16 block: COO blocks) crossing
    # many segments, and every ninth row of the rest non-empty
    n = 16 * 60000
    rows = np.concatenate([np.full(60000, 7), (rng.integers(0, 4000, 20000) // 9) * 9])
    cols = np.concatenate([np.arange(60000) * 16 + 3, rng.integers(0, n, 20000)])
    out.append(("huge-row-empty-rows", _coo(4000, n, rows, cols, rng)))
    # whole chunks of 128 entries exactly, and one entry past them
    for nnz in (128 * 40, 128 * 40 + 1):
        r = np.arange(nnz) // 3
        c = (np.arange(nnz) * 977) % 50000
        out.append((f"entries-{nnz}", _coo(int(r.max()) + 1, 50000, r, c, rng)))
    out.append(("one-entry", _coo(40, 30, [17], [29], rng)))
    return out


CASES = _cases()


def _check(y, yref, absrow, f32, what):
    err = np.abs(np.asarray(y, np.float64) - yref)
    bound = TOL[f32] * absrow + (1e-30 if f32 else 1e-300)
    worst = float(np.max(err / bound)) if err.size else 0.0
    assert worst <= 1.0, f"{what}: error {worst:.3g} x tolerance"


@pytest.mark.parametrize("name,coo", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("f32", [False, True])
@pytest.mark.parametrize("kernel", [0, 5])
def test_rowseg_matches_oracle(cuda, name, coo, f32, kernel):
    import torch
    import cbspmv
    import cbdump as cd
    from cbspmv import gen
    plan = cbspmv.Plan(coo, value_type=int(f32), kernel=kernel)
    x = gen.uniform_x(coo.n, 5)
    if f32:
        x = x.astype(np.float32).astype(np.float64)
    dt = torch.float32 if f32 else torch.float64
    xd = torch.from_numpy(x).to(cuda, dt)
    y = torch.full((coo.m,), float("nan"), dtype=dt, device=cuda)
    plan.spmv(xd, y)
    info = plan.info()
    assert info["csr_blocks"] == 0 and info["dense_blocks"] == 0
    assert info["rowseg_bytes"] > 0, "the row-segment stream was not built"
    torch.cuda.synchronize()
    y1 = y.cpu().numpy().copy()
    yref, ab = cd.oracle_spmm_ld(coo, x[None, :])
    _check(y1[None, :], yref, ab, f32, f"{name} kernel {kernel}")
    # a second launch: the span counters were reset, the sums are bitwise equal
    y.fill_(float("nan"))
    plan.spmv(xd, y)
    torch.cuda.synchronize()
    assert np.array_equal(y.cpu().numpy(), y1)
    plan.check()


@pytest.mark.parametrize("f32", [False, True])
def test_rowseg_set_values_and_transpose(cuda, f32):
    """New values reach the row-segment copy (set_values), and A^T x runs
    on the transposed layout's own stream."""
    import torch
    import cbspmv
    import cbdump as cd
    from cbspmv import gen
    rng = np.random.default_rng(23)
    coo = gen.random_small(rng, 5000, 4000, 60000)
    plan = cbspmv.Plan(coo, value_type=int(f32), want_transpose=1)
    dt = torch.float32 if f32 else torch.float64
    x = gen.uniform_x(coo.n, 9)
    g = gen.uniform_x(coo.m, 10)
    if f32:
        x = x.astype(np.float32).astype(np.float64)
        g = g.astype(np.float32).astype(np.float64)
    xd = torch.from_numpy(x).to(cuda, dt)
    gd = torch.from_numpy(g).to(cuda, dt)
    y = plan.spmv(xd)
    assert plan.info()["rowseg_bytes"] > 0
    vals = rng.standard_normal(coo.nnz)
    if f32:
        vals = vals.astype(np.float32).astype(np.float64)
    plan.set_values(torch.from_numpy(vals).to(cuda, dt))
    coo2 = gen.Coo(coo.m, coo.n, coo.row, coo.col, vals)
    y = plan.spmv(xd)
    gx = plan.spmv_t(gd)
    torch.cuda.synchronize()
    yref, ab = cd.oracle_spmm_ld(coo2, x[None, :])
    _check(y.cpu().numpy()[None, :], yref, ab, f32, "after set_values")
    gref, gab = cd.oracle_spmm_ld(coo2, g[None, :], transpose=True)
    _check(gx.cpu().numpy()[None, :], gref, gab, f32, "transpose after set_values")
    k, _ = plan.autotune(1)
    assert k in (1, 2, 3, 5)
    y2 = plan.spmv(xd)
    torch.cuda.synchronize()
    _check(y2.cpu().numpy()[None, :], yref, ab, f32, f"autotuned kernel {k}")


@pytest.mark.parametrize("name", ["random", "huge-row-empty-rows", "entries-5121", "power-law",
                                  "unit"])
@pytest.mark.parametrize("f32", [False, True])
@pytest.mark.parametrize("nrhs", [2, 3, 5, 8, 13, 16, 20])
def test_rowseg_several_rhs(cuda, name, f32, nrhs):
    """Several right-hand sides over the stream (lanes per entry chosen from
    nrhs; more than 16 in slabs of 16), against the oracle; with leading
    dimensions wider than nrhs (no vector loads) through the C ABI."""
    import ctypes
    import torch
    import cbspmv
    import cbdump as cd
    from cbspmv import gen
    coo = dict(CASES)[name]
    plan = cbspmv.Plan(coo, value_type=int(f32))
    X = gen.uniform_x(coo.n, 7, nrhs=nrhs)  # (nrhs, n)
    if f32:
        X = X.astype(np.float32).astype(np.float64)
    dt = torch.float32 if f32 else torch.float64
    Xd = torch.from_numpy(np.ascontiguousarray(X.T)).to(cuda, dt)
    Y = plan.spmv(Xd)
    assert plan.info()["rowseg_bytes"] > 0
    torch.cuda.synchronize()
    yref, ab = cd.oracle_spmm_ld(coo, X)
    _check(Y.cpu().numpy().T, yref, ab, f32, f"{name} nrhs {nrhs}")
    # padded leading dimensions
    ldx, ldy = nrhs + 3, nrhs + 5
    Xp = torch.zeros(coo.n, ldx, dtype=dt, device=cuda)
    Xp[:, :nrhs] = Xd
    Yp = torch.full((coo.m, ldy), float("nan"), dtype=dt, device=cuda)
    P = ctypes.c_void_p
    rc = cbspmv.lib().cbspmv_spmv(plan._h, P(Xp.data_ptr()), P(Yp.data_ptr()), nrhs, ldx, ldy,
                                  P(torch.cuda.current_stream().cuda_stream))
    assert rc == 0, cbspmv.last_error()
    torch.cuda.synchronize()
    Yh = Yp.cpu().numpy()
    _check(Yh[:, :nrhs].T, yref, ab, f32, f"{name} nrhs {nrhs} padded")
    assert np.all(np.isnan(Yh[:, nrhs:]))  # columns past nrhs untouched
    plan.check()
