"""GPU parity of the CB-SpMV kernels against the oracle, through the C ABI.

Tolerance (per row i, right-hand side j):
    |y_ij - y_ref_ij| <= tol * sum_k |a_ik x_kj|
with y_ref the oracle's long-double restatement of the reference's CPU SpMV
(cb-spmv-dcu/src/utils.h:98-111); tol = 1e-12 for FP64, 1e-5 for FP32 (FP32
values, FP32 accumulation, error measured against the FP64 oracle).  A plain
relative error is ill-defined where y ~ 0 (N(0,1) values), so the bound is
scaled by each row's absolute sum.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = {False: 1e-12, True: 1e-5}


def _cases():
    from cbspmv import gen
    rng = np.random.default_rng(7)
    out = [
        ("rand-small", gen.random_small(rng, 50, 40, 300)),
        ("rand-dups", gen.random_small(rng, 300, 300, 3000, dup=True)),
        ("rand-mid", gen.random_small(rng, 1000, 800, 20000)),
        ("rand-wide", gen.random_small(rng, 400, 70000, 30000)),
        ("rand-dense", gen.random_small(rng, 100, 100, 9000)),
        ("dense-dups", gen.random_small(rng, 64, 64, 40000, dup=True)),
        ("ragged", gen.random_small(rng, 37, 41, 1500, dup=True)),
        ("unit", gen.random_small(rng, 500, 500, 8000, unit=True)),
        ("lap64", gen.laplacian_2d(64, 64)),
        ("st6", gen.stencil_27pt(6)),
        ("pl8192", gen.power_law(8192, kmax=8192, band=512, seed=11)),
    ]
    m, n = 200, 300
    cols = np.array([3, 7, 40, 41, 42, 100, 250])
    out.append(("uniform", gen.Coo(m, n, np.repeat(np.arange(m), 7).astype(np.int32),
                                   np.tile(cols, m).astype(np.int32),
                                   np.ones(7 * m))))
    return out


CASES = _cases()


def _check(y, yref, absrow, f32, what):
    err = np.abs(np.asarray(y, np.float64) - yref)
    bound = TOL[f32] * absrow + (1e-300 if not f32 else 1e-30)
    worst = float(np.max(err / bound)) if err.size else 0.0
    assert worst <= 1.0, f"{what}: error {worst:.3g} x tolerance"
    return worst


@pytest.mark.parametrize("name,coo", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("bs", [16, 32])
@pytest.mark.parametrize("f32", [False, True])
@pytest.mark.parametrize("tile_entries", [0, 64])
@pytest.mark.parametrize("kernel", [1, 2, 3])
def test_spmv_matches_oracle(cuda, name, coo, bs, f32, tile_entries, kernel):
    import torch
    import cbspmv
    import cbdump as cd
    from cbspmv import gen
    dt = torch.float32 if f32 else torch.float64
    plan = cbspmv.Plan(coo, block_size=bs, value_type=int(f32),
                       tile_entries=tile_entries, kernel=kernel)
    x = gen.uniform_x(coo.n, 5)
    if f32:
        x = x.astype(np.float32).astype(np.float64)  # same x for both
    yref, ab = cd.oracle_spmm_ld(coo, x[None, :])
    xd = torch.from_numpy(x).to(cuda, dt)
    y = torch.full((coo.m,), float("nan"), dtype=dt, device=cuda)
    plan.spmv(xd, y)
    torch.cuda.synchronize()
    y1 = y.cpu().numpy()
    _check(y1, yref[0], ab[0], f32, f"{name} bs{bs} f32={f32}")
    # repeated launches reuse the split-row counters (reset by the last tile
    # of each row); every launch must still be within tolerance
    for _ in range(3):
        y.fill_(float("nan"))
        plan.spmv(xd, y)
        torch.cuda.synchronize()
        _check(y.cpu().numpy(), yref[0], ab[0], f32, f"{name} repeat")


@pytest.mark.parametrize("nrhs", [2, 5])
@pytest.mark.parametrize("f32", [False, True])
@pytest.mark.parametrize("kernel", [1, 2])
def test_multi_rhs(cuda, nrhs, f32, kernel):
    import torch
    import cbspmv
    import cbdump as cd
    from cbspmv import gen
    coo = gen.power_law(4096, kmax=4096, band=256, seed=3, mean=24)
    dt = torch.float32 if f32 else torch.float64
    plan = cbspmv.Plan(coo, value_type=int(f32), tile_entries=128, kernel=kernel)
    X = gen.uniform_x(coo.n, 9, nrhs=nrhs)  # (nrhs, n)
    if f32:
        X = X.astype(np.float32).astype(np.float64)
    yref, ab = cd.oracle_spmm_ld(coo, X)
    Y = plan.spmv(torch.from_numpy(np.ascontiguousarray(X.T)).to(cuda, dt))
    torch.cuda.synchronize()
    _check(Y.cpu().numpy().T, yref, ab, f32, f"nrhs={nrhs}")


@pytest.mark.parametrize("name", ["pl8192", "st6", "lap64", "rand-dense"])
@pytest.mark.parametrize("nrhs", [1, 4])
def test_autotune_keeps_a_correct_kernel(cuda, name, nrhs):
    """cbspmv_autotune picks one of the kernels that can run the plan and later
    calls use it with unchanged results."""
    import torch
    import cbspmv
    import cbdump as cd
    from cbspmv import gen
    coo = dict(CASES)[name]
    plan = cbspmv.Plan(coo, want_transpose=1)
    k, ms = plan.autotune(nrhs)
    assert k in ((1, 2, 3, 4, 5) if nrhs == 1 else (3, 5)) and ms > 0
    X = gen.uniform_x(coo.n, 31, nrhs=max(nrhs, 2))[:nrhs]
    yref, ab = cd.oracle_spmm_ld(coo, X)
    xd = torch.from_numpy(np.ascontiguousarray(X.T)).to(cuda)
    if nrhs == 1:
        xd = xd[:, 0].contiguous()
    y = plan.spmv(xd)
    torch.cuda.synchronize()
    _check(y.cpu().numpy().reshape(coo.m, nrhs).T, yref, ab, False, f"autotuned {k}")
    G = gen.uniform_x(coo.m, 32, nrhs=max(nrhs, 2))[:nrhs]
    gref, gab = cd.oracle_spmm_ld(coo, G, transpose=True)
    gd = torch.from_numpy(np.ascontiguousarray(G.T)).to(cuda)
    if nrhs == 1:
        gd = gd[:, 0].contiguous()
    gx = plan.spmv_t(gd)
    torch.cuda.synchronize()
    _check(gx.cpu().numpy().reshape(coo.n, nrhs).T, gref, gab, False, f"autotuned {k} A^T")


def test_host_entry_points(cuda):
    """cb_spmv (the reference's one-call surface) and spmv_host."""
    import cbspmv
    import cbdump as cd
    from cbspmv import gen
    coo = gen.laplacian_2d(128, 128)
    plan = cbspmv.Plan(coo)
    x = gen.uniform_x(coo.n, 0)
    yref, ab = cd.oracle_spmm_ld(coo, x[None, :])
    y, met = plan.cb_spmv(x)
    _check(y, yref[0], ab[0], False, "cb_spmv")
    assert met["runtime"] > 0 and met["gflops"] > 0
    y2 = plan.spmv_host(x)
    _check(y2, yref[0], ab[0], False, "spmv_host")


@pytest.mark.parametrize("nrhs", [1, 3])
def test_host_async_pipeline(cuda, nrhs):
    """cbspmv_spmv_host_async: several calls in flight on pinned host buffers,
    each result equal to the oracle's once the caller's stream is synced; a
    call with more right-hand sides regrows the pipeline."""
    import ctypes
    import torch
    import cbspmv
    import cbdump as cd
    from cbspmv import gen
    coo = gen.power_law(20000, kmax=5000, band=600, seed=9)
    plan = cbspmv.Plan(coo).upload()
    lib = cbspmv.lib()
    stream = torch.cuda.current_stream()
    sp = ctypes.c_void_p(stream.cuda_stream)
    calls = []
    for i in range(5):
        X = gen.uniform_x(coo.n, 40 + i, nrhs=max(nrhs, 2))[:nrhs]
        xh = torch.from_numpy(np.ascontiguousarray(X.T)).pin_memory()
        yh = torch.full((coo.m, nrhs), float("nan"), dtype=torch.float64).pin_memory()
        rc = lib.cbspmv_spmv_host_async(plan._h, ctypes.c_void_p(xh.data_ptr()),
                                        ctypes.c_void_p(yh.data_ptr()), nrhs, sp)
        assert rc == 0, cbspmv.last_error()
        calls.append((X, xh, yh))
    stream.synchronize()
    for i, (X, _, yh) in enumerate(calls):
        yref, ab = cd.oracle_spmm_ld(coo, X)
        _check(yh.numpy().T, yref, ab, False, f"async call {i}")
    # more right-hand sides than before: the buffers grow
    X = gen.uniform_x(coo.n, 60, nrhs=nrhs + 2)
    xh = torch.from_numpy(np.ascontiguousarray(X.T)).pin_memory()
    yh = torch.zeros((coo.m, nrhs + 2), dtype=torch.float64).pin_memory()
    assert lib.cbspmv_spmv_host_async(plan._h, ctypes.c_void_p(xh.data_ptr()),
                                      ctypes.c_void_p(yh.data_ptr()), nrhs + 2, sp) == 0
    stream.synchronize()
    yref, ab = cd.oracle_spmm_ld(coo, X)
    _check(yh.numpy().T, yref, ab, False, "async regrown")


def test_loaded_plan_gives_the_same_y(cuda, tmp_path):
    """A plan saved after autotuning and loaded back runs the same kernel on
    the same layout: bit-identical y."""
    import torch
    import cbspmv
    from cbspmv import gen
    for coo, spmv_only in ((dict(CASES)["pl8192"], False), (dict(CASES)["st6"], False),
                           (dict(CASES)["pl8192"], True), (dict(CASES)["st6"], True)):
        p = cbspmv.Plan(coo, want_transpose=1)
        p.autotune(1)
        path = tmp_path / "p.cbplan"
        p.save(path, spmv_only=spmv_only)
        q = cbspmv.Plan.load(path)
        assert q.opts.kernel == p.opts.kernel
        x = torch.from_numpy(gen.uniform_x(coo.n, 8)).to(cuda)
        X = torch.from_numpy(gen.uniform_x(coo.n, 9, nrhs=4).T.copy()).to(cuda)
        g = torch.from_numpy(gen.uniform_x(coo.m, 10)).to(cuda)
        y1, y2 = p.spmv(x), q.spmv(x)
        Y1, Y2 = p.spmv(X), q.spmv(X)
        t1, t2 = p.spmv_t(g), q.spmv_t(g)
        torch.cuda.synchronize()
        assert torch.equal(y1, y2) and torch.equal(Y1, Y2) and torch.equal(t1, t2)
        if spmv_only:  # no per-value data: value updates and gradients refused
            for call in (lambda: q.set_values(torch.ones(coo.nnz, dtype=torch.float64,
                                                         device=cuda)),
                         lambda: q.grad_vals(g, x)):
                with pytest.raises(cbspmv.CBSpMVError) as e:
                    call()
                assert e.value.status == "STATE"


def test_empty_and_degenerate(cuda):
    import torch
    import cbspmv
    from cbspmv import gen
    # no nonzeros: y must be all zeros (cb-spmv-dcu.hpp:1091-1098)
    e = gen.Coo(33, 17, np.zeros(0, np.int32), np.zeros(0, np.int32), np.zeros(0))
    p = cbspmv.Plan(e)
    y = p.spmv(torch.ones(17, dtype=torch.float64, device=cuda),
               torch.full((33,), 5.0, dtype=torch.float64, device=cuda))
    assert torch.count_nonzero(y).item() == 0
    yh, _ = p.cb_spmv(np.ones(17))
    assert not yh.any()
    # a single nonzero in a corner, empty rows around it
    c = gen.Coo(1000, 1000, np.array([999], np.int32), np.array([0], np.int32),
                np.array([2.5]))
    p = cbspmv.Plan(c)
    x = torch.arange(1000, dtype=torch.float64, device=cuda) + 1
    y = p.spmv(x, torch.full((1000,), 7.0, dtype=torch.float64, device=cuda))
    yy = y.cpu().numpy()
    assert yy[999] == 2.5 and not yy[:999].any()


def _unit_cases():
    from cbspmv import gen
    rng = np.random.default_rng(78)
    band = gen.banded(rng, 3000, 40)
    return [("coo", gen.random_small(rng, 4000, 3000, 60000, unit=True)),
            ("dense", gen.random_small(rng, 256, 256, 60000, unit=True)),
            ("banded", gen.Coo(band.m, band.n, band.row, band.col, np.ones(band.nnz)))]


UNIT = _unit_cases()


@pytest.mark.parametrize("name,coo", UNIT, ids=[c[0] for c in UNIT])
@pytest.mark.parametrize("bs", [16, 32])
@pytest.mark.parametrize("f32", [False, True])
@pytest.mark.parametrize("kernel", [1, 2, 3])
@pytest.mark.parametrize("nrhs", [1, 4])
def test_unit_valued_plans(cuda, name, coo, bs, f32, kernel, nrhs):
    """Unit-valued matrices run without stored values (DENSE blocks as
    bitmasks) in every kernel, and refuse set_values."""
    import torch
    import cbspmv
    import cbdump as cd
    from cbspmv import gen
    dt = torch.float32 if f32 else torch.float64
    plan = cbspmv.Plan(coo, block_size=bs, value_type=int(f32), kernel=kernel, tile_entries=128)
    assert plan.info()["unit_values"] == 1
    X = gen.uniform_x(coo.n, 6, nrhs=max(nrhs, 2))[:nrhs]
    if f32:
        X = X.astype(np.float32).astype(np.float64)
    yref, ab = cd.oracle_spmm_ld(coo, X)
    xd = torch.from_numpy(np.ascontiguousarray(X.T)).to(cuda, dt)
    if nrhs == 1:
        xd = xd[:, 0].contiguous()
    for _ in range(2):
        y = plan.spmv(xd)
        torch.cuda.synchronize()
        _check(y.cpu().numpy().reshape(coo.m, nrhs).T, yref, ab, f32, f"unit {name}")
    with pytest.raises(cbspmv.CBSpMVError) as e:
        plan.set_values(torch.ones(coo.nnz, dtype=dt, device=cuda))
    assert e.value.status == "UNSUPPORTED"


@pytest.mark.parametrize("nrhs", [1, 6])
@pytest.mark.parametrize("f32", [False, True])
def test_tuner_over_block_size_tiles_kernels_lanes(cuda, nrhs, f32):
    """cbspmv_tune tries block size 16/32 x tile size auto/128 x kernel (x
    lanes per entry for several right-hand sides); the plan it keeps, and every
    forced lane split, give the oracle's result."""
    import torch
    import cbspmv
    import cbdump as cd
    from cbspmv import gen
    coo = gen.power_law(20000, kmax=3000, band=800, seed=12)
    plan, rep = cbspmv.tune(coo, nrhs, value_type=int(f32))
    assert rep["tried"] == 4 and rep["block_size"] in (16, 32) and rep["ms"] > 0
    assert plan.bs == rep["block_size"]
    dt = torch.float32 if f32 else torch.float64
    X = gen.uniform_x(coo.n, 8, nrhs=max(nrhs, 2))[:nrhs]
    if f32:
        X = X.astype(np.float32).astype(np.float64)
    yref, ab = cd.oracle_spmm_ld(coo, X)
    xd = torch.from_numpy(np.ascontiguousarray(X.T)).to(cuda, dt)
    if nrhs == 1:
        xd = xd[:, 0].contiguous()
    for lanes in ([rep["rhs_lanes"]] if nrhs == 1 else [rep["rhs_lanes"], 0, 1, 2, 4]):
        plan.set_rhs_lanes(lanes)
        y = plan.spmv(xd)
        torch.cuda.synchronize()
        _check(y.cpu().numpy().reshape(coo.m, nrhs).T, yref, ab, f32, f"tuned lanes={lanes}")


def _patterned(m=3000, n=2500, npat=70, seed=21):
    """Unit-valued rows drawn from a few column patterns (the structure the
    reference's pattern schedule exploits): each row takes one of npat random
    column sets, some of them empty."""
    from cbspmv import gen
    rng = np.random.default_rng(seed)
    pats = [np.sort(rng.choice(n, size=int(rng.integers(0, 90)), replace=False))
            for _ in range(npat)]
    which = rng.integers(0, npat, size=m)
    rows = np.concatenate([np.full(len(pats[w]), r) for r, w in enumerate(which)])
    cols = np.concatenate([pats[w] for w in which])
    return gen.Coo(m, n, rows.astype(np.int32), cols.astype(np.int32), np.ones(rows.size))


@pytest.mark.parametrize("f32", [False, True])
@pytest.mark.parametrize("bs", [16, 32])
def test_pattern_reuse_schedule(cuda, f32, bs):
    """Unit values with few row patterns: the automatic choice is the
    pattern-reuse schedule (one sum per pattern, written to all its rows); it,
    and every other kernel on the same plan, give the oracle's y."""
    import torch
    import cbspmv
    import cbdump as cd
    from cbspmv import gen
    coo = _patterned()
    plan = cbspmv.Plan(coo, value_type=int(f32), block_size=bs)
    info = plan.info()
    assert info["unit_values"] and 0 < info["patterns"] * 2 < coo.m
    x = gen.uniform_x(coo.n, 3)
    if f32:
        x = x.astype(np.float32).astype(np.float64)
    yref, ab = cd.oracle_spmm_ld(coo, x[None, :])
    dt = torch.float32 if f32 else torch.float64
    xd = torch.from_numpy(x).to(cuda, dt)
    for kernel in (0, 4, 1, 2, 3):
        p = plan if kernel == 0 else cbspmv.Plan(coo, value_type=int(f32), block_size=bs,
                                                 kernel=kernel)
        y = torch.full((coo.m,), float("nan"), dtype=dt, device=cuda)
        for _ in range(2):
            p.spmv(xd, y)
        torch.cuda.synchronize()
        _check(y.cpu().numpy()[None, :], yref, ab, f32, f"kernel {kernel}")
    k, _ = plan.autotune(1)
    assert k in (1, 2, 3, 4)


def test_small_direct_schedule(cuda):
    """Small unit-valued gathered matrices (the reference's small-direct
    case): the automatic choice is the direct kernel, exact."""
    import torch
    import cbspmv
    import cbdump as cd
    from cbspmv import gen
    rng = np.random.default_rng(5)
    coo = gen.random_small(rng, 900, 700, 6000, unit=True)
    plan = cbspmv.Plan(coo)
    ex = plan.export()
    assert ex["gather_flag"] and ex["compact_coo_indices"] and coo.nnz < 10000
    x = gen.uniform_x(coo.n, 4)
    yref, ab = cd.oracle_spmm_ld(coo, x[None, :])
    y = plan.spmv(torch.from_numpy(x).to(cuda))
    torch.cuda.synchronize()
    _check(y.cpu().numpy()[None, :], yref, ab, False, "small direct")
