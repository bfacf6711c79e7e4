"""CPU checks of the row-segment stream's host build (cb_rowseg.cpp): read
back through cbspmv_export and evaluated exactly as the kernel adds it
(layout_decode.rowseg_spmv), it gives the oracle's y for several resident
warp counts (one segment per chunk up to one segment for everything), and
its value positions are a permutation holding the layout's stored values."""
import numpy as np
import pytest

TOL = {False: 1e-12, True: 1e-5}


def _small_cases():
    from cbspmv import gen
    rng = np.random.default_rng(31)
    out = [("random", gen.random_small(rng, 700, 600, 6000)),
           ("dups", gen.random_small(rng, 300, 300, 2500, dup=True)),
           ("power-law", gen.power_law(1 << 11, seed=4)),
           ("unit", gen.random_small(rng, 700, 600, 6000, unit=True))]
    n = 16 * 3000
    rows = np.concatenate([np.full(3000, 5), (rng.integers(0, 900, 2000) // 7) * 7])
    cols = np.concatenate([np.arange(3000) * 16 + 1, rng.integers(0, n, 2000)])
    key = np.unique(rows.astype(np.int64) * n + cols)
    out.append(("huge-row-empty-rows",
                gen.Coo(900, n, (key // n).astype(np.int32), (key % n).astype(np.int32),
                        rng.standard_normal(key.size))))
    for nnz in (128 * 9, 128 * 9 + 1, 1):
        r = np.arange(nnz) // 2
        c = (np.arange(nnz) * 61) % 4000
        out.append((f"entries-{nnz}", gen.Coo(int(r.max()) + 1, 4000, r.astype(np.int32),
                                              c.astype(np.int32), rng.standard_normal(nnz))))
    return out


CASES = _small_cases()


@pytest.mark.parametrize("name,coo", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("f32", [False, True])
@pytest.mark.parametrize("warps", [1, 3, 64, 4736])
def test_rowseg_layout_decodes_to_oracle(name, coo, f32, warps):
    import cbspmv
    import cbdump as cd
    from cbspmv import gen
    from layout_decode import rowseg_arrays, rowseg_spmv
    plan = cbspmv.Plan(coo, value_type=int(f32))
    rs = rowseg_arrays(plan, warps)
    assert rs is not None
    x = gen.uniform_x(coo.n, 2)
    if f32:
        x = x.astype(np.float32).astype(np.float64)
    y = rowseg_spmv(rs, x, coo.m, f32)
    assert np.all(np.isfinite(y)), "a row was never written"
    yref, ab = cd.oracle_spmm_ld(coo, x[None, :])
    err = np.abs(y.astype(np.float64)[None, :] - yref)
    assert np.all(err <= TOL[f32] * ab + 1e-300)
    nch, M, nseg, nord, G, W = (int(v) for v in rs["sizes"])
    assert G == max(1, warps // 32) and W == (32768 if f32 else 16384)
    assert nseg == -(-nch // M) and nseg <= max(warps, 1) + 1
    if plan.info()["unit_values"]:  # words only, no values to place
        assert rs["vpos"].size == 0 and rs["chunks"].size == nch * 128 * 4
        return
    # every stored value sits once in the stream, at its value position
    vp = rs["vpos"]
    assert np.array_equal(np.sort(vp), np.arange(vp.size))
    cnt = cbspmv.lib().cbspmv_export(plan._h, b"dev_values", None)
    dv = np.zeros(cnt, np.float64)
    cbspmv.lib().cbspmv_export(plan._h, b"dev_values", dv.ctypes.data_as(cbspmv.ctypes.c_void_p))
    T = np.float32 if f32 else np.float64
    vsz = 4 if f32 else 8
    C, nv = 128, 16 // vsz
    i = vp % C
    pos = ((i % 4) // nv) * 32 * nv + (i // 4) * nv + (i % 4) % nv
    flat = rs["chunks"].reshape(nch, -1)[vp // C, :]
    got = np.array([flat[k, 4 * C + pos[k] * vsz: 4 * C + (pos[k] + 1) * vsz].view(T)[0]
                    for k in range(vp.size)])
    assert np.array_equal(got.astype(np.float64), dv)


def _csr_dense_cases():
    from cbspmv import gen
    rng = np.random.default_rng(3)
    return [("dense", gen.random_small(rng, 100, 100, 9000)),
            ("dense-unit", gen.random_small(rng, 100, 100, 9000, unit=True)),
            ("banded", gen.banded(rng, 3000, 40)),
            ("stencil", gen.stencil_27pt(6)),
            ("laplacian", gen.laplacian_2d(40))]


@pytest.mark.parametrize("name,coo", _csr_dense_cases(), ids=[c[0] for c in _csr_dense_cases()])
@pytest.mark.parametrize("f32", [False, True])
@pytest.mark.parametrize("bs", [16, 32])
def test_rowseg_layout_with_csr_dense_blocks(name, coo, f32, bs):
    """Layouts with CSR and DENSE blocks: their entries are expanded into the
    stream (DENSE blocks within their valid columns and rows; unit-valued
    masks by their set bits), which decodes to the oracle's y; every stored
    value inside those bounds has its stream position."""
    import cbspmv
    import cbdump as cd
    from cbspmv import gen
    from layout_decode import rowseg_arrays, rowseg_spmv
    plan = cbspmv.Plan(coo, value_type=int(f32), block_size=bs)
    info = plan.info()
    rs = rowseg_arrays(plan, 64)
    assert rs is not None
    x = gen.uniform_x(coo.n, 4)
    if f32:
        x = x.astype(np.float32).astype(np.float64)
    y = rowseg_spmv(rs, x, coo.m, f32)
    assert np.all(np.isfinite(y))
    yref, ab = cd.oracle_spmm_ld(coo, x[None, :])
    err = np.abs(y.astype(np.float64)[None, :] - yref)
    assert np.all(err <= TOL[f32] * ab + 1e-300), name
    if not info["unit_values"]:
        vp = rs["vpos"]
        placed = vp[vp >= 0]
        assert np.array_equal(np.sort(placed), np.arange(placed.size))


@pytest.mark.parametrize("spmv_only", [False, True])
def test_rowseg_same_stream_after_plan_file(tmp_path, spmv_only):
    """A plan loaded from a plan file (SpMV-only files carry no per-value
    arrays) builds the same stream as the plan it was saved from, so both
    give bit-identical sums."""
    import cbspmv
    from cbspmv import gen
    from layout_decode import rowseg_arrays
    coo = gen.power_law(1 << 11, seed=6)
    p = cbspmv.Plan(coo)
    path = tmp_path / "p.cbplan"
    p.save(path, spmv_only=spmv_only)
    q = cbspmv.Plan.load(path)
    a, b = rowseg_arrays(p, 64), rowseg_arrays(q, 64)
    assert a is not None and b is not None
    for k in ("sizes", "chunks", "meta", "spans", "rowmap", "empty", "wbase"):
        assert np.array_equal(a[k], b[k]), k
    assert b["vpos"].size == (0 if spmv_only else coo.nnz)


def _suite_cases():
    import test_gpu_spmv as tg
    import test_gpu_batch as tb
    seen, out = set(), []
    for name, coo in list(tg.CASES) + list(getattr(tb, "CASES", [])):
        if name not in seen:
            seen.add(name)
            out.append((name, coo))
    return out


@pytest.mark.parametrize("name,coo", _suite_cases(), ids=[c[0] for c in _suite_cases()])
@pytest.mark.parametrize("bs", [16, 32])
def test_rowseg_layout_on_the_gpu_suite_matrices(name, coo, bs):
    """Every matrix the GPU parity tests run, through the stream as the
    device builds it for a full B200 (4736 warps): decodes to the oracle, and
    every column lies inside x (the host build refuses anything else)."""
    import cbspmv
    import cbdump as cd
    from cbspmv import gen
    from layout_decode import rowseg_arrays, rowseg_spmv
    plan = cbspmv.Plan(coo, block_size=bs, tile_entries=64)
    rs = rowseg_arrays(plan, 4736)
    if coo.nnz == 0:
        assert rs is None
        return
    words = rs["chunks"].reshape(int(rs["sizes"][0]), -1)[:, :512].view(np.uint32)
    assert int((words & ((1 << 30) - 1)).max()) < coo.n
    x = gen.uniform_x(coo.n, 6)
    y = rowseg_spmv(rs, x, coo.m, False)
    yref, ab = cd.oracle_spmm_ld(coo, x[None, :])
    assert np.all(np.abs(y[None, :] - yref) <= TOL[False] * ab + 1e-300)
