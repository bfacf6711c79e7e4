"""CPU checks of the balanced (non-row-owned) schedule's stream for plans
built with row_owned = 0: read back through cbspmv_export and evaluated as
the kernel adds it (every non-skip entry's product added into its row), it
gives the oracle's y; and its groups follow the plan's block order (the
reference's balance permutation when it balanced, coo2block.h:382-498) --
group g holds only entries of the blocks g*W .. g*W+W-1."""
import numpy as np
import pytest

TOL = {False: 1e-12, True: 1e-5}
SKIP = 0xFFFFFFFF


def _bal(plan, f32):
    import cbspmv
    lib = cbspmv.lib()
    out = {}
    for name, dt in (("bal_rows", np.uint32), ("bal_cols", np.uint32),
                     ("bal_vals", np.float32 if f32 else np.float64), ("bal_gstart", np.int64)):
        cnt = lib.cbspmv_export(plan._h, name.encode(), None)
        if cnt < 0:
            return None
        a = np.zeros(cnt, dt)
        if cnt:
            lib.cbspmv_export(plan._h, name.encode(), a.ctypes.data_as(cbspmv.ctypes.c_void_p))
        out[name[4:]] = a
    return out


def _cases():
    from cbspmv import gen
    rng = np.random.default_rng(41)
    return [("random", gen.random_small(rng, 900, 700, 9000)),
            ("dups", gen.random_small(rng, 300, 300, 3000, dup=True)),
            ("power-law", gen.power_law(1 << 11, seed=5)),
            ("dense", gen.random_small(rng, 100, 100, 9000)),
            ("stencil", gen.stencil_27pt(6)),
            ("banded", gen.banded(rng, 2000, 30))]


CASES = _cases()


@pytest.mark.parametrize("name,coo", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("f32", [False, True])
@pytest.mark.parametrize("bs,waves", [(16, 4), (32, 2), (16, 1)])
def test_balanced_stream_decodes_and_follows_the_permutation(name, coo, f32, bs, waves):
    import cbspmv
    import cbdump as cd
    from cbspmv import gen
    plan = cbspmv.Plan(coo, value_type=int(f32), block_size=bs, row_owned=0,
                       waves_per_block=waves)
    b = _bal(plan, f32)
    assert b is not None
    rows, cols, vals, gs = b["rows"], b["cols"], b["vals"], b["gstart"]
    assert rows.size == cols.size == vals.size == 4 * gs[-1]
    real = rows != SKIP
    assert int(cols[real].max(initial=0)) < coo.n and int(rows[real].max(initial=0)) < coo.m
    x = gen.uniform_x(coo.n, 3)
    if f32:
        x = x.astype(np.float32).astype(np.float64)
    y = np.zeros(coo.m)
    np.add.at(y, rows[real].astype(np.int64), vals[real].astype(np.float64) * x[cols[real]])
    yref, ab = cd.oracle_spmm_ld(coo, x[None, :])
    assert np.all(np.abs(y - yref[0]) <= TOL[f32] * ab[0] + 1e-300)
    # the groups follow the balanced block order
    ex = plan.export()
    gr, gc = ex["gb_row_idx"], ex["gb_col_idx"]
    W = waves
    if ex["gather_flag"]:
        off, bcols = ex["block_cols_offset"], ex["block_cols"]
    for g in range(gs.size - 1):
        e0, e1 = 4 * gs[g], 4 * gs[g + 1]
        rr, cc = rows[e0:e1], cols[e0:e1]
        keep = rr != SKIP
        rr, cc = rr[keep].astype(np.int64), cc[keep].astype(np.int64)
        R = rr // bs
        if ex["gather_flag"]:
            pos = np.array([int(np.nonzero(bcols[off[r]:off[r + 1]] == c)[0][0])
                            for r, c in zip(R, cc)], np.int64)
            C = pos // bs
        else:
            C = cc // bs
        want = {(int(gr[i]), int(gc[i])) for i in range(g * W, min(g * W + W, gr.size))
                if gr[i] >= 0}
        assert set(zip(R.tolist(), C.tolist())) <= want


def test_no_balanced_stream_without_the_permutation():
    import cbspmv
    from cbspmv import gen
    coo = gen.random_small(np.random.default_rng(1), 200, 200, 2000)
    assert _bal(cbspmv.Plan(coo), False) is None  # row_owned = 1


def test_kernel_option_bounds():
    """Kernel options 0-6 are accepted (6: the balanced schedule, taken only by
    plans built with row_owned = 0); others are refused."""
    import cbspmv
    from cbspmv import gen
    coo = gen.random_small(np.random.default_rng(2), 100, 100, 500)
    for k in range(7):
        cbspmv.Plan(coo, kernel=k)
    for k in (-1, 7):
        with pytest.raises(cbspmv.CBSpMVError) as e:
            cbspmv.Plan(coo, kernel=k)
        assert e.value.status == "INVALID"
