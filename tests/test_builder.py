"""The product CB builder (libcbspmv.so) against the golden fixtures and the
oracle, bit for bit; input validation; device-layout reading on CPU."""
import pathlib
import re

import numpy as np
import pytest

import cbdump as cd
import layout_decode as ld

GOLDEN = sorted((pathlib.Path(__file__).parent / "golden").glob("*.npz"))


def _coo(f):
    from cbspmv.gen import Coo
    m, n = (int(v) for v in f["in_shape"])
    return Coo(m, n, f["in_row"], f["in_col"], f["in_val"])


@pytest.mark.parametrize("path", GOLDEN, ids=[p.stem for p in GOLDEN])
def test_builder_matches_golden(path):
    import cbspmv
    f = np.load(path)
    bs, ro = (int(v) for v in f["cfg"])
    want = {k: (int(f[k]) if k in cd.SCALARS else float(f[k]) if k in cd.FSCALARS
                else f[k]) for k in list(cd.SCALARS) + list(cd.FSCALARS) + list(cd.DTYPES)}
    got = cbspmv.Plan(_coo(f), block_size=bs, row_owned=ro).export()
    cd.compare_dumps(want, got, path.stem)


def _cases():
    from cbspmv import gen
    rng = np.random.default_rng(123)
    out = []
    for (m, n, nnz, dup, unit) in [(1, 1, 1, False, False), (15, 17, 40, True, False),
                                   (33, 31, 900, True, False), (1000, 800, 20000, False, False),
                                   (900, 900, 30000, True, True), (400, 500, 3000, False, False),
                                   (3000, 66000, 14000, False, False),
                                   (100, 100, 9000, False, False), (64, 64, 40000, True, False),
                                   (128, 130, 12000, False, False)]:
        out.append((f"r{m}x{n}_{nnz}_{int(dup)}{int(unit)}",
                    gen.random_small(rng, m, n, nnz, dup, unit)))
    out.append(("lap", gen.laplacian_2d(40, 50)))
    out.append(("st", gen.stencil_27pt(6)))
    out.append(("pl", gen.power_law(3000, kmax=3000, band=200, seed=8)))
    m, n = 160, 300
    cols = np.array([3, 7, 40, 41, 42, 100, 250])
    out.append(("uniform", gen.Coo(m, n, np.repeat(np.arange(m), 7).astype(np.int32),
                                   np.tile(cols, m).astype(np.int32), np.ones(7 * m))))
    # cancelling duplicates: a COO block whose dense image is all zero
    out.append(("cancel", gen.Coo(20, 20, np.array([0, 0, 5], np.int32),
                                  np.array([3, 3, 9], np.int32),
                                  np.array([1.5, -1.5, 0.0]))))
    return out


CASES = _cases()


@pytest.mark.parametrize("name,coo", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("bs", [16, 32])
@pytest.mark.parametrize("ro", [1, 0])
def test_builder_matches_oracle(name, coo, bs, ro):
    import cbspmv
    got = cbspmv.Plan(coo, block_size=bs, row_owned=ro).export()
    cd.compare_dumps(cd.oracle_build(coo, bs, ro), got, f"{name} bs{bs} ro{ro}")


@pytest.mark.parametrize("opt", [dict(force_coo64=1), dict(dense_sixteenths=12),
                                 dict(dense_sixteenths=16), dict(waves_per_block=8),
                                 dict(waves_per_block=1, row_owned=0)])
def test_builder_options_match_oracle(opt):
    """The reference's other compile-time macros (macros.h:79-94) as options."""
    import cbspmv
    o = dict(block_size=16, row_owned=1, waves_per_block=4, dense_sixteenths=15,
             force_coo64=0)
    o.update(opt)
    for name, coo in CASES:
        got = cbspmv.Plan(coo, **o).export()
        want = cd.oracle_build(coo, o["block_size"], o["row_owned"],
                               o["waves_per_block"], o["dense_sixteenths"],
                               o["force_coo64"])
        cd.compare_dumps(want, got, f"{name} {opt}")


def test_transpose_structure():
    """A^T's structure is the CB build of the transposed, row-sorted COO."""
    import cbspmv
    from cbspmv.gen import Coo
    for name, coo in CASES[3:8]:
        p = cbspmv.Plan(coo, want_transpose=1)
        order = np.lexsort((coo.row, coo.col))
        t = Coo(coo.n, coo.m, coo.col[order], coo.row[order], coo.val[order])
        cd.compare_dumps(cd.oracle_build(t), p.export(transpose=True), name)


def test_input_validation():
    import cbspmv
    from cbspmv.gen import Coo
    bad_order = Coo(4, 4, np.array([1, 0], np.int32), np.array([0, 0], np.int32),
                    np.ones(2))
    oob = Coo(4, 4, np.array([0, 4], np.int32), np.array([0, 0], np.int32), np.ones(2))
    neg = Coo(4, 4, np.array([0, 1], np.int32), np.array([-1, 0], np.int32), np.ones(2))
    big_col = Coo(4, 4, np.array([0, 1], np.int32), np.array([0, 9], np.int32), np.ones(2))
    # the same answers with A^T built alongside (on its own host thread)
    for t in (0, 1):
        for coo, status in ((bad_order, "UNSORTED"), (oob, "BOUNDS"), (neg, "BOUNDS"),
                            (big_col, "BOUNDS")):
            with pytest.raises(cbspmv.CBSpMVError) as e:
                cbspmv.Plan(coo, want_transpose=t)
            assert e.value.status == status, (t, status)
    ok = Coo(4, 4, np.array([0], np.int32), np.array([0], np.int32), np.ones(1))
    for opt in (dict(block_size=8), dict(block_size=64), dict(dense_sixteenths=0),
                dict(waves_per_block=0), dict(value_type=2)):
        with pytest.raises(cbspmv.CBSpMVError) as e:
            cbspmv.Plan(ok, **opt)
        assert e.value.status == "INVALID"
    assert "must" in cbspmv.last_error()


def test_unuploaded_plan_reports_state():
    import cbspmv
    from cbspmv.gen import Coo
    p = cbspmv.Plan(Coo(4, 4, np.array([0], np.int32), np.array([0], np.int32),
                        np.ones(1)))
    rc = cbspmv.lib().cbspmv_spmv(p._h, None, None, 1, 1, 1, None)
    assert cbspmv.STATUS[rc] == "STATE"
    rc = cbspmv.lib().cbspmv_spmv_t(p._h, None, None, 1, 1, 1, None)
    assert cbspmv.STATUS[rc] == "STATE"


@pytest.mark.parametrize("name,coo", CASES[:12], ids=[c[0] for c in CASES[:12]])
@pytest.mark.parametrize("bs", [16, 32])
@pytest.mark.parametrize("f32", [0, 1])
def test_device_layout_reads_back(name, coo, bs, f32):
    """The packed device layout, read on CPU exactly as the kernel reads it,
    gives the oracle's y (forward and transpose; small tiles force split
    block rows)."""
    import cbspmv
    from cbspmv import gen
    p = cbspmv.Plan(coo, block_size=bs, value_type=f32, tile_entries=64,
                    want_transpose=1)
    tol = 1e-6 if f32 else 1e-13
    x = gen.uniform_x(coo.n, 3)
    yref, ab = cd.oracle_spmm_ld(coo, x[None, :])
    assert np.all(np.abs(ld.decode_spmv(p, x) - yref[0]) <= tol * ab[0] + 1e-300)
    g = gen.uniform_x(coo.m, 4)
    gref, gab = cd.oracle_spmm_ld(coo, g[None, :], transpose=True)
    assert np.all(np.abs(ld.decode_spmv(p, g, transpose=True) - gref[0])
                  <= tol * gab[0] + 1e-300)


def test_value_slots_and_coords():
    """Stored slots: every input nonzero is summed into exactly one slot whose
    coordinates are the input's (row, col)."""
    import cbspmv
    for name, coo in CASES:
        p = cbspmv.Plan(coo)
        r, c, first = p.value_coords()
        slots = p.input_slots()
        assert slots.min() >= 0 and slots.max() < p.num_values()
        assert np.array_equal(r[slots], coo.row) and np.array_equal(c[slots], coo.col)
        assert np.all(first[first >= 0] < coo.nnz)


def test_header_symbols_exported():
    """libcbspmv.so exports every function include/cbspmv.h declares."""
    import cbspmv
    hdr = (pathlib.Path(__file__).resolve().parent.parent / "include" / "cbspmv.h").read_text()
    names = set(re.findall(r"\b(cbspmv_[a-z_0-9]+)\s*\(", hdr))
    assert len(names) >= 19
    missing = [n for n in sorted(names) if not hasattr(cbspmv.lib(), n)]
    assert not missing, missing


def test_info_counts():
    import cbspmv
    from cbspmv import gen
    coo = gen.stencil_27pt(6)
    p = cbspmv.Plan(coo)
    i = p.info()
    d = p.export()
    t = d["type_per_blk"] & 0x7F
    assert i["gb_nnzb"] == d["gb_nnzb"] == t.size
    assert i["coo_blocks"] == np.sum(t == 0) and i["csr_blocks"] == np.sum(t == 1)
    assert i["dense_blocks"] == np.sum(t == 3)
    assert i["algorithmic_bytes"] > 0 and i["tiles"] >= 1


def _unit_cases():
    from cbspmv import gen
    rng = np.random.default_rng(77)
    band = gen.banded(rng, 700, 20)
    return [("coo", gen.random_small(rng, 1500, 1200, 20000, unit=True)),
            ("dense", gen.random_small(rng, 128, 128, 15000, unit=True)),
            ("banded", gen.Coo(band.m, band.n, band.row, band.col, np.ones(band.nnz)))]


UNIT_CASES = _unit_cases()


@pytest.mark.parametrize("name,coo", UNIT_CASES, ids=[c[0] for c in UNIT_CASES])
@pytest.mark.parametrize("bs", [16, 32])
@pytest.mark.parametrize("f32", [0, 1])
def test_unit_layout_reads_back(name, coo, bs, f32):
    """Unit-valued matrices (the reference's UNIT_VALUES, cb-spmv-dcu.hpp:
    1105-1127): the layout stores no values and DENSE blocks as bitmasks,
    evaluates to the oracle's y, and is smaller than the valued layout."""
    import cbspmv
    from cbspmv import gen
    p = cbspmv.Plan(coo, block_size=bs, value_type=f32, tile_entries=64, want_transpose=1)
    k = cbspmv.Plan(coo, block_size=bs, value_type=f32, tile_entries=64, keep_values=1)
    assert p.info()["unit_values"] == 1
    assert p.info()["device_bytes"] < k.info()["device_bytes"]
    assert p.info()["algorithmic_bytes"] < k.info()["algorithmic_bytes"]
    tol = 1e-6 if f32 else 1e-13
    x = gen.uniform_x(coo.n, 3)
    yref, ab = cd.oracle_spmm_ld(coo, x[None, :])
    for plan in (p, k):
        assert np.all(np.abs(ld.decode_spmv(plan, x) - yref[0]) <= tol * ab[0] + 1e-300)
    g = gen.uniform_x(coo.m, 4)
    gref, gab = cd.oracle_spmm_ld(coo, g[None, :], transpose=True)
    assert np.all(np.abs(ld.decode_spmv(p, g, transpose=True) - gref[0]) <= tol * gab[0] + 1e-300)


@pytest.mark.parametrize("name,coo", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("tile_entries", [0, 64, 100])
def test_coo_sections_in_lane_slices(name, coo, tile_entries):
    """Each tile's COO section is stored in 32 lane slices: read back as
    slice 0, 1, ... 31 (slice l = positions 32 j + l < E, in j order) the
    entries are in strictly increasing (row, column) order, slice lengths
    differ by at most one (longer slices first), and the positions fill
    [0, E) exactly."""
    import cbspmv
    p = cbspmv.Plan(coo, tile_entries=tile_entries)
    fn = cbspmv.lib().cbspmv_export

    def raw(nm, dt):
        cnt = fn(p._h, nm.encode(), None)
        a = np.zeros(cnt, dt)
        if cnt:
            fn(p._h, nm.encode(), a.ctypes.data_as(cbspmv.ctypes.c_void_p))
        return a

    tiles = raw("dev_tiles", np.uint32).reshape(-1, 8)
    pay = raw("dev_payload", np.uint8)
    for t in tiles:
        E = int(t[4])
        if E == 0:
            continue
        idx = pay[int(t[3]) * 16:int(t[3]) * 16 + 4 * E].view(np.uint32).astype(np.int64)
        lens = [len(range(l, E, 32)) for l in range(32)]
        assert max(lens) - min(lens) <= 1 and lens == sorted(lens, reverse=True)
        order = np.concatenate([idx[l:E:32] for l in range(32)])
        assert order.size == E and np.all(np.diff(order) > 0)

