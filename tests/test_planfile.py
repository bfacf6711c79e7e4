"""Plan files (.cbplan): a saved and reloaded plan holds the same CB structure
and device layout, bit for bit, as the plan that was built; damaged files and
files of another version are refused.  Host only (no GPU)."""
import numpy as np
import pytest

import cbdump as cd
import layout_decode as ld


def _cases():
    from cbspmv import gen
    rng = np.random.default_rng(5)
    return [("pl", gen.power_law(6000, kmax=3000, band=300, seed=4)),
            ("st", gen.stencil_27pt(5)),
            ("dups", gen.random_small(rng, 300, 250, 4000, dup=True)),
            ("empty", gen.Coo(20, 30, np.zeros(0, np.int32), np.zeros(0, np.int32),
                              np.zeros(0)))]


CASES = _cases()
DEV = ["dev_tiles", "dev_blocks", "dev_payload", "dev_values"]


def _raw(plan, name, transpose=False):
    import cbspmv
    fn = cbspmv.lib().cbspmv_export_t if transpose else cbspmv.lib().cbspmv_export
    cnt = fn(plan._h, name.encode(), None)
    a = np.zeros(max(cnt, 0), np.uint8 if name == "dev_payload" else np.float64
                 if name == "dev_values" else np.uint32)
    if cnt > 0:
        fn(plan._h, name.encode(), a.ctypes.data_as(cbspmv.ctypes.c_void_p))
    return a


@pytest.mark.parametrize("name,coo", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("opts", [dict(), dict(block_size=32, value_type=1, want_transpose=1),
                                  dict(row_owned=0, tile_entries=64, kernel=2)])
def test_save_load_round_trip(tmp_path, name, coo, opts):
    import cbspmv
    p = cbspmv.Plan(coo, **opts)
    path = tmp_path / f"{name}.cbplan"
    p.save(path)
    q = cbspmv.Plan.load(path)
    assert q.info() == p.info()
    for f in ("block_size", "row_owned", "value_type", "want_transpose", "tile_entries",
              "kernel"):
        assert getattr(q.opts, f) == getattr(p.opts, f), f
    cd.compare_dumps(p.export(), q.export(), f"{name} {opts}")
    for dn in DEV:
        assert np.array_equal(_raw(p, dn), _raw(q, dn)), dn
    assert np.array_equal(p.input_slots(), q.input_slots())
    if opts.get("want_transpose"):
        cd.compare_dumps(p.export(transpose=True), q.export(transpose=True), f"{name} A^T")
        for dn in DEV:
            assert np.array_equal(_raw(p, dn, True), _raw(q, dn, True)), dn
    if coo.nnz:  # the loaded layout evaluates to the same y on the CPU
        from cbspmv import gen
        x = gen.uniform_x(coo.n, 2)
        assert np.array_equal(ld.decode_spmv(p, x), ld.decode_spmv(q, x))


@pytest.mark.parametrize("name,coo", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("opts", [dict(), dict(block_size=32, value_type=1, want_transpose=1)])
def test_spmv_only_files(tmp_path, name, coo, opts):
    """An SpMV-only file: the same device layout (tiles, blocks, payload),
    info and scalars, a fraction of the size; calls needing per-value data or
    host block arrays are refused; it saves again only SpMV-only."""
    import cbspmv
    p = cbspmv.Plan(coo, **opts)
    full, lean = tmp_path / "full.cbplan", tmp_path / "lean.cbplan"
    p.save(full)
    p.save(lean, spmv_only=True)
    if coo.nnz:
        assert lean.stat().st_size < full.stat().st_size / 2
    q = cbspmv.Plan.load(lean)
    assert q.info() == p.info()
    for f in ("block_size", "value_type", "want_transpose", "tile_entries", "kernel"):
        assert getattr(q.opts, f) == getattr(p.opts, f), f
    sp, sq = np.zeros(12, np.int64), np.zeros(12, np.int64)
    fp, fq = np.zeros(3), np.zeros(3)
    lib = cbspmv.lib()
    for t in ((0, 1) if opts.get("want_transpose") else (0,)):
        lib.cbspmv_export_scalars(p._h, t, sp.ctypes.data_as(cbspmv.ctypes.c_void_p),
                                  fp.ctypes.data_as(cbspmv.ctypes.c_void_p))
        lib.cbspmv_export_scalars(q._h, t, sq.ctypes.data_as(cbspmv.ctypes.c_void_p),
                                  fq.ctypes.data_as(cbspmv.ctypes.c_void_p))
        assert np.array_equal(sp, sq) and np.array_equal(fp, fq)
        for dn in ("dev_tiles", "dev_blocks", "dev_payload"):
            assert np.array_equal(_raw(p, dn, bool(t)), _raw(q, dn, bool(t))), dn
        fn = lib.cbspmv_export_t if t else lib.cbspmv_export
        for dn in ("dev_values", "gb_row_idx", "block_cols"):
            assert fn(q._h, dn.encode(), None) == -1, dn
    with pytest.raises(cbspmv.CBSpMVError) as e:
        q.input_slots()
    assert e.value.status == "STATE"
    with pytest.raises(cbspmv.CBSpMVError) as e:
        q.save(tmp_path / "again.cbplan")
    assert e.value.status == "STATE"
    q.save(tmp_path / "again.cbplan", spmv_only=True)
    assert (tmp_path / "again.cbplan").read_bytes() == lean.read_bytes()


def test_damaged_files_are_refused(tmp_path):
    import cbspmv
    p = cbspmv.Plan(CASES[0][1])
    path = tmp_path / "a.cbplan"
    p.save(path)
    data = bytearray(path.read_bytes())
    cases = {
        "truncated": data[: len(data) // 2],
        "flipped": data[:5000] + bytes([data[5000] ^ 0x10]) + data[5001:],
        "version": data[:8] + (99).to_bytes(4, "little") + data[12:],
        "magic": b"NOTAPLAN" + data[8:],
    }
    for what, blob in cases.items():
        bad = tmp_path / f"{what}.cbplan"
        bad.write_bytes(bytes(blob))
        with pytest.raises(cbspmv.CBSpMVError) as e:
            cbspmv.Plan.load(bad)
        assert e.value.status == "INVALID", what
    with pytest.raises(cbspmv.CBSpMVError):
        cbspmv.Plan.load(tmp_path / "missing.cbplan")
    assert "version 99" in str(_load_error(tmp_path / "version.cbplan"))


def _load_error(path):
    import cbspmv
    try:
        cbspmv.Plan.load(path)
    except cbspmv.CBSpMVError as e:
        return e
    return None
