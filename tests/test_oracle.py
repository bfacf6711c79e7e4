"""The oracle, pinned: against the committed golden fixtures (made by the
reference's own host code, tests/golden/make_golden.py) always, and against
the reference compiled here (oracle/_ref) when it is present."""
import os
import pathlib

import numpy as np
import pytest

import cbdump as cd

GOLDEN = sorted((pathlib.Path(__file__).parent / "golden").glob("*.npz"))


def _coo(f):
    from cbspmv.gen import Coo
    m, n = (int(v) for v in f["in_shape"])
    return Coo(m, n, f["in_row"], f["in_col"], f["in_val"])


def _as_dump(f):
    d = {}
    for k in cd.SCALARS:
        d[k] = int(f[k])
    for k in cd.FSCALARS:
        d[k] = float(f[k])
    for k in cd.DTYPES:
        d[k] = f[k]
    return d


def test_golden_fixtures_present():
    assert len(GOLDEN) >= 15


@pytest.mark.parametrize("path", GOLDEN, ids=[p.stem for p in GOLDEN])
def test_oracle_matches_golden(path):
    f = np.load(path)
    bs, ro = (int(v) for v in f["cfg"])
    got = cd.oracle_build(_coo(f), bs, ro)
    cd.compare_dumps(_as_dump(f), got, path.stem)


@pytest.mark.parametrize("path", GOLDEN, ids=[p.stem for p in GOLDEN])
def test_golden_structure_decodes_to_coo_spmv(path):
    """Reading the reference's structure as its kernels do gives the
    reference's CPU SpMV (utils.h:98-111)."""
    f = np.load(path)
    bs, _ = (int(v) for v in f["cfg"])
    coo = _coo(f)
    x = np.random.default_rng(1).uniform(-1, 1, coo.n)
    y = cd.decode_spmv(_as_dump(f), bs, x)
    yref, ab = cd.oracle_spmm_ld(coo, x[None, :])
    assert np.all(np.abs(y - yref[0]) <= 1e-13 * ab[0] + 1e-300)


def _random_cases():
    from cbspmv import gen
    rng = np.random.default_rng(99)
    out = []
    for (m, n, nnz, dup, unit) in [(1, 1, 1, False, False), (17, 33, 100, True, False),
                                   (800, 700, 25000, False, False),
                                   (900, 900, 30000, True, True),
                                   (5000, 70000, 15000, False, False),
                                   (64, 64, 30000, True, False)]:
        out.append((f"r{m}x{n}_{nnz}", gen.random_small(rng, m, n, nnz, dup, unit)))
    out.append(("lap", gen.laplacian_2d(48, 40)))
    out.append(("st5", gen.stencil_27pt(5)))
    return out


@pytest.mark.skipif(not cd.have_ref(), reason="reference not compiled here")
@pytest.mark.parametrize("bs", [16, 32])
@pytest.mark.parametrize("ro", [1, 0])
def test_oracle_matches_reference(bs, ro):
    for name, coo in _random_cases():
        cd.compare_dumps(cd.ref_build(coo, bs, ro), cd.oracle_build(coo, bs, ro),
                         f"{name} bs{bs} ro{ro}")


@pytest.mark.skipif(not cd.have_ref(), reason="reference not compiled here")
def test_reference_checker_accepts_oracle_y():
    """The reference's own check_results_consistency (utils.h:85-136) accepts
    the oracle's y and rejects a perturbed one."""
    from cbspmv import gen
    coo = gen.power_law(2048, kmax=2048, band=128, seed=4)
    x = gen.uniform_x(coo.n, 2)
    y = cd.oracle_spmv(coo, x)
    assert cd.ref_check(coo, x, y)
    y[7] += 1.0
    assert not cd.ref_check(coo, x, y)


REF_DATA = pathlib.Path(os.environ.get("CB_REFERENCE", "/root/reference")) / "cb-spmv-dcu" / "data"


@pytest.mark.skipif(not (cd.have_ref() and REF_DATA.is_dir()),
                    reason="reference data files not present")
@pytest.mark.parametrize("name", ["1138_bus", "heart2"])
def test_reference_data_files(name):
    """The reference's bundled matrices at unit values (as its reader loads
    them, io/mmio_highlevel.h:201-203): builder parity for both block sizes,
    and the product builder on the same input."""
    import mtx
    import cbspmv
    coo = mtx.read_mtx_unit(REF_DATA / f"{name}.mtx")
    for bs in (16, 32):
        ref = cd.ref_build(coo, bs, 1)
        cd.compare_dumps(ref, cd.oracle_build(coo, bs, 1), f"{name} oracle")
        cd.compare_dumps(ref, cbspmv.Plan(coo, block_size=bs).export(), f"{name} product")
