"""Generates the golden CB-build fixtures in this directory by running the
REFERENCE's own host code (coo2block_gather, cb-spmv-dcu/src/coo2block.h:628,
compiled from its headers into oracle/_ref/ by `make -C oracle ref`) on small
seeded synthetic matrices.  Each fixture stores the input COO and every
GLOBAL_BLOCK array the reference produced, so the oracle and the product
builder can be checked bit for bit without the reference present.

    python tests/golden/make_golden.py
"""
import pathlib
import sys

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
REPO = HERE.parent.parent
sys.path.insert(0, str(REPO / "cb-sparse-dcu_b200"))
sys.path.insert(0, str(REPO / "tests"))

from cbspmv import gen  # noqa: E402
import cbdump as cd  # noqa: E402


def cases():
    rng = np.random.default_rng(2024)
    m, n = 256, 64
    rows = np.repeat(np.arange(m), n)
    uni = gen.Coo(m, n, rows.astype(np.int32), np.tile(np.arange(n), m).astype(np.int32),
                  np.tile(np.linspace(-1, 1, n), m))
    return [
        ("lap32", gen.laplacian_2d(32, 32), [(16, 1), (32, 1)]),
        ("lap64", gen.laplacian_2d(64, 64), [(16, 1), (16, 0), (32, 0)]),
        ("pl1024", gen.power_law(1024, kmax=1024, band=96, seed=1), [(16, 1), (16, 0)]),
        ("st4", gen.stencil_27pt(4), [(16, 1), (32, 1)]),
        ("rand_dups", gen.random_small(rng, 300, 300, 3000, dup=True), [(16, 1), (32, 1)]),
        ("compact", gen.random_small(rng, 500, 500, 3000), [(16, 1)]),
        ("direct", gen.random_small(rng, 3000, 60000, 12000), [(16, 1), (16, 0)]),
        ("dense_uniform", uni, [(16, 1), (32, 1), (16, 0)]),
        ("mixed", gen.random_small(rng, 100, 100, 6000, dup=True), [(16, 1), (32, 1)]),
    ]


def main():
    if cd.ref_lib(16, 1) is None:
        raise SystemExit("oracle/_ref not built: run `make -C oracle ref` first")
    total = 0
    for name, coo, cfgs in cases():
        for bs, ro in cfgs:
            d = cd.ref_build(coo, bs, ro)
            arrays = {f"in_{k}": getattr(coo, k) for k in ("row", "col", "val")}
            arrays["in_shape"] = np.array([coo.m, coo.n], np.int64)
            arrays["cfg"] = np.array([bs, ro], np.int64)
            for k, v in d.items():
                arrays[k] = np.asarray(v)
            path = HERE / f"{name}_bs{bs}_ro{ro}.npz"
            np.savez_compressed(path, **arrays)
            total += path.stat().st_size
            print(f"{path.name}: nnz={coo.nnz} nnzb={d['gb_nnzb']} "
                  f"gather={d['gather_flag']} {path.stat().st_size} B")
    print("total", total)


if __name__ == "__main__":
    main()
