"""Matrix Market reader with the reference reader's semantics (test helper).

Restates cb-spmv-dcu/src/io/mmio_highlevel.h:62-293 and :313-403:
coordinate files only; every value is forced to 1.0 (:201-203); symmetric,
skew and hermitian files are expanded by mirroring each off-diagonal entry
(:214-233); the result is emitted row by row, and inside a row in file order
(each mirrored entry sits where its generating line was read), :259-293 and
:392-398.  Used only for the reference's bundled data files, which are read in
place and never copied into this repository.
"""
from __future__ import annotations

import numpy as np

from cbdump import REPO  # noqa: F401  (keeps tests importable from anywhere)


def read_mtx_unit(path):
    import sys
    sys.path.insert(0, str(REPO / "cb-sparse-dcu_b200"))
    from cbspmv.gen import Coo

    with open(path) as f:
        banner = f.readline().lower().split()
        assert banner[0] == "%%matrixmarket" and banner[2] == "coordinate"
        symmetric = banner[4] in ("symmetric", "hermitian", "skew-symmetric")
        line = f.readline()
        while line.startswith("%"):
            line = f.readline()
        m, n, nz = (int(t) for t in line.split())
        data = np.loadtxt(f, usecols=(0, 1), dtype=np.int64, ndmin=2)
    i = data[:, 0] - 1
    j = data[:, 1] - 1
    assert i.shape[0] == nz
    if symmetric:
        off = i != j
        # interleave: entry k contributes (i,j) then, if off-diagonal, (j,i)
        seq = np.arange(nz) * 2
        rows = np.concatenate([i, j[off]])
        cols = np.concatenate([j, i[off]])
        order_key = np.concatenate([seq, seq[off] + 1])
    else:
        rows, cols, order_key = i, j, np.arange(nz)
    order = np.lexsort((order_key, rows))  # by row, then file order
    rows, cols = rows[order], cols[order]
    return Coo(m, n, rows.astype(np.int32), cols.astype(np.int32),
               np.ones(rows.shape[0], np.float64))
