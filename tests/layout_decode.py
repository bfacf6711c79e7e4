"""Host-side reading of the device layout exactly as the tile kernel reads it
(cb-sparse-dcu_b200/csrc/cb_kernels.cu), to check a plan's layout on CPU
before any GPU run.  Test infrastructure; small matrices only (Python loops).
"""
from __future__ import annotations

import numpy as np


def _a16(x: int) -> int:
    return (x + 15) & ~15


def decode_spmv(plan, x: np.ndarray, transpose: bool = False) -> np.ndarray:
    """y = A x (or A^T x) evaluated from dev_tiles / dev_blocks / dev_payload,
    with long-double accumulation."""
    d = plan.export(transpose=transpose)
    import cbspmv
    fn = cbspmv.lib().cbspmv_export_t if transpose else cbspmv.lib().cbspmv_export

    def raw(name, dt):
        cnt = fn(plan._h, name.encode(), None)
        a = np.zeros(cnt, dt)
        if cnt:
            fn(plan._h, name.encode(), a.ctypes.data_as(cbspmv.ctypes.c_void_p))
        return a

    tiles = raw("dev_tiles", np.uint32).reshape(-1, 8)
    blocks = raw("dev_blocks", np.uint32).reshape(-1, 4)
    pay = raw("dev_payload", np.uint8)
    bs = plan.bs
    vt = np.float32 if plan.f32 else np.float64
    vsz = 4 if plan.f32 else 8
    isz = 1 if bs == 16 else 2
    it = np.uint8 if bs == 16 else np.uint16
    gather = d["gather_flag"]
    # unit-valued layouts store no values and DENSE blocks as bitmasks
    unit = bool(plan.info()["unit_values"]) and not plan.opts.keep_values
    bcols = d["block_cols"]
    m = d["m"]
    y = np.zeros(m, np.longdouble)
    seen_rows = np.zeros(m, bool)
    for t in tiles:
        begin, brow, counts, p16, E, slot, first, ntiles = (int(v) for v in t)
        nb, ncoo, nxt = counts & 0xFF, (counts >> 8) & 0xFF, (counts >> 16) & 0xFF
        assert nb == ncoo + nxt and nb <= 32 and E <= 512
        base = p16 * 16
        idx = pay[base:base + 4 * E].view(np.uint32)
        cv = (np.ones(E, vt) if unit else
              pay[base + _a16(4 * E):base + _a16(4 * E) + vsz * E].view(vt))
        r0 = brow * bs
        rows = np.arange(r0, min(r0 + bs, m))
        seen_rows[rows] = True
        e_seen = 0
        for q in range(nb):
            off, meta, xbase, _ = (int(v) for v in blocks[begin + q])
            typ, k, valid = meta & 3, (meta >> 3) & 2047, (meta >> 14) & 63
            if q < ncoo:
                assert typ == 0 and off == e_seen
                for e in range(off, off + k):
                    w = int(idx[e])
                    r, col = w >> 27, w & ((1 << 27) - 1)
                    y[r0 + r] += np.longdouble(cv[e]) * x[col]
                e_seen += k
                continue

            def xcol(c):
                if c >= valid:
                    return None
                return int(bcols[xbase + c]) if gather else xbase + c

            pb = base + off
            if typ == 1:
                rp = pay[pb:pb + (bs + 1) * isz].view(it)
                ci = pay[pb + (bs + 1) * isz:pb + (bs + 1 + k) * isz].view(it)
                vo = pb + _a16((bs + 1 + k) * isz)
                vv = np.ones(k, vt) if unit else pay[vo:vo + k * vsz].view(vt)
                for r in range(bs):
                    for kk in range(int(rp[r]), int(rp[r + 1])):
                        y[r0 + r] += np.longdouble(vv[kk]) * x[xcol(int(ci[kk]))]
            else:
                assert typ == 3
                if unit:
                    vv = np.unpackbits(pay[pb:pb + bs * bs // 8],
                                       bitorder="little").astype(vt)
                else:
                    vv = pay[pb:pb + bs * bs * vsz].view(vt)
                for r in range(bs):
                    if r0 + r >= m:
                        continue
                    for c in range(bs):
                        col = xcol(c)
                        if col is not None:
                            y[r0 + r] += np.longdouble(vv[r * bs + c]) * x[col]
        assert e_seen == E
    assert seen_rows.all(), "a row is not covered by any tile"
    return y.astype(np.float64)

