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



def rowseg_arrays(plan, warps: int, transpose: bool = False) -> dict | None:
    """The row-segment stream of a plan as built for `warps` resident warps
    (cbspmv_export names rs_*:W), or None when the layout does not take it."""
    import cbspmv
    fn = cbspmv.lib().cbspmv_export_t if transpose else cbspmv.lib().cbspmv_export
    out = {}
    for name, dt in (("sizes", np.int32), ("chunks", np.uint8), ("meta", np.int32),
                     ("spans", np.int32), ("rowmap", np.int32), ("empty", np.int32),
                     ("vpos", np.int32), ("wbase", np.int32)):
        key = f"rs_{name}:{warps}".encode()
        cnt = fn(plan._h, key, None)
        if cnt < 0:
            return None
        a = np.zeros(cnt, dt)
        if cnt:
            fn(plan._h, key, a.ctypes.data_as(cbspmv.ctypes.c_void_p))
        out[name] = a
    return out


def rowseg_spmv(rs: dict, x: np.ndarray, m: int, f32: bool) -> np.ndarray:
    """y = A x evaluated from the row-segment stream exactly as the kernel
    (cb-sparse-dcu_b200/csrc/cb_rowseg_kernels.cu) adds it: per lane in entry
    order, then the segmented scan in lane order, spans in segment order, in
    the value type.  Rows never written stay NaN."""
    K, C = 4, 128
    T = np.float32 if f32 else np.float64
    x = np.asarray(x, T)
    nch, M, nseg, nord, G, W = (int(v) for v in rs["sizes"])
    vsz = 4 if f32 else 8
    CB = rs["chunks"].size // max(nch, 1)
    unit = CB == 4 * C  # words only: every stored value is 1
    chunks = rs["chunks"].reshape(nch, CB)
    meta = rs["meta"].reshape(-1, 4)
    spans = rs["spans"].reshape(-1, 4)
    rowmap = rs["rowmap"] if rs["rowmap"].size else None
    rid = (lambda o: int(rowmap[o])) if rowmap is not None else int
    y = np.full(m, np.nan, T)
    y[rs["empty"]] = 0
    part = np.full(2 * nseg, np.nan, T)
    cnt = np.zeros(spans.shape[0], np.int64)
    nv = 16 // vsz
    e = np.arange(C)
    ll, jj = e // K, e % K
    vpos = (jj // nv) * 32 * nv + ll * nv + jj % nv

    def arrive(sp, v, slot):
        part[slot] = v
        cnt[sp] += 1
        sa, sb, o = (int(t) for t in spans[sp][:3])
        if cnt[sp] == sb - sa + 1:
            tot = part[2 * sa + 1]
            for q in range(sa + 1, sb + 1):
                tot = T(tot + part[2 * q])
            y[rid(o)] = tot
            cnt[sp] = 0

    for s in range(nseg):
        wb = int(rs["wbase"][next(b for b in range(G) if s < (b + 1) * nseg // G)])
        first, starts, hs, ts = (int(t) for t in meta[s])
        ord0, carry = first, T(0)
        for c in range(s * M, min(nch, (s + 1) * M)):
            words = chunks[c, :4 * C].view(np.uint32).reshape(32, K)
            vals = (np.ones((32, K), T) if unit
                    else chunks[c, 4 * C:].view(T)[vpos].reshape(32, K))
            flags = (words >> 31).astype(np.int64)
            cntl = flags.sum(axis=1)
            ordS = ord0 + np.cumsum(cntl) - cntl
            run = np.zeros(32, T)
            head = np.zeros(32, T)
            seen = np.zeros(32, bool)
            ordE = ordS.copy()
            for ln in range(32):
                o = int(ordS[ln])
                for j in range(K):
                    f = bool(flags[ln, j])
                    if f and seen[ln]:
                        y[rid(o)] = run[ln]
                    if f and not seen[ln]:
                        head[ln] = run[ln]
                    seen[ln] |= f
                    o += int(f)
                    col = int(words[ln, j]) & ((1 << 30) - 1)
                    if words[ln, j] & (1 << 30):  # the CTA's window of x
                        assert wb <= col < wb + W
                    p = T(vals[ln, j]) * x[col]
                    run[ln] = p if f else T(run[ln] + p)
                ordE[ln] = o
            sc = run.copy()
            if not seen[0]:
                sc[0] = T(sc[0] + carry)
            for ln in range(1, 32):
                if not seen[ln]:
                    sc[ln] = T(sc[ln] + sc[ln - 1])
            for ln in range(32):
                if not seen[ln]:
                    continue
                cin = carry if ln == 0 else sc[ln - 1]
                o, v = int(ordS[ln]), T(cin + head[ln])
                if o == first and hs >= 0:
                    arrive(hs, v, 2 * s)
                elif not (o == first and starts) and o < nord:
                    y[rid(o)] = v
            carry, ord0 = sc[31], int(ordE[31])
        if ord0 == first and hs >= 0:
            arrive(hs, carry, 2 * s)
        elif ts >= 0:
            arrive(ts, carry, 2 * s + 1)
        elif ord0 < nord and not (ord0 == first and starts):
            y[rid(ord0)] = carry
    return y
