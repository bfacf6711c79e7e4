"""One matrix sharded by block rows over the ranks of a process group.

Rank r owns rows [rb[r], rb[r+1]) of A, cut on block-row boundaries so that
every rank holds about the same number of stored values, and the entries
[cb[r], cb[r+1]) of x (the same cuts when A is square).  y = A x on rank r
needs x at the columns its rows use: its own entries plus a halo held by the
other ranks.  x travels by one all-gather (NCCL over NVLink on GPUs, gloo on
CPUs) of each rank's x range padded to the longest range (equal pieces), so
x_all holds range s at s * L.  Two ways to run a rank's rows:

* one plan (default): every column renumbered into x_all; the all-gather,
  then one SpMV.  The CB build gathers each block row's columns, so the
  scattered columns of other ranks cost no more than they do unsharded.
* own + halo (overlap=True): A_own (the rank's own columns, renumbered to its
  x range) runs while the all-gather is in flight, then A_halo (every other
  column, renumbered into x_all) is added.  The overlap pays only when the
  halo is a small, clustered part of the rows: widely scattered halo columns
  make a plan of nearly one-value blocks, and the second launch and the sum
  cost more than the exchange they hide.

No reduction on y is needed: each rank's rows are its own.  The adjoint
g_x = A^T g is the other way round: every rank's rows touch every column, so
each rank computes the partial A_rows^T g_rows in the padded layout (on the
transposed CB layout of its plans) and one reduce-scatter (sum) hands each
rank its own x range.  Every part is an ordinary CB plan (the reference's
coo2block_gather + cb_spmv per rank), so a rank runs the single-GPU kernels
unchanged.  staging="host" runs the exchange through host memory (for a
process group whose backend has no device transport, e.g. gloo).
"""
from __future__ import annotations

import numpy as np

from .gen import Coo


def block_row_bounds(coo: Coo, parts: int, bs: int = 16) -> np.ndarray:
    """Row cuts 0 = b[0] <= ... <= b[parts] = m on multiples of bs (m at the
    end), each part holding about nnz / parts stored values: cut k is the
    first block row whose stored-value prefix reaches k * nnz / parts."""
    if parts < 1:
        raise ValueError("parts must be >= 1")
    nbr = (coo.m + bs - 1) // bs
    per = np.bincount(np.asarray(coo.row, np.int64) // bs, minlength=nbr)
    prefix = np.concatenate([[0], np.cumsum(per)])  # stored values before block row i
    cuts = [0]
    for k in range(1, parts):
        br = int(np.searchsorted(prefix, k * coo.nnz / parts, side="left"))
        cuts.append(max(cuts[-1], min(br * bs, coo.m)))
    cuts.append(coo.m)
    return np.asarray(cuts, np.int64)


def even_bounds(n: int, parts: int, bs: int = 16) -> np.ndarray:
    """Cuts of [0, n) into `parts` ranges of whole blocks, as equal as they
    can be (x of a rectangular matrix)."""
    nb = (n + bs - 1) // bs
    cuts = [min(n, (nb * k // parts) * bs) for k in range(parts)] + [n]
    return np.asarray(cuts, np.int64)


def rows_of(coo: Coo, lo: int, hi: int) -> Coo:
    """Rows [lo, hi) of a row-sorted COO, renumbered from 0."""
    a, b = np.searchsorted(coo.row, [lo, hi], side="left")
    return Coo(int(hi - lo), coo.n, (coo.row[a:b] - lo).astype(np.int32),
               coo.col[a:b].copy(), coo.val[a:b].copy())


def split_columns(rows: Coo, cb: np.ndarray, rank: int):
    """(A_own, A_halo) of one rank's rows: A_own holds the columns in
    [cb[rank], cb[rank+1]) renumbered from 0; A_halo the others, renumbered
    into the padded all-gather layout (range s at s * L, L = the longest
    range).  Row order, and so the builder's input order, is kept."""
    lo, hi = int(cb[rank]), int(cb[rank + 1])
    L = int(np.max(np.diff(cb))) if len(cb) > 1 else 0
    col = rows.col.astype(np.int64)
    own = (col >= lo) & (col < hi)
    a = Coo(rows.m, hi - lo, rows.row[own].copy(), (col[own] - lo).astype(np.int32),
            rows.val[own].copy())
    hc = col[~own]
    s = np.searchsorted(cb, hc, side="right") - 1  # the range holding each column
    padded = s * L + (hc - cb[s])
    world = len(cb) - 1
    h = Coo(rows.m, world * L, rows.row[~own].copy(), padded.astype(np.int32),
            rows.val[~own].copy())
    return a, h


def padded_columns(rows: Coo, cb: np.ndarray) -> Coo:
    """One rank's rows with every column renumbered into the padded
    all-gather layout (range s at s * L)."""
    L = int(np.max(np.diff(cb)))
    col = rows.col.astype(np.int64)
    s = np.searchsorted(cb, col, side="right") - 1
    return Coo(rows.m, (len(cb) - 1) * L, rows.row.copy(),
               (s * L + (col - cb[s])).astype(np.int32), rows.val.copy())


class RowShard:
    """One rank's share of y = A x: plans for A_own and A_halo.

    coo: the whole matrix (every rank passes the same one and keeps its own
    rows); bounds: row cuts (default: block_row_bounds); cbounds: x cuts
    (default: the row cuts when A is square, else even_bounds); overlap:
    own + halo plans instead of one.  Plan options (block_size, value_type,
    ...) pass through to the plans."""

    def __init__(self, coo: Coo, world: int, rank: int, bounds=None, cbounds=None,
                 overlap: bool = False, **plan_opts):
        from . import Plan
        bs = int(plan_opts.get("block_size", 16) or 16)
        self.world, self.rank = world, rank
        self.bounds = np.asarray(bounds if bounds is not None
                                 else block_row_bounds(coo, world, bs), np.int64)
        if cbounds is None:
            cbounds = self.bounds if coo.m == coo.n else even_bounds(coo.n, world, bs)
        self.cbounds = np.asarray(cbounds, np.int64)
        self.r0, self.r1 = int(self.bounds[rank]), int(self.bounds[rank + 1])
        self.c0, self.c1 = int(self.cbounds[rank]), int(self.cbounds[rank + 1])
        self.L = int(np.max(np.diff(self.cbounds)))
        self.m, self.n = coo.m, coo.n
        self.overlap = bool(overlap) and world > 1
        rows = rows_of(coo, self.r0, self.r1)
        self.own = self.halo = self.full = None
        if self.overlap:
            own, halo = split_columns(rows, self.cbounds, rank)
            self.own_coo, self.halo_coo = own, halo
            self.own = Plan(own, **plan_opts)
            self.halo = Plan(halo, **plan_opts) if halo.nnz else None
            self.f32 = self.own.f32
        else:
            self.full_coo = padded_columns(rows, self.cbounds) if world > 1 else rows
            self.full = Plan(self.full_coo, **plan_opts)
            self.f32 = self.full.f32

    def pad(self, x_own):
        """This rank's x range padded to L rows (the all-gather piece)."""
        import torch
        shape = (self.L,) + tuple(x_own.shape[1:])
        xp = torch.zeros(shape, dtype=x_own.dtype, device=x_own.device)
        xp[: x_own.shape[0]] = x_own
        return xp

    def _gather(self, x_own, group, staging):
        """The padded ranges of every rank end to end (every rank takes part)
        and the async work handle (device staging) or None."""
        import torch
        import torch.distributed as dist
        piece = self.pad(x_own)
        shape = (self.world * self.L,) + tuple(piece.shape[1:])
        if staging == "host":
            host = torch.empty(shape, dtype=piece.dtype)
            dist.all_gather_into_tensor(host, piece.cpu(), group=group)
            return host.to(x_own.device), None
        x_all = torch.empty(shape, dtype=piece.dtype, device=piece.device)
        work = dist.all_gather_into_tensor(x_all, piece, group=group, async_op=True)
        return x_all, work

    def spmv_t(self, g_own, gx=None, group=None, staging="device"):
        """gx (this rank's x range, (c1 - c0,) or (c1 - c0, k)) = (A^T g) on
        that range, from g_own (this rank's rows of g).  The plans need
        want_transpose.  Partial A_rows^T g_own in the padded layout, then a
        reduce-scatter over the ranks (every rank takes part); staging="host"
        sums through host memory (all-reduce, then this rank's range)."""
        import torch
        k = 1 if g_own.dim() == 1 else g_own.shape[1]
        if self.world == 1:
            part = self.full.spmv_t(g_own)
        else:
            part = torch.zeros((self.world * self.L,) + tuple(g_own.shape[1:]),
                               dtype=g_own.dtype, device=g_own.device)
            if self.full is not None:
                part += self.full.spmv_t(g_own)
            else:
                part[self.rank * self.L: self.rank * self.L + self.c1 - self.c0] += \
                    self.own.spmv_t(g_own)
                if self.halo is not None:
                    part += self.halo.spmv_t(g_own)
        width = self.c1 - self.c0
        if gx is None:
            gx = torch.empty((width,) if g_own.dim() == 1 else (width, k), dtype=g_own.dtype,
                             device=g_own.device)
        if self.world == 1:
            gx.copy_(part[:width])
            return gx
        import torch.distributed as dist
        if staging == "host":
            host = part.cpu()
            dist.all_reduce(host, group=group)
            gx.copy_(host[self.rank * self.L: self.rank * self.L + width].to(gx.device))
            return gx
        mine = torch.empty((self.L,) + tuple(part.shape[1:]), dtype=part.dtype,
                           device=part.device)
        dist.reduce_scatter_tensor(mine, part, group=group)
        gx.copy_(mine[:width])
        return gx

    def spmv(self, x_own, y=None, group=None, x_all=None, staging="device"):
        """y (this rank's rows) = A x on the current stream.  x_own: this
        rank's x range (CUDA tensor, (c1 - c0,) or (c1 - c0, k)).  Without
        `x_all`, every rank of `group` (a torch process group; None = the
        default one) takes part in the all-gather of the padded ranges --
        also a rank whose rows need no halo, so the ranks' collectives stay
        in step -- and it overlaps A_own x_own.  With `x_all` (the padded
        ranges of every rank laid end to end) there is no collective.
        staging="host": the all-gather runs through host memory."""
        import torch
        k = 1 if x_own.dim() == 1 else x_own.shape[1]
        if y is None:
            y = torch.empty((self.r1 - self.r0,) if x_own.dim() == 1
                            else (self.r1 - self.r0, k), dtype=x_own.dtype,
                            device=x_own.device)
        work = None
        if x_all is None and self.world > 1:
            x_all, work = self._gather(x_own, group, staging)
        if self.full is not None:
            if work is not None:
                work.wait()  # the current stream waits for the gathered x
            return self.full.spmv(x_own if self.world == 1 else x_all, y)
        self.own.spmv(x_own, y)
        if work is not None:
            work.wait()
        if self.halo is not None:
            y.add_(self.halo.spmv(x_all))
        return y
