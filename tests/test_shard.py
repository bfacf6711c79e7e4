"""Block-row sharding of one matrix (cbspmv.shard): the cuts, the split of a
rank's rows into own and halo columns, and the padded all-gather layout,
checked on CPU against the oracle's SpMV (tests/cbdump.py); the exchange
itself between two gloo ranks; the per-rank plans on the GPU with the ranks
run one after another in one process (their all-gathered x laid out by
hand, no collective)."""
import os
import socket

import numpy as np
import pytest


def _cases():
    from cbspmv import gen
    rng = np.random.default_rng(9)
    return [("pl", gen.power_law(6000, kmax=3000, band=300, seed=5, mean=12)),
            ("lap", gen.laplacian_2d(40, 50)),
            ("rect", gen.random_small(rng, 700, 1300, 9000)),
            ("tiny", gen.random_small(rng, 20, 20, 60))]


CASES = _cases()


def _x_all(coo, cb, x):
    """The padded all-gather layout of x (ranges of length L end to end)."""
    L = int(np.max(np.diff(cb)))
    out = np.zeros((len(cb) - 1) * L)
    for s in range(len(cb) - 1):
        out[s * L: s * L + cb[s + 1] - cb[s]] = x[cb[s]:cb[s + 1]]
    return out


@pytest.mark.parametrize("name,coo", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("world", [1, 2, 3, 8])
@pytest.mark.parametrize("bs", [16, 32])
def test_cuts_split_and_layout(name, coo, world, bs):
    import cbdump as cd
    from cbspmv import shard
    rb = shard.block_row_bounds(coo, world, bs)
    assert rb[0] == 0 and rb[-1] == coo.m and np.all(np.diff(rb) >= 0)
    assert all(c % bs == 0 or c == coo.m for c in rb)
    # balance: each part within one block row's stored values of nnz / world
    per_br = np.bincount(coo.row // bs, minlength=(coo.m + bs - 1) // bs)
    counts = np.diff(np.searchsorted(coo.row, rb))
    assert np.all(np.abs(counts - coo.nnz / world) <= per_br.max() + 1)
    cb = rb if coo.m == coo.n else shard.even_bounds(coo.n, world, bs)
    assert cb[0] == 0 and cb[-1] == coo.n and np.all(np.diff(cb) >= 0)
    x = np.random.default_rng(1).uniform(-1, 1, coo.n)
    xa = _x_all(coo, cb, x)
    yref = cd.oracle_spmv(coo, x)
    for r in range(world):
        rows = shard.rows_of(coo, rb[r], rb[r + 1])
        own, halo = shard.split_columns(rows, cb, r)
        assert own.nnz + halo.nnz == rows.nnz
        assert np.all(np.diff(own.row) >= 0) and np.all(np.diff(halo.row) >= 0)
        y = cd.oracle_spmv(own, x[cb[r]:cb[r + 1]]) + cd.oracle_spmv(halo, xa)
        assert np.allclose(y, yref[rb[r]:rb[r + 1]], rtol=1e-12, atol=1e-12)
        full = shard.padded_columns(rows, cb)
        assert np.allclose(cd.oracle_spmv(full, xa), yref[rb[r]:rb[r + 1]],
                           rtol=1e-12, atol=1e-12)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port),
                      WORLD_SIZE=str(world), RANK=str(rank), LOCAL_RANK=str(rank))
    import sys
    import pathlib
    repo = pathlib.Path(__file__).resolve().parent.parent
    sys.path.insert(0, str(repo / "cb-sparse-dcu_b200"))
    sys.path.insert(0, str(repo / "tests"))
    import torch
    import torch.distributed as dist
    import cbdump as cd
    from cbspmv import gen, shard
    dist.init_process_group("gloo", timeout=__import__("datetime").timedelta(seconds=60))
    coo = gen.power_law(5000, kmax=2500, band=200, seed=6, mean=10)
    x = np.random.default_rng(2).uniform(-1, 1, coo.n)
    want = cd.oracle_spmv(coo, x)
    ok = True
    for overlap in (False, True):  # the plans are built on the host
        sh = shard.RowShard(coo, world, rank, overlap=overlap)
        piece = sh.pad(torch.from_numpy(x[sh.c0:sh.c1].copy()))
        x_all = torch.empty(world * sh.L, dtype=piece.dtype)
        dist.all_gather_into_tensor(x_all, piece)
        if overlap:
            y = cd.oracle_spmv(sh.own_coo, x[sh.c0:sh.c1])
            if sh.halo is not None:
                y = y + cd.oracle_spmv(sh.halo_coo, x_all.numpy())
        else:
            y = cd.oracle_spmv(sh.full_coo, x_all.numpy())
        ok = ok and np.allclose(y, want[sh.r0:sh.r1], rtol=1e-12, atol=1e-12)
    had_halo = sh.halo is not None
    # the adjoint's exchange: partial A_rows^T g in the padded layout, summed
    # over the ranks (all-reduce here; reduce-scatter on NCCL), own range kept
    g = np.random.default_rng(3).uniform(-1, 1, coo.m)
    gref = cd.oracle_spmm_ld(coo, g[None, :], transpose=True)[0][0]
    sh = shard.RowShard(coo, world, rank)
    part = cd.oracle_spmm_ld(sh.full_coo, g[None, sh.r0:sh.r1], transpose=True)[0][0]
    tot = torch.from_numpy(part.copy())
    dist.all_reduce(tot)
    mine = tot.numpy()[rank * sh.L: rank * sh.L + sh.c1 - sh.c0]
    ok = ok and np.allclose(mine, gref[sh.c0:sh.c1], rtol=1e-12, atol=1e-12)
    dist.barrier()
    dist.destroy_process_group()
    out.put((rank, bool(ok), had_halo))


@pytest.mark.timeout(180)
def test_two_ranks_exchange_x():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=150) for _ in procs)
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [True, True]
    assert any(r[2] for r in res)  # the halo part was exercised


@pytest.mark.gpu
@pytest.mark.parametrize("name,coo", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("world", [1, 3])
@pytest.mark.parametrize("f32", [False, True])
@pytest.mark.parametrize("nrhs", [1, 4])
@pytest.mark.parametrize("overlap", [False, True])
def test_row_shards_on_gpu(cuda, name, coo, world, f32, nrhs, overlap):
    import torch
    import cbdump as cd
    from cbspmv import gen, shard
    dt = torch.float32 if f32 else torch.float64
    X = gen.uniform_x(coo.n, 3, nrhs=max(nrhs, 2))[:nrhs]
    if f32:
        X = X.astype(np.float32).astype(np.float64)
    yref, ab = cd.oracle_spmm_ld(coo, X)
    shards = [shard.RowShard(coo, world, r, overlap=overlap, value_type=int(f32))
              for r in range(world)]
    xd = torch.from_numpy(np.ascontiguousarray(X.T)).to(cuda, dt)
    if nrhs == 1:
        xd = xd[:, 0].contiguous()
    x_all = torch.cat([s.pad(xd[s.c0:s.c1]) for s in shards]) if world > 1 else None
    ys = [s.spmv(xd[s.c0:s.c1].contiguous(), x_all=x_all) for s in shards]
    torch.cuda.synchronize()
    y = torch.cat(ys).cpu().numpy().reshape(coo.m, nrhs).T
    tol = 1e-5 if f32 else 1e-12
    assert np.all(np.abs(y - yref) <= tol * ab + 1e-300)


def _gpu_rank(rank, world, port, out):
    """One rank of a two-process run on one GPU: its own plans, its own
    exchange (gloo, staged through host memory), forward and adjoint."""
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port),
                      WORLD_SIZE=str(world), RANK=str(rank), LOCAL_RANK=str(rank))
    import sys
    import pathlib
    repo = pathlib.Path(__file__).resolve().parent.parent
    sys.path.insert(0, str(repo / "cb-sparse-dcu_b200"))
    sys.path.insert(0, str(repo / "tests"))
    import torch
    import torch.distributed as dist
    import cbdump as cd
    from cbspmv import gen, shard
    dist.init_process_group("gloo", timeout=__import__("datetime").timedelta(seconds=60))
    dev = torch.device("cuda:0")
    coo = gen.power_law(20000, kmax=4000, band=600, seed=6, mean=12)
    X = gen.uniform_x(coo.n, 4, nrhs=3)  # (3, n)
    G = gen.uniform_x(coo.m, 5, nrhs=3)
    errs = []
    for nrhs in (1, 3):
        Xk, Gk = X[:nrhs], G[:nrhs]
        yref, ab = cd.oracle_spmm_ld(coo, Xk)
        gref, gab = cd.oracle_spmm_ld(coo, Gk, transpose=True)
        for overlap in (False, True):
            sh = shard.RowShard(coo, world, rank, overlap=overlap, want_transpose=1)
            x_own = torch.from_numpy(np.ascontiguousarray(Xk[:, sh.c0:sh.c1].T)).to(dev)
            g_own = torch.from_numpy(np.ascontiguousarray(Gk[:, sh.r0:sh.r1].T)).to(dev)
            if nrhs == 1:
                x_own, g_own = x_own[:, 0].contiguous(), g_own[:, 0].contiguous()
            y = sh.spmv(x_own, staging="host").cpu().numpy().reshape(-1, nrhs).T
            gx = sh.spmv_t(g_own, staging="host").cpu().numpy().reshape(-1, nrhs).T
            e1 = np.max(np.abs(y - yref[:, sh.r0:sh.r1]) / (ab[:, sh.r0:sh.r1] + 1e-300))
            e2 = np.max(np.abs(gx - gref[:, sh.c0:sh.c1]) / (gab[:, sh.c0:sh.c1] + 1e-300))
            errs.append(float(max(e1, e2)))
    dist.barrier()
    dist.destroy_process_group()
    out.put((rank, max(errs)))


@pytest.mark.gpu
@pytest.mark.timeout(300)
def test_two_processes_share_one_gpu(cuda):
    """Two ranks as two processes on the one GPU, each running RowShard's own
    exchange (gloo, through host memory) around its own kernels -- forward
    y = A x (all-gather of x) and adjoint A^T g (sum of the partials, each rank
    keeping its range) -- checked against the oracle.  The kernels of the two
    processes never wait on each other."""
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_gpu_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=280) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert all(e <= 1e-12 for _, e in res), res
