"""The N > 1 path on CPU: two gloo ranks line up and time a step as the
maximum over ranks (cbspmv.dist, used by bench.py), and each rank builds its
own replica of a plan with identical structure."""
import os
import socket

import pytest


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
    import numpy as np
    import cbspmv
    from cbspmv import gen
    from cbspmv.dist import Group
    g = Group("gloo", timeout_s=60)
    g.barrier()
    mx = g.max(1.5 + rank)          # per-rank "step time"
    p = cbspmv.Plan(gen.laplacian_2d(32, 32))
    d = p.export()
    digest = float(np.sum(d["gb_col_idx"]) + d["gb_nnzb"])
    same = g.max(digest) == digest  # every replica built the same structure
    g.close()
    out.put((rank, mx, same))


@pytest.mark.timeout(120)
def test_two_ranks_max_and_replicas():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=100) for _ in procs)
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [2.5, 2.5]
    assert all(r[2] for r in res)
