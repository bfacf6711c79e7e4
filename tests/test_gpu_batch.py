"""Batches and several right-hand sides on the GPU, against the oracle.

The batch entry points (cbspmv_batch_*) have no counterpart in the reference;
each matrix's result is checked against the oracle's long-double restatement
of the reference's CPU SpMV (cb-spmv-dcu/src/utils.h:98-111), one right-hand
side at a time, with the per-row bound of test_gpu_spmv.py.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = {False: 1e-12, True: 1e-5}


def _check(y, yref, absrow, f32, what):
    err = np.abs(np.asarray(y, np.float64) - yref)
    bound = TOL[f32] * absrow + (1e-300 if not f32 else 1e-30)
    worst = float(np.max(err / bound)) if err.size else 0.0
    assert worst <= 1.0, f"{what}: error {worst:.3g} x tolerance"


def _x(coo, nrhs, seed, f32):
    from cbspmv import gen
    X = gen.uniform_x(coo.n, seed, nrhs=max(nrhs, 2))[:nrhs]  # (nrhs, n)
    if f32:
        X = X.astype(np.float32).astype(np.float64)
    return X


def _small_batch(seed=4, count=24):
    from cbspmv import gen
    items = gen.batch_uneven(count=count, seed=seed, nmin=200, nmax=6000)
    rng = np.random.default_rng(seed)
    # a matrix with no entries and one with more than 32 right-hand sides
    items.append(gen.BatchItem("empty", gen.Coo(50, 40, np.zeros(0, np.int32),
                                                np.zeros(0, np.int32), np.zeros(0)), 3))
    items.append(gen.BatchItem("wide", gen.random_small(rng, 300, 200, 3000), 35))
    return items


@pytest.mark.parametrize("bs", [16, 32])
@pytest.mark.parametrize("f32", [False, True])
def test_batch_matches_oracle(cuda, bs, f32):
    import torch
    import cbspmv
    import cbdump as cd
    items = _small_batch()
    dt = torch.float32 if f32 else torch.float64
    plans = [cbspmv.Plan(it.coo, block_size=bs, value_type=int(f32),
                         tile_entries=(64 if i % 3 == 0 else 0))
             for i, it in enumerate(items)]
    xs, refs = [], []
    for i, it in enumerate(items):
        X = _x(it.coo, it.nrhs, 100 + i, f32)
        refs.append(cd.oracle_spmm_ld(it.coo, X))
        xs.append(torch.from_numpy(np.ascontiguousarray(X.T)).to(cuda, dt))
    ys = [torch.full((it.coo.m, it.nrhs), float("nan"), dtype=dt, device=cuda)
          for it in items]
    b = cbspmv.Batch(plans, [it.nrhs for it in items]).bind(xs, ys)

    def verify(how):
        torch.cuda.synchronize()
        for i, it in enumerate(items):
            yref, ab = refs[i]
            _check(ys[i].cpu().numpy().T, yref, ab, f32, f"{how} #{i} {it.kind}")

    def clear():
        for y in ys:
            y.fill_(float("nan"))

    for how, fn in (("run", b.run), ("run_each", b.run_each),
                    ("graph", lambda: b.graph_launch(False)),
                    ("graph_each", lambda: b.graph_launch(True))):
        for rep in range(2):  # repeated launches reuse the split-row counters
            clear()
            fn()
            verify(f"{how} {rep}")


def test_batch_rebind_and_errors(cuda):
    import torch
    import cbspmv
    import cbdump as cd
    from cbspmv import gen
    coos = [gen.laplacian_2d(20, 30), gen.power_law(3000, kmax=3000, band=128, seed=2)]
    plans = [cbspmv.Plan(c) for c in coos]
    b = cbspmv.Batch(plans, [1, 4])
    with pytest.raises(cbspmv.CBSpMVError) as e:
        b.run()
    assert e.value.status == "STATE"
    for seed in (1, 2):  # a re-bind redirects both the kernel and the graphs
        Xs = [_x(c, k, seed + 10 * i, False) for i, (c, k) in enumerate(zip(coos, [1, 4]))]
        xs = [torch.from_numpy(np.ascontiguousarray(X.T)).to(cuda) for X in Xs]
        ys = [torch.zeros((c.m, k), dtype=torch.float64, device=cuda)
              for c, k in zip(coos, [1, 4])]
        b.bind(xs, ys)
        for per_matrix in (False, True):
            for y in ys:
                y.zero_()
            b.graph_launch(per_matrix)
            torch.cuda.synchronize()
            for c, X, y in zip(coos, Xs, ys):
                yref, ab = cd.oracle_spmm_ld(c, X)
                _check(y.cpu().numpy().T, yref, ab, False, f"rebind {seed}")
    f32plan = cbspmv.Plan(coos[0], value_type=1)
    with pytest.raises(cbspmv.CBSpMVError) as e:
        cbspmv.Batch([plans[0], f32plan], [1, 1])
    assert e.value.status == "INVALID"


def _mrhs_cases():
    from cbspmv import gen
    rng = np.random.default_rng(17)
    return [
        ("rand-mid", gen.random_small(rng, 1000, 800, 20000)),
        ("rand-dense", gen.random_small(rng, 100, 100, 9000)),
        ("dense-dups", gen.random_small(rng, 64, 64, 40000, dup=True)),
        ("ragged", gen.random_small(rng, 37, 41, 1500, dup=True)),
        ("lap64", gen.laplacian_2d(64, 64)),
        ("st6", gen.stencil_27pt(6)),
        ("pl8192", gen.power_law(8192, kmax=8192, band=512, seed=11)),
        ("banded", gen.banded(rng, 3000, 40)),
    ]


MRHS = _mrhs_cases()


@pytest.mark.parametrize("name,coo", MRHS, ids=[c[0] for c in MRHS])
@pytest.mark.parametrize("bs", [16, 32])
@pytest.mark.parametrize("f32", [False, True])
@pytest.mark.parametrize("nrhs", [3, 8, 33])
def test_multi_rhs_kernel(cuda, name, coo, bs, f32, nrhs):
    """Y = A X through the multi-right-hand-side kernel, contiguous and with
    leading dimensions larger than nrhs, split rows included."""
    import torch
    import cbspmv
    import cbdump as cd
    dt = torch.float32 if f32 else torch.float64
    plan = cbspmv.Plan(coo, block_size=bs, value_type=int(f32), tile_entries=64).upload()
    X = _x(coo, nrhs, 5, f32)
    yref, ab = cd.oracle_spmm_ld(coo, X)
    ldx, ldy = nrhs + 3, nrhs + 1
    xd = torch.zeros((coo.n, ldx), dtype=dt, device=cuda)
    xd[:, :nrhs] = torch.from_numpy(np.ascontiguousarray(X.T)).to(cuda, dt)
    yd = torch.full((coo.m, ldy), float("nan"), dtype=dt, device=cuda)
    for _ in range(2):
        cbspmv._check(cbspmv.lib().cbspmv_spmv(plan._h, cbspmv._dptr(xd), cbspmv._dptr(yd),
                                               nrhs, ldx, ldy, cbspmv._stream(None)))
        torch.cuda.synchronize()
        got = yd.cpu().numpy()
        _check(got[:, :nrhs].T, yref, ab, f32, f"{name} nrhs={nrhs}")
        assert np.isnan(got[:, nrhs:]).all(), "wrote outside the nrhs columns"
