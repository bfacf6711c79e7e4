"""GPU parity of the balanced (non-row-owned) schedule -- plans built with
row_owned = 0, one right-hand side, kernel 6 or automatic -- against the
oracle (per row |y - y_ref| <= tol * sum |a x|; tol 1e-12 FP64, 1e-5 FP32:
the atomics change the order of the sums, not their bound), after new
values too; several right-hand sides and A^T x of the same plans keep their
own kernels."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = {False: 1e-12, True: 1e-5}


def _cases():
    from cbspmv import gen
    rng = np.random.default_rng(43)
    return [("random", gen.random_small(rng, 3000, 2500, 40000)),
            ("small", gen.random_small(rng, 300, 200, 2000)),
            ("power-law", gen.power_law(1 << 14, seed=7)),
            ("dense-dups", gen.random_small(rng, 64, 64, 40000, dup=True)),
            ("stencil", gen.stencil_27pt(10)),
            ("banded", gen.banded(rng, 5000, 40))]


CASES = _cases()


def _check(y, yref, absrow, f32, what):
    err = np.abs(np.asarray(y, np.float64) - yref)
    bound = TOL[f32] * absrow + (1e-30 if f32 else 1e-300)
    worst = float(np.max(err / bound)) if err.size else 0.0
    assert worst <= 1.0, f"{what}: error {worst:.3g} x tolerance"


@pytest.mark.parametrize("name,coo", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("f32", [False, True])
@pytest.mark.parametrize("kernel", [0, 6])
@pytest.mark.parametrize("bs", [16, 32])
def test_balanced_schedule(cuda, name, coo, f32, kernel, bs):
    import torch
    import cbspmv
    import cbdump as cd
    from cbspmv import gen
    plan = cbspmv.Plan(coo, value_type=int(f32), block_size=bs, row_owned=0, kernel=kernel,
                       want_transpose=1)
    dt = torch.float32 if f32 else torch.float64
    x = gen.uniform_x(coo.n, 11)
    if f32:
        x = x.astype(np.float32).astype(np.float64)
    xd = torch.from_numpy(x).to(cuda, dt)
    y = torch.full((coo.m,), float("nan"), dtype=dt, device=cuda)
    for _ in range(2):  # y is zeroed by each call, not accumulated
        plan.spmv(xd, y)
    torch.cuda.synchronize()
    yref, ab = cd.oracle_spmm_ld(coo, x[None, :])
    _check(y.cpu().numpy()[None, :], yref, ab, f32, f"{name} kernel {kernel}")
    # new values reach the balanced copy
    rng = np.random.default_rng(5)
    vals = rng.standard_normal(coo.nnz)
    if f32:
        vals = vals.astype(np.float32).astype(np.float64)
    plan.set_values(torch.from_numpy(vals).to(cuda, dt))
    coo2 = gen.Coo(coo.m, coo.n, coo.row, coo.col, vals)
    y2 = plan.spmv(xd)
    X = gen.uniform_x(coo.n, 12, nrhs=3)
    if f32:
        X = X.astype(np.float32).astype(np.float64)
    Y = plan.spmv(torch.from_numpy(np.ascontiguousarray(X.T)).to(cuda, dt))
    g = gen.uniform_x(coo.m, 13)
    if f32:
        g = g.astype(np.float32).astype(np.float64)
    gx = plan.spmv_t(torch.from_numpy(g).to(cuda, dt))
    torch.cuda.synchronize()
    yref2, ab2 = cd.oracle_spmm_ld(coo2, x[None, :])
    _check(y2.cpu().numpy()[None, :], yref2, ab2, f32, f"{name} after set_values")
    Yref, Ab = cd.oracle_spmm_ld(coo2, X)
    _check(Y.cpu().numpy().T, Yref, Ab, f32, f"{name} 3 rhs")
    gref, gab = cd.oracle_spmm_ld(coo2, g[None, :], transpose=True)
    _check(gx.cpu().numpy()[None, :], gref, gab, f32, f"{name} transpose")
    plan.check()
    if kernel == 0:
        k, _ = plan.autotune(1)
        assert k in (1, 2, 3, 5, 6)
