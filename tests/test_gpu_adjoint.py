"""GPU checks of the adjoint: g_x = A^T g on the transposed CB layout, the
value gradient, and the autograd harness (FP64 reference gradients and
central finite differences on an n=4,096 power-law instance)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _plan(coo, f32=False, **kw):
    import cbspmv
    return cbspmv.Plan(coo, value_type=int(f32), want_transpose=1, **kw)


@pytest.mark.parametrize("bs", [16, 32])
@pytest.mark.parametrize("f32", [False, True])
@pytest.mark.parametrize("nrhs", [1, 3, 4, 8, 16, 33])
def test_transpose_and_value_gradient(cuda, bs, f32, nrhs):
    import torch
    import cbdump as cd
    from cbspmv import gen
    coo = gen.power_law(4096, kmax=4096, band=256, seed=3, mean=24)
    plan = _plan(coo, f32, block_size=bs, tile_entries=128)
    dt = torch.float32 if f32 else torch.float64
    tol = 1e-5 if f32 else 1e-12
    G = gen.uniform_x(coo.m, 21, nrhs=max(nrhs, 2))[:nrhs]
    X = gen.uniform_x(coo.n, 22, nrhs=max(nrhs, 2))[:nrhs]
    if f32:
        G = G.astype(np.float32).astype(np.float64)
        X = X.astype(np.float32).astype(np.float64)
    gd = torch.from_numpy(np.ascontiguousarray(G.T)).to(cuda, dt)
    xd = torch.from_numpy(np.ascontiguousarray(X.T)).to(cuda, dt)
    if nrhs == 1:
        gd, xd = gd[:, 0].contiguous(), xd[:, 0].contiguous()
    gx = plan.spmv_t(gd).cpu().numpy().reshape(coo.n, nrhs).T
    ref, ab = cd.oracle_spmm_ld(coo, G, transpose=True)
    assert np.all(np.abs(gx - ref) <= tol * ab + 1e-300)
    gv = plan.grad_vals(gd, xd).cpu().numpy().astype(np.float64)
    gin = gv[plan.input_slots()]
    want = cd.oracle_grad_vals(coo, G, X)
    scale = np.sum(np.abs(G[:, coo.row] * X[:, coo.col]), axis=0)
    assert np.all(np.abs(gin - want) <= tol * scale + 1e-300)
    # the combined call runs the same kernels: identical results
    gx2, gv2 = plan.adjoint(gd, xd)
    torch.cuda.synchronize()
    assert np.array_equal(gx2.cpu().numpy().reshape(coo.n, nrhs).T, gx)
    assert np.array_equal(gv2.cpu().numpy().astype(np.float64), gv)


@pytest.mark.parametrize("f32", [False, True])
@pytest.mark.parametrize("nrhs", [1, 8, 33])
def test_value_gradient_sparse_rows(cuda, f32, nrhs):
    """About one stored value per row: a block of the value-gradient kernel
    sees more g rows than it stages in shared memory and reads g directly."""
    import torch
    import cbdump as cd
    from cbspmv import gen
    rng = np.random.default_rng(12)
    coo = gen.random_small(rng, 5000, 4000, 5000)
    plan = _plan(coo, f32)
    dt = torch.float32 if f32 else torch.float64
    tol = 1e-5 if f32 else 1e-12
    G = gen.uniform_x(coo.m, 31, nrhs=max(nrhs, 2))[:nrhs]
    X = gen.uniform_x(coo.n, 32, nrhs=max(nrhs, 2))[:nrhs]
    if f32:
        G = G.astype(np.float32).astype(np.float64)
        X = X.astype(np.float32).astype(np.float64)
    gd = torch.from_numpy(np.ascontiguousarray(G.T)).to(cuda, dt)
    xd = torch.from_numpy(np.ascontiguousarray(X.T)).to(cuda, dt)
    gv = plan.grad_vals(gd, xd).cpu().numpy().astype(np.float64)
    want = cd.oracle_grad_vals(coo, G, X)
    scale = np.sum(np.abs(G[:, coo.row] * X[:, coo.col]), axis=0)
    assert np.all(np.abs(gv[plan.input_slots()] - want) <= tol * scale + 1e-300)


def test_adjoint_streams_graph_and_errors(cuda):
    """cbspmv_adjoint: the value gradient's second stream joins back before
    work issued later on the caller's stream; captured in a CUDA graph it
    replays with new inputs; bad calls return statuses."""
    import torch
    import cbspmv
    from cbspmv import gen
    coo = gen.power_law(20000, kmax=4000, band=512, seed=8, mean=20)
    plan = _plan(coo, True)
    k = 8
    g = torch.rand(coo.m, k, device=cuda)
    x = torch.rand(coo.n, k, device=cuda)
    gx_ref, gv_ref = plan.spmv_t(g), plan.grad_vals(g, x)
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        gx, gv = plan.adjoint(g, x, stream=s)
        both = torch.cat([gx.flatten(), gv])  # ordered after both outputs
    s.synchronize()
    assert torch.equal(both, torch.cat([gx_ref.flatten(), gv_ref]))
    gx.zero_()
    gv.zero_()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        plan.adjoint(g, x, gx, gv)
    for seed in range(2):
        torch.manual_seed(seed)
        g.copy_(torch.rand_like(g))
        x.copy_(torch.rand_like(x))
        graph.replay()
        torch.cuda.synchronize()
        assert torch.equal(gx, plan.spmv_t(g))
        assert torch.equal(gv, plan.grad_vals(g, x))
    del graph
    only_v = plan.adjoint(g, x, want_gx=False)
    assert only_v[0] is None and torch.equal(only_v[1], plan.grad_vals(g, x))
    with pytest.raises(cbspmv.CBSpMVError) as e:
        plan.adjoint(g, x, want_gx=False, want_gvals=False)
    assert e.value.status == "INVALID"
    no_t = cbspmv.Plan(coo, value_type=1)
    with pytest.raises(cbspmv.CBSpMVError) as e:
        no_t.adjoint(g, x)
    assert e.value.status == "STATE"
    assert no_t.adjoint(g, x, want_gx=False)[1].shape == (no_t.num_values(),)


def test_gradcheck_small(cuda):
    """torch.autograd.gradcheck on a small FP64 matrix with duplicates,
    dense and CSR blocks."""
    import torch
    import cbspmv
    from cbspmv import gen
    rng = np.random.default_rng(5)
    coo = gen.random_small(rng, 40, 36, 900, dup=True)
    plan = _plan(coo)
    vals = torch.from_numpy(coo.val.copy()).to(cuda).requires_grad_(True)
    x = torch.randn(36, 3, dtype=torch.float64, device=cuda, requires_grad=True)
    assert torch.autograd.gradcheck(
        lambda v, xx: cbspmv.cbspmv_apply(plan, v, xx), (vals, x),
        eps=1e-6, atol=1e-8, rtol=1e-6)


def test_finite_differences_n4096(cuda):
    """Loss 0.5 ||A X - T||^2 (8 right-hand sides): analytic gradients
    against the FP64 oracle gradient and central differences."""
    import torch
    import cbspmv
    import cbdump as cd
    from cbspmv import gen
    coo = gen.power_law(4096, kmax=4096, band=256, seed=3, mean=24)
    plan = _plan(coo)
    k = 8
    rng = np.random.default_rng(3)
    T = torch.from_numpy(rng.standard_normal((coo.m, k))).to(cuda)
    X0 = np.ascontiguousarray(gen.uniform_x(coo.n, 33, nrhs=k).T)
    vals = torch.from_numpy(coo.val.copy()).to(cuda).requires_grad_(True)
    X = torch.from_numpy(X0).to(cuda).requires_grad_(True)
    Y = cbspmv.cbspmv_apply(plan, vals, X)
    loss = 0.5 * ((Y - T) ** 2).sum()
    loss.backward()
    # FP64 oracle gradient: G = A X - T; dX = A^T G; dvals = G[row] . X[col]
    Yref, _ = cd.oracle_spmm_ld(coo, X0.T)
    G = Yref - T.cpu().numpy().T
    dX, abx = cd.oracle_spmm_ld(coo, G, transpose=True)
    dv = cd.oracle_grad_vals(coo, G, X0.T)
    assert np.allclose(X.grad.cpu().numpy().T, dX, rtol=1e-10, atol=1e-10 * abx.max())
    assert np.allclose(vals.grad.cpu().numpy(), dv, rtol=1e-10, atol=1e-10 * np.abs(dv).max())

    def loss_at(v, x):
        y, _ = cd.oracle_spmm_ld(gen.Coo(coo.m, coo.n, coo.row, coo.col, v), x.T)
        return 0.5 * np.sum((y - T.cpu().numpy().T) ** 2)

    h = 1e-6
    for idx in rng.choice(coo.nnz, 5, replace=False):
        vp, vm = coo.val.copy(), coo.val.copy()
        vp[idx] += h
        vm[idx] -= h
        fd = (loss_at(vp, X0) - loss_at(vm, X0)) / (2 * h)
        assert abs(fd - vals.grad[idx].item()) <= 1e-5 * max(1.0, abs(fd))
    for (i, j) in [(0, 0), (coo.n - 1, k - 1), (1234, 3)]:
        xp, xm = X0.copy(), X0.copy()
        xp[i, j] += h
        xm[i, j] -= h
        fd = (loss_at(coo.val, xp) - loss_at(coo.val, xm)) / (2 * h)
        assert abs(fd - X.grad[i, j].item()) <= 1e-5 * max(1.0, abs(fd))


@pytest.mark.parametrize("bs", [16, 32])
@pytest.mark.parametrize("f32", [False, True])
@pytest.mark.parametrize("nrhs", [1, 3, 8, 16, 21])
@pytest.mark.parametrize("name", ["pl", "mixed"])
@pytest.mark.parametrize("kernel", [0, 3])
def test_fused_adjoint(cuda, bs, f32, nrhs, name, kernel):
    """cbspmv_adjoint_fused: A^T g and the value gradient in one launch on the
    transposed layout -- its row-segment stream (kernel 0) or its tiles
    (kernel 3, no stream) -- against the FP64 oracle (COO, CSR and DENSE
    blocks; more than 16 right-hand sides in slabs whose gradients add)."""
    import torch
    import cbdump as cd
    from cbspmv import gen
    if name == "pl":
        coo = gen.power_law(4096, kmax=4096, band=256, seed=3, mean=24)
    else:  # stencil rows: CSR blocks, and dense couplings
        coo = gen.stencil_27pt(6)
    plan = _plan(coo, f32, block_size=bs, tile_entries=128, kernel=kernel)
    dt = torch.float32 if f32 else torch.float64
    tol = 1e-5 if f32 else 1e-12
    G = gen.uniform_x(coo.m, 41, nrhs=max(nrhs, 2))[:nrhs]
    X = gen.uniform_x(coo.n, 42, nrhs=max(nrhs, 2))[:nrhs]
    if f32:
        G = G.astype(np.float32).astype(np.float64)
        X = X.astype(np.float32).astype(np.float64)
    gd = torch.from_numpy(np.ascontiguousarray(G.T)).to(cuda, dt)
    xd = torch.from_numpy(np.ascontiguousarray(X.T)).to(cuda, dt)
    if nrhs == 1:
        gd, xd = gd[:, 0].contiguous(), xd[:, 0].contiguous()
    for _ in range(2):  # twice: the value gradient is stored, not accumulated
        gx, gpay = plan.adjoint_fused(gd, xd)
        torch.cuda.synchronize()
    gx = gx.cpu().numpy().reshape(coo.n, nrhs).T
    ref, ab = cd.oracle_spmm_ld(coo, G, transpose=True)
    assert np.all(np.abs(gx - ref) <= tol * ab + 1e-300)
    gin = gpay.cpu().numpy().astype(np.float64)[plan.grad_positions_t()]
    want = cd.oracle_grad_vals(coo, G, X)
    scale = np.sum(np.abs(G[:, coo.row] * X[:, coo.col]), axis=0)
    assert np.all(np.abs(gin - want) <= tol * scale + 1e-300)
