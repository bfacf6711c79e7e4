"""Device-side failure reporting, without a GPU fault.

Every mbarrier wait in the kernels is bounded; a wait that runs out sets the
plan's error word and its warp stops.  The tests make the waits run out on
purpose -- cbspmv_debug_wait_polls(0) gives every wait zero polls, so each one
gives up before its (legitimate, in-bounds) bulk copy is looked at; the kernel
still drains its copies in flight with the normal limit before it exits -- and
check that the host sees CBSPMV_ERR_DEVICE, that the plan's scratch is reset,
and that the next launches are exact again.  Nothing here faults, traps or
hangs the GPU: the kernel returns early and the context stays usable.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _plan_and_x(kernel, f32=False):
    import cbspmv
    from cbspmv import gen
    # rows long enough to be split over several tiles and warps
    coo = gen.power_law(16384, kmax=4000, band=1024, seed=5)
    plan = cbspmv.Plan(coo, kernel=kernel, value_type=int(f32), tile_entries=64)
    return coo, plan, gen.uniform_x(coo.n, 9)


def _err(y, coo, x):
    import cbdump as cd
    yref, ab = cd.oracle_spmm_ld(coo, x.T if x.ndim == 2 else x[None, :])
    yy = y.T if y.ndim == 2 else y[None, :]
    return float(np.max(np.abs(yy - yref) / (ab + 1e-300)))


@pytest.mark.parametrize("kernel,nrhs", [(1, 1), (3, 1), (3, 3)])
def test_giveup_is_reported_and_reset(cuda, kernel, nrhs):
    import torch
    import cbspmv
    coo, plan, x1 = _plan_and_x(kernel)
    x = np.stack([x1 * (j + 1) for j in range(nrhs)], 1) if nrhs > 1 else x1
    xd = torch.from_numpy(np.ascontiguousarray(x)).to(cuda)
    y = plan.spmv(xd)  # a normal launch first: exact
    plan.check()
    assert _err(y.cpu().numpy(), coo, x) <= 1e-12
    try:
        cbspmv.debug_wait_polls(0)
        y.fill_(float("nan"))
        plan.spmv(xd, y)
    finally:
        cbspmv.debug_wait_polls(-1)
    with pytest.raises(cbspmv.CBSpMVError) as ei:
        plan.check()
    assert ei.value.status == "DEVICE"
    assert np.isnan(y.cpu().numpy()).any()  # the launch stopped early
    plan.check()  # reported once
    for _ in range(3):  # counters were reset: every later launch is exact
        y.fill_(float("nan"))
        plan.spmv(xd, y)
        plan.check()
        assert _err(y.cpu().numpy(), coo, x) <= 1e-12


def test_giveup_refuses_next_launch(cuda):
    """A launching call that finds the error word set reports it instead of
    launching; the call after it runs normally."""
    import torch
    import cbspmv
    coo, plan, x = _plan_and_x(1)
    xd = torch.from_numpy(x).to(cuda)
    y = plan.spmv(xd)
    try:
        cbspmv.debug_wait_polls(0)
        plan.spmv(xd, y)
    finally:
        cbspmv.debug_wait_polls(-1)
    torch.cuda.synchronize()
    with pytest.raises(cbspmv.CBSpMVError) as ei:
        plan.spmv(xd, y)
    assert ei.value.status == "DEVICE"
    plan.spmv(xd, y)
    plan.check()
    assert _err(y.cpu().numpy(), coo, x) <= 1e-12


def test_giveup_host_call_reports(cuda):
    """The synchronous host-buffer call returns the status itself."""
    import cbspmv
    coo, plan, x = _plan_and_x(1)
    plan.spmv_host(x)
    try:
        cbspmv.debug_wait_polls(0)
        with pytest.raises(cbspmv.CBSpMVError) as ei:
            plan.spmv_host(x)
    finally:
        cbspmv.debug_wait_polls(-1)
    assert ei.value.status == "DEVICE"
    y = plan.spmv_host(x)
    assert _err(y, coo, x) <= 1e-12


def test_batch_giveup_is_reported_and_reset(cuda):
    """The same for the one-launch batch of the staged kernel (plans pinned
    to kernel 3 carry no row-segment stream, whose batch kernel has no waits):
    cbspmv_batch_check reports the give-up, the batch's scratch is reset, and
    the next launches are exact."""
    import torch
    import cbspmv
    import cbdump as cd
    from cbspmv import gen
    items = gen.batch_uneven(count=12, seed=6, nmin=500, nmax=20000)
    plans = [cbspmv.Plan(it.coo, tile_entries=64, kernel=3) for it in items]
    Xs = [np.ascontiguousarray(gen.uniform_x(it.coo.n, 50 + i, nrhs=max(it.nrhs, 2))[:it.nrhs].T)
          for i, it in enumerate(items)]
    xs = [torch.from_numpy(X).to(cuda) for X in Xs]
    ys = [torch.empty(it.coo.m, it.nrhs, dtype=torch.float64, device=cuda) for it in items]
    b = cbspmv.Batch(plans, [it.nrhs for it in items]).bind(xs, ys)

    def exact():
        for it, X, y in zip(items, Xs, ys):
            yref, ab = cd.oracle_spmm_ld(it.coo, X.T)
            assert np.all(np.abs(y.cpu().numpy().T - yref) <= 1e-12 * ab + 1e-300)

    b.run()
    b.check()
    exact()
    try:
        cbspmv.debug_wait_polls(0)
        b.run()
    finally:
        cbspmv.debug_wait_polls(-1)
    with pytest.raises(cbspmv.CBSpMVError) as ei:
        b.check()
    assert ei.value.status == "DEVICE"
    for _ in range(2):
        for y in ys:
            y.fill_(float("nan"))
        b.run()
        b.check()
        exact()
