"""cbspmv_spmv_noalloc: SpMV for callers that may not allocate device memory
while they run (a framework plugin's execute step, a fixed-budget serving
loop).  Its scratch is a fixed 8 MiB array inside the library instead of the
plan's own allocations.  Checked through the C ABI against cbspmv_spmv on two
calls in a row, and against the oracle; a plan that needs more scratch than
the array holds is refused with a clear message.

Kept in a file of its own that pytest collects last.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = {False: 1e-12, True: 1e-5}


def _fn():
    import cbspmv
    f = cbspmv.lib().cbspmv_spmv_noalloc
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                  ctypes.c_int64, ctypes.c_int64, ctypes.c_void_p]
    return f


@pytest.mark.parametrize("f32", [False, True])
@pytest.mark.parametrize("nrhs,kernel", [(1, 0), (1, 2), (3, 0)])
def test_noalloc_matches_spmv(cuda, f32, nrhs, kernel):
    import torch
    import cbspmv
    import cbdump as cd
    from cbspmv import gen
    # small tiles: many block rows are split, so the partials and counters in
    # the fixed scratch are exercised
    coo = gen.power_law(1 << 15, kmax=4096, band=1024, seed=5)
    plan = cbspmv.Plan(coo, value_type=int(f32), tile_entries=64, kernel=kernel)
    assert plan.info()["split_rows"] > 0
    dt = torch.float32 if f32 else torch.float64
    X = gen.uniform_x(coo.n, 13, nrhs=max(nrhs, 2))[:nrhs]
    if f32:
        X = X.astype(np.float32).astype(np.float64)
    xd = torch.from_numpy(np.ascontiguousarray(X.T)).to(cuda, dt)
    if nrhs == 1:
        xd = xd[:, 0].contiguous()
    want = plan.spmv(xd)  # the existing entry point (uploads the plan)
    torch.cuda.synchronize()
    yref, ab = cd.oracle_spmm_ld(coo, X)
    fn = _fn()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    for call in range(2):
        y = torch.full_like(want, float("nan"))
        rc = fn(plan._h, ctypes.c_void_p(xd.data_ptr()), ctypes.c_void_p(y.data_ptr()),
                nrhs, nrhs, nrhs, stream)
        assert rc == 0, cbspmv.last_error()
        torch.cuda.synchronize()
        got = y.cpu().numpy().reshape(coo.m, nrhs).T.astype(np.float64)
        ref = want.cpu().numpy().reshape(coo.m, nrhs).T.astype(np.float64)
        assert np.all(np.abs(got - ref) <= TOL[f32] * ab + 1e-300), f"call {call}"
        assert np.all(np.abs(got - yref) <= TOL[f32] * ab + 1e-300), f"call {call}"
        # the plan's own entry point between the calls is unaffected
        y2 = plan.spmv(xd)
        torch.cuda.synchronize()
        got2 = y2.cpu().numpy().reshape(coo.m, nrhs).T.astype(np.float64)
        assert np.all(np.abs(got2 - yref) <= TOL[f32] * ab + 1e-300), f"spmv after {call}"


def test_noalloc_refuses_oversized_plan(cuda):
    import torch
    import cbspmv
    from cbspmv import gen
    coo = gen.power_law(1 << 19, seed=6)
    plan = cbspmv.Plan(coo, tile_entries=64)  # ~10^5 split tiles: > 8 MiB of partials
    x = torch.ones(coo.n, dtype=torch.float64, device=cuda)
    y = plan.spmv(x)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = _fn()(plan._h, ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(y.data_ptr()),
               1, 1, 1, stream)
    assert cbspmv.STATUS[rc] == "UNSUPPORTED"
    msg = cbspmv.last_error()
    assert "8388608" in msg and "bytes of scratch" in msg
