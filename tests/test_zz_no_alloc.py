"""The allocation-free batched solve (ixb_tridiag_f64_noalloc) gives the
results of ixb_tridiag_f64 on two calls in a row.

It exists for callers that must not let a library allocate device memory
while they run (a driver whose GPU memory belongs to its OpenACC runtime or
to a pool reserved at start-up, a solver under a fixed memory budget on a
shared GPU, a loop that cannot afford the synchronisation an allocation may
cause).  Its interleaved layout keeps scratch in a fixed array of the
library's device image instead of asking the allocator.  This file is
collected last on purpose and needs nothing from the other tests.
"""
import numpy as np
import pytest

from ixchel2d_b200 import _ffi as F

pytestmark = pytest.mark.gpu

TOL = 1e-12  # hybrid solver; the exact solver must match bit for bit


@pytest.fixture(autouse=True)
def _need_gpu():
    if F.lib.ixb_device_count() < 1:
        pytest.skip("no CUDA device")


def _systems(n, nsys, seed):
    rng = np.random.default_rng(seed)
    a = rng.uniform(-1, 0, (nsys, n))
    c = rng.uniform(-1, 0, (nsys, n))
    b = np.abs(a) + np.abs(c) + rng.uniform(0.1, 1, (nsys, n))
    d = rng.uniform(-1, 1, (nsys, n))
    return a, b, c, d


def _solve(fn, arrs, n, nsys, layout, solver):
    import torch
    dev = [torch.tensor(np.ascontiguousarray(x if layout == 0 else x.T), dtype=torch.float64, device="cuda")
           for x in arrs]
    out = torch.full_like(dev[3], float("nan"))
    st = fn(*(t.data_ptr() for t in dev), out.data_ptr(), n, nsys, layout, solver,
            torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    res = out.cpu().numpy()
    return st, (res if layout == 0 else res.T)


@pytest.mark.parametrize("layout", [1, 0])
@pytest.mark.parametrize("solver", [F.SOLVER_EXACT, F.SOLVER_HYBRID])
def test_noalloc_matches_allocating_entry_point_twice(layout, solver):
    for call, (n, nsys) in enumerate([(702, 300), (302, 700)]):
        arrs = _systems(n, nsys, seed=10 * call + layout)
        st_ref, ref = _solve(F.lib.ixb_tridiag_f64, arrs, n, nsys, layout, solver)
        st, got = _solve(F.lib.ixb_tridiag_f64_noalloc, arrs, n, nsys, layout, solver)
        assert st_ref == F.OK and st == F.OK
        assert np.all(np.isfinite(got))
        if solver == F.SOLVER_EXACT:
            assert np.array_equal(got, ref), call
        else:
            err = np.max(np.abs(got - ref)) / np.max(np.abs(ref))
            assert err < TOL, (call, err)


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch
    n, nsys = 1025, 1024  # n*nsys > IXB_NOALLOC_MAX_ELEMS
    assert n * nsys > F.NOALLOC_MAX_ELEMS
    t = torch.zeros(n * nsys, dtype=torch.float64, device="cuda")
    p = t.data_ptr()
    st = F.lib.ixb_tridiag_f64_noalloc(p, p, p, p, p, n, nsys, 1, F.SOLVER_HYBRID,
                                       torch.cuda.current_stream().cuda_stream)
    assert st == F.EINVAL


def test_noalloc_calls_leave_device_memory_unchanged():
    # the property the entry point exists for: after a first call on the
    # device, further calls (both layouts, both solvers) take no device
    # memory.  torch's cache is emptied and the device's free memory compared
    # around 20 calls; the comparison is retried so that a change made by
    # another process on the same GPU cannot fail it.
    import torch
    n, nsys = 702, 300
    arrs = _systems(n, nsys, seed=7)
    dev = {lay: [torch.tensor(np.ascontiguousarray(x if lay == 0 else x.T), dtype=torch.float64, device="cuda")
                 for x in arrs] for lay in (0, 1)}
    out = {lay: torch.empty_like(dev[lay][3]) for lay in (0, 1)}
    stream = torch.cuda.current_stream().cuda_stream

    def calls(k):
        for _ in range(k):
            for lay in (0, 1):
                for solver in (F.SOLVER_EXACT, F.SOLVER_HYBRID):
                    st = F.lib.ixb_tridiag_f64_noalloc(*(t.data_ptr() for t in dev[lay]), out[lay].data_ptr(), n,
                                                       nsys, lay, solver, stream)
                    assert st == F.OK
        torch.cuda.synchronize()

    calls(1)  # first calls: module loading and the scratch address lookup
    torch.cuda.empty_cache()
    same = []
    for _ in range(3):
        free0, _ = torch.cuda.mem_get_info()
        calls(5)
        free1, _ = torch.cuda.mem_get_info()
        same.append(free1 == free0)
        if same[-1]:
            break
    assert any(same), "device memory changed across ixb_tridiag_f64_noalloc calls"
