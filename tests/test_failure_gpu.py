"""Failure detection without a GPU fault: a bounded copy wait that expires.

The streamed contiguous line solve (hybrid solver, layout 0) waits on the
bulk-copy engine with a bounded wait.  ixb_tridiag_set_first_wait_limit(0)
makes the first wait of every CTA expire at once although its copies are
on their way: each CTA then records the timeout, drains its copies at the
default bound, and returns without writing.  The host sees IXB_ETIMEOUT from
ixb_tridiag_status, the outputs are untouched, and the next call, with the
default limit restored, is clean and correct.  Nothing here faults, traps or
hangs the GPU: every wait ends, and every copy lands before its CTA exits."""
import numpy as np
import pytest

from ixchel2d_b200 import _ffi as F

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _need_gpu(has_gpu):
    if not has_gpu:
        pytest.skip("no CUDA device")


def _systems(n, nsys, seed, dtype):
    rng = np.random.default_rng(seed)
    a = rng.uniform(-1, 0, (nsys, n))
    c = rng.uniform(-1, 0, (nsys, n))
    b = np.abs(a) + np.abs(c) + rng.uniform(0.1, 1, (nsys, n))
    d = rng.uniform(-1, 1, (nsys, n))
    return [x.astype(dtype) for x in (a, b, c, d)]


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_expired_copy_wait_is_reported_and_the_next_call_is_clean(dtype):
    import torch
    n, nsys = 4096, 400  # contiguous systems in the streamed kernel's range; more systems than CTAs
    fn = F.lib.ixb_tridiag_f64 if dtype == np.float64 else F.lib.ixb_tridiag_f32
    tdt = torch.float64 if dtype == np.float64 else torch.float32
    arrs = [torch.tensor(x, dtype=tdt, device="cuda") for x in _systems(n, nsys, 3, dtype)]
    out = torch.full((nsys, n), float("nan"), dtype=tdt, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream

    def solve():
        return fn(*(t.data_ptr() for t in arrs), out.data_ptr(), n, nsys, 0, F.SOLVER_HYBRID, stream)

    assert F.lib.ixb_tridiag_status() in (F.OK, F.ETIMEOUT)  # start from a clear record
    try:
        assert F.lib.ixb_tridiag_set_first_wait_limit(0) == F.OK
        assert solve() == F.OK
        torch.cuda.synchronize()
        assert F.lib.ixb_tridiag_status() == F.ETIMEOUT
        assert torch.isnan(out).all().item()  # no CTA wrote anything
    finally:
        assert F.lib.ixb_tridiag_set_first_wait_limit(-1) == F.OK
    assert F.lib.ixb_tridiag_status() == F.OK  # the record was cleared by the read above
    assert solve() == F.OK
    torch.cuda.synchronize()
    assert F.lib.ixb_tridiag_status() == F.OK
    ref = torch.empty_like(out)
    assert fn(*(t.data_ptr() for t in arrs), ref.data_ptr(), n, nsys, 0, F.SOLVER_EXACT, stream) == F.OK
    torch.cuda.synchronize()
    tol = 1e-12 if dtype == np.float64 else 1e-4
    err = (out - ref).abs().max().item() / ref.abs().max().item()
    assert err < tol, err
