"""Asynchronous state downloads (ixb_download_state_async / ixb_download_wait),
which let the case driver write its restart and output files while the next
package of time steps runs: the snapshot is the state at the call, even when
iterations run before the copies have been waited for."""
import ctypes as C

import numpy as np
import pytest

from ixchel2d_b200 import Simple2D, cases
from ixchel2d_b200 import _ffi as F

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _need_gpu(has_gpu):
    if not has_gpu:
        pytest.skip("no CUDA device")


def _pinned(shape):
    p = C.c_void_p()
    n = int(np.prod(shape))
    F.check(F.lib.ixb_host_alloc(n * 8, C.byref(p)), "ixb_host_alloc")
    arr = np.ctypeslib.as_array((C.c_double * n).from_address(p.value)).reshape(shape[::-1]).T
    return p, arr


def test_async_download_is_the_state_at_the_call():
    case = cases.lid_driven_mixed(45, 29)
    g = Simple2D.from_case(case)
    g.iterations(20)
    ref = g.download()
    keys = ("u", "v", "p", "T")
    bufs = {k: _pinned(ref[k].shape) for k in keys}
    try:
        for rnd in range(2):  # the second call reuses the snapshot after the first one's copies
            for k in keys:
                bufs[k][1][...] = np.nan
            F.check(F.lib.ixb_download_state_async(g.h, *(F.dptr(bufs[k][1]) for k in keys), None, None, None),
                    "ixb_download_state_async")
            g.iterations(7)  # the state moves on before the copies are waited for
            F.check(F.lib.ixb_download_wait(g.h), "ixb_download_wait")
            for k in keys:
                assert np.array_equal(bufs[k][1], ref[k]), (rnd, k)
            ref = g.download()
        assert not np.array_equal(ref["u"], bufs["u"][1])
    finally:
        for p, _ in bufs.values():
            F.lib.ixb_host_free(p)
    assert F.lib.ixb_download_wait(None) == F.EINVAL
