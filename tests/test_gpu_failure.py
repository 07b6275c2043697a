"""Failure detection without a GPU fault: the stencil kernels' bounded
mbarrier wait gives up by itself when nothing arrives, the host reads the
error flag as SWFWI_ERR_TIMEOUT, and the context stays usable."""
import numpy as np
import pytest

from tests.gpu_helpers import small_method, t

pytestmark = pytest.mark.gpu

SWFWI_ERR_TIMEOUT = 3   # include/swfwi_gpu.h


def test_bounded_wait_times_out_and_context_survives(cuda):
    import time
    import swfwi_b200 as S
    torch = cuda
    t0 = time.perf_counter()
    status = S.lib().swfwi_selftest_bounded_wait(S._stream())
    waited = time.perf_counter() - t0
    assert status == SWFWI_ERR_TIMEOUT, (status, S.lib().swfwi_last_error())
    assert waited < 30.0
    # the same context still computes the reference's seismogram bit for bit
    s, m, g, _ = small_method(torch)
    d = torch.zeros((s.nt, s.ng), device="cuda")
    m.FwiForwardModeling(t(torch, g["wlt"]), d, 1)
    np.testing.assert_array_equal(d.cpu().numpy(), g["dcal"][1])
