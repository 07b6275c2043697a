"""The allocation-free objective entry point (for callers that cannot call
cudaMalloc): same sums as swfwi_cal_objective, its scratch in a static
device array.  Collected last so a stop-at-first-failure run has already run
everything else."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_static_objective_matches_allocating_entry_point(cuda):
    import swfwi_b200 as S
    torch = cuda
    rng = np.random.default_rng(17)
    for call in range(2):           # two calls in a row share the static scratch
        nslots = 7 + call * 20
        n = 3001 + 977 * call
        r = torch.from_numpy(rng.standard_normal((nslots, n)).astype(np.float32)).cuda()
        out = torch.zeros(nslots, dtype=torch.float64, device="cuda")
        S.cal_objective_static(r, out)
        got = out.cpu().numpy()
        for s in range(nslots):
            # the same kernels, grid and partial count: the same bits
            want = S.cal_objective(r[s].contiguous())
            assert got[s] == want, (call, s, got[s], want)
        # and against an FP64 sum on the host
        ref = (r.double() ** 2).sum(dim=1).cpu().numpy()
        np.testing.assert_allclose(got, ref, rtol=1e-10)


def test_static_objective_rejects_too_many_slots(cuda):
    import swfwi_b200 as S
    torch = cuda
    r = torch.zeros((33, 10), device="cuda")
    out = torch.zeros(33, dtype=torch.float64, device="cuda")
    with pytest.raises(S.SwfwiError) as e:
        S.cal_objective_static(r, out)
    assert e.value.status == 1
    assert b"32" in S.lib().swfwi_last_error()
