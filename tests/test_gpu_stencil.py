"""Stencil parity on the GPU: the drop-in steps against the reference."""
import numpy as np
import pytest

from tests.conftest import golden, rel_l2
from tests.golden.make_golden import pthread_inputs, sha, wrap_inputs

pytestmark = pytest.mark.gpu


def _t(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def test_wrap_case_bit_exact(cuda):
    import swfwi_b200 as S
    torch = cuda
    g = golden("wrap_533x193")
    prev, curr, vel, nb = wrap_inputs()
    p = _t(torch, prev)
    S.fd4t10s_damp_zjh_2d_vtrans(p, _t(torch, curr), _t(torch, vel), nb)
    out = p.cpu().numpy()
    np.testing.assert_array_equal(out.ravel()[::101], g["sub"])
    assert sha(out) == str(g["sha256"])


def test_pthread_case_bit_exact(cuda):
    import swfwi_b200 as S
    torch = cuda
    g = golden("pthread_20x20")
    p0, p1, vel = pthread_inputs()
    a, b, v = _t(torch, p0), _t(torch, p1), _t(torch, vel)
    for k in range(2):
        S.fd4t10s_zjh_2d_vtrans(a, b, v)
        np.testing.assert_array_equal(a.cpu().numpy(), g["p0_steps"][k])
        a, b = b, a


SIZES = [(20, 20, 1), (40, 30, 12), (97, 61, 20), (533, 193, 36), (993, 337, 36), (45, 1042, 36)]


@pytest.mark.parametrize("nx,nz,nb", SIZES)
@pytest.mark.parametrize("damped", [True, False])
def test_step_bit_exact_vs_reference(cuda, ref, nx, nz, nb, damped):
    import swfwi_b200 as S
    torch = cuda
    rng = np.random.default_rng(nx + 7 * nz)
    curr = rng.standard_normal((nx, nz)).astype(np.float32)
    prev = rng.standard_normal((nx, nz)).astype(np.float32)
    vt = rng.uniform(3.0, 80.0, (nx, nz)).astype(np.float32)
    want = prev.copy()
    ref.step(want, curr, vt, nb if damped else None)
    p = _t(torch, prev)
    if damped:
        S.fd4t10s_damp_zjh_2d_vtrans(p, _t(torch, curr), _t(torch, vt), nb)
    else:
        S.fd4t10s_zjh_2d_vtrans(p, _t(torch, curr), _t(torch, vt))
    got = p.cpu().numpy()
    np.testing.assert_array_equal(got.view(np.int32), want.view(np.int32))
    # the 6-cell frame keeps its old values
    np.testing.assert_array_equal(got[:6], prev[:6])
    np.testing.assert_array_equal(got[:, -6:], prev[:, -6:])


@pytest.mark.parametrize("damped", [True, False])
def test_fast_step_within_tolerance(cuda, ref, damped):
    import swfwi_b200 as S
    torch = cuda
    nx, nz, nb = 533, 193, 36
    rng = np.random.default_rng(5)
    curr = rng.standard_normal((3, nx, nz)).astype(np.float32)
    prev = rng.standard_normal((3, nx, nz)).astype(np.float32)
    vt = rng.uniform(3.0, 80.0, (nx, nz)).astype(np.float32)
    p = _t(torch, prev)
    S.fd4t10s_step_batch(p, _t(torch, curr), _t(torch, vt), nb, damped, S.ARITH_FAST)
    got = p.cpu().numpy()
    for s in range(3):
        want = prev[s].copy()
        ref.step(want, curr[s], vt, nb if damped else None)
        assert rel_l2(got[s], want) < 1e-6


def test_batched_ref_step_equals_single(cuda):
    import swfwi_b200 as S
    torch = cuda
    nx, nz, nb = 97, 61, 20
    rng = np.random.default_rng(9)
    curr = rng.standard_normal((4, nx, nz)).astype(np.float32)
    prev = rng.standard_normal((4, nx, nz)).astype(np.float32)
    vt = _t(torch, rng.uniform(3.0, 80.0, (nx, nz)).astype(np.float32))
    pb = _t(torch, prev)
    S.fd4t10s_step_batch(pb, _t(torch, curr), vt, nb, True, S.ARITH_REF)
    for s in range(4):
        p = _t(torch, prev[s])
        S.fd4t10s_damp_zjh_2d_vtrans(p, _t(torch, curr[s]), vt, nb)
        assert torch.equal(p, pb[s])


def test_f64_step_matches_f64_oracle(cuda, fdo):
    import swfwi_b200 as S
    torch = cuda
    nx, nz, nb = 97, 61, 20
    rng = np.random.default_rng(11)
    curr = rng.standard_normal((nx, nz))
    prev = rng.standard_normal((nx, nz))
    vt = rng.uniform(3.0, 80.0, (nx, nz))
    want = prev.copy()
    fdo.step_f64(want, curr, vt, nb, True)
    p = torch.from_numpy(prev.copy()).cuda()
    S.fd4t10s_step_f64(p, torch.from_numpy(curr).cuda(), torch.from_numpy(vt).cuda(), nb, True)
    # the GPU contracts double multiply-adds into FMAs: agreement to ~1e-10
    assert rel_l2(p.cpu().numpy(), want) < 1e-9


def test_step_rejects_bad_arguments(cuda):
    import swfwi_b200 as S
    torch = cuda
    p = torch.zeros((10, 10), device="cuda")
    with pytest.raises(S.SwfwiError):
        S.fd4t10s_damp_zjh_2d_vtrans(p, p, p, 3)   # grid smaller than the stencil frame
