"""The EnKF analysis on the GPU (src/enfwi/enkfanalyze.cpp) against the
oracle's restatement: HA by batched member modelling (bit-exact against the
compiled reference), the FP64 gain, and the member update."""
import numpy as np
import pytest

from oracle import enkf_oracle as E
from tests.gpu_helpers import small_method, t

pytestmark = pytest.mark.gpu


def _case(n, rows, seed):
    rng = np.random.default_rng(seed)
    base = rng.standard_normal(rows).astype(np.float32)
    hona = (base[None, :] + 0.3 * rng.standard_normal((n, rows))).astype(np.float32)
    dobs = (base + 0.1 * rng.standard_normal(rows)).astype(np.float32)
    z = rng.standard_normal((n, rows))
    return hona, dobs, z


@pytest.mark.parametrize("n,rows", [(64, 40000), (16, 5003), (2, 999)])
def test_gain_matrix_matches_oracle(cuda, n, rows):
    import swfwi_b200 as S
    torch = cuda
    hona, dobs, z = _case(n, rows, seed=n)
    want, sigma, clip = E.gain_matrix(hona, dobs, z, 0.05)
    got, gs, gclip = S.enkf_gain_matrix(t(torch, hona), t(torch, dobs), t(torch, z), sigfac=0.05)
    assert gs == sigma                      # same element, same double
    assert gclip == clip
    err = np.linalg.norm(got - want) / np.linalg.norm(want)
    assert err < 1e-8, err
    # a second call with sigma kept (as the reference keeps sigmaIter0)
    got2, gs2, _ = S.enkf_gain_matrix(t(torch, hona), t(torch, dobs), t(torch, z), sigfac=0.05, sigma=gs)
    assert gs2 == gs and np.array_equal(got2, got)


def test_gain_matrix_device_draws_deterministic(cuda):
    import swfwi_b200 as S
    torch = cuda
    hona, dobs, _ = _case(32, 20000, seed=5)
    h, d = t(torch, hona), t(torch, dobs)
    a, s1, _ = S.enkf_gain_matrix(h, d, None, sigfac=0.05, seed=7)
    b, s2, _ = S.enkf_gain_matrix(h, d, None, sigfac=0.05, seed=7)
    c, _, _ = S.enkf_gain_matrix(h, d, None, sigfac=0.05, seed=8)
    assert s1 == s2 and np.array_equal(a, b) and np.isfinite(a).all()
    assert not np.array_equal(a, c)


def test_update_matches_oracle(cuda):
    import swfwi_b200 as S
    torch = cuda
    rng = np.random.default_rng(3)
    n, model = 24, 50000
    dx, dt = 20.0, 0.002
    vphys = (2500 + 300 * rng.standard_normal((n, model))).astype(np.float32)
    vels = E.vel_trans(vphys, dx, dt)
    t4 = 0.02 * rng.standard_normal((n, n))
    want = E.analyze_update(vels, t4, dx, dt)
    g = t(torch, vels)
    S.enkf_update(g, t4, dx, dt)
    got = g.cpu().numpy()
    rel = np.abs(got - want) / np.abs(want)
    assert rel.max() < 1e-6, rel.max()
    mean = torch.empty(model, device="cuda")
    S.enkf_mean(mean, t(torch, vels))
    np.testing.assert_array_equal(mean.cpu().numpy(), E.create_a_mean(vels))


def test_members_forward_matches_reference(cuda, ref):
    # HA: the encoded supershot modelled with each member's velocity in one
    # batch, against the compiled reference's EssForwardModeling per member
    import swfwi_b200 as S
    from tests.golden.make_golden import small_survey
    torch = cuda
    s, m, g, _ = small_method(torch)
    rng = np.random.default_rng(4)
    base = g["exvel_init"]
    n = 5
    vels = np.stack([(base * (1 + 0.02 * rng.standard_normal(base.shape))).astype(np.float32)
                     for _ in range(n)])
    codes = np.array([1, -1, 1][: s.ns] + [1] * max(0, s.ns - 3), np.int32)
    enc = (g["wlt"][:, None] * codes[None, :].astype(np.float32)).astype(np.float32)
    nxpad, nzpad, ns, ng, nt = m.dims()
    hona = torch.zeros((n, ng * nt), device="cuda")
    m.ess_forward_members(t(torch, enc), t(torch, vels), hona)
    got = hona.cpu().numpy()
    M = ref.model(small_survey()[0])
    for i in range(n):
        M.bind_velocity(vels[i])
        want = M.ess_forward(enc)                       # [nt][ng]
        np.testing.assert_array_equal(got[i], want.T.reshape(-1))


def test_enkf_analyze_pipeline_matches_oracle(cuda):
    # the whole analysis through the Python mirror of EnkfAnalyze: encoded
    # data, HA, gain and update, against the oracle fed the same HA and draws
    import swfwi_b200 as S
    torch = cuda
    s, m, g, _ = small_method(torch)
    rng = np.random.default_rng(6)
    base = g["exvel_init"]
    n = 8
    vels = np.stack([(base * (1 + 0.03 * rng.standard_normal(base.shape))).astype(np.float32)
                     for _ in range(n)])
    codes = np.where(rng.random(s.ns) < 0.5, -1, 1).astype(np.int32)
    nxpad, nzpad, ns, ng, nt = m.dims()
    z = rng.standard_normal((n, ng * nt))
    an = S.EnkfAnalyze(m, t(torch, g["wlt"]), t(torch, g["dobs"]), 0.05)
    vg = t(torch, vels)
    hona = torch.zeros((n, ng * nt), device="cuda")
    enc = (g["wlt"][:, None] * codes[None, :].astype(np.float32)).astype(np.float32)
    m.ess_forward_members(t(torch, enc), vg, hona)
    t4, clip = an.analyze(vg, codes, t(torch, z))
    encobs = np.zeros((nt, ng), np.float32)
    for i in range(ns):
        encobs = (encobs + g["dobs"][i] * np.float32(codes[i])).astype(np.float32)
    want_t4, sigma, wclip = E.gain_matrix(hona.cpu().numpy(), encobs.T.reshape(-1), z, 0.05)
    assert an.sigma == sigma and clip == wclip
    assert np.linalg.norm(t4 - want_t4) / np.linalg.norm(want_t4) < 1e-8
    want = E.analyze_update(vels.reshape(n, -1), want_t4, s.dx, s.dt).reshape(vels.shape)
    got = vg.cpu().numpy()
    assert (np.abs(got - want) / np.abs(want)).max() < 1e-5


def test_analysis_in_one_call_matches_gain_then_update(cuda):
    # the gain kept in device memory and applied at once gives the bits of
    # the two-call form; a non-finite gain leaves the members unchanged
    import swfwi_b200 as S
    torch = cuda
    n, rows, model = 40, 30000, 20000
    dx, dt = 20.0, 0.002
    hona, dobs, z = _case(n, rows, seed=11)
    rng = np.random.default_rng(12)
    vels = E.vel_trans((2500 + 200 * rng.standard_normal((n, model))).astype(np.float32), dx, dt)
    h, d, zz = t(torch, hona), t(torch, dobs), t(torch, z)
    t4a, sa, ca = S.enkf_gain_matrix(h, d, zz, sigfac=0.05)
    va = t(torch, vels).clone()
    S.enkf_update(va, t4a, dx, dt)
    vb = t(torch, vels).clone()
    t4b, sb, cb = S.enkf_analyze(h, d, vb, dx, dt, z=zz, sigfac=0.05)
    assert sa == sb and ca == cb
    np.testing.assert_array_equal(t4a, t4b)
    np.testing.assert_array_equal(va.cpu().numpy(), vb.cpu().numpy())
    bad = hona.copy()
    bad[3, 17] = np.nan
    vc = t(torch, vels).clone()
    with pytest.raises(S.SwfwiError) as e:
        S.enkf_analyze(t(torch, bad), d, vc, dx, dt, z=zz, sigfac=0.05, sigma=sa)
    assert e.value.status == 4              # SWFWI_ERR_NONFINITE
    np.testing.assert_array_equal(vc.cpu().numpy(), vels)
