"""The EnFWI driver (main-enfwi-damp.cpp:406-631) on the GPU: a small
ensemble run end to end, and its first analysis against the EnKF oracle
fed the same modelled data, codes and draws."""
import numpy as np
import pytest

from oracle import enkf_oracle as E

pytestmark = pytest.mark.gpu


def _setup(n=4):
    import swfwi_b200 as S
    from swfwi_b200 import survey as sv
    s = sv.small(nx=50, nz=40, nt=200, ns=3)
    vt = sv.layered_model(s.nx, s.nz, seed=7)
    vi = sv.smooth(vt, 3.0).astype(np.float32)
    m = S.Damp4t10d.from_survey(s)
    ext, exi = m.expandDomain(vt), m.expandDomain(vi)
    nxpad, nzpad = ext.shape
    pert = np.stack([sv.gaussian_random_field(nxpad, nzpad, s.dx, 200.0, 60.0, seed=100 + i) for i in range(n)])
    wlt = S.ricker_wavelet(s.nt, s.fm, s.dt)
    import torch
    dobs = torch.zeros((s.ns, s.nt, s.ng), device="cuda")
    vel = torch.from_numpy(ext).cuda()
    m.bindVelocity(vel)
    m.forward_batch(torch.from_numpy(wlt).cuda(), dobs, list(range(s.ns)))
    return s, m, ext, exi, pert, wlt, dobs.cpu().numpy()


def test_enfwi_runs_and_logs(cuda):
    from swfwi_b200.enfwi import EnFwi
    s, m, ext, exi, pert, wlt, dobs = _setup()
    en = EnFwi(s, exi, pert, wlt, dobs, vmin=1400.0, vmax=5000.0, nita=2, maxdv=200.0, sigfac=0.05,
               niterenkf=1, exvel_true=ext)
    rng = np.random.default_rng(3)
    rows = s.nt * s.ng
    absobj, norobj = en.run(2, z_draws=lambda i: cuda.from_numpy(rng.standard_normal((4, rows))).cuda())
    assert len(absobj) == 3 and norobj[0] == 1.0 and np.all(np.isfinite(absobj))
    assert len(en.logs) == 2 * 4
    for row in en.logs:
        assert np.isfinite(row["data_rss"]) and 0 < row["slowness_l2"] < 1 and 0 < row["slowness_l1"] < 1


def test_enfwi_first_analysis_matches_oracle(cuda):
    import swfwi_b200 as S
    from swfwi_b200.enfwi import EnFwi, ENKF_SEED
    torch = cuda
    s, m, ext, exi, pert, wlt, dobs = _setup()
    en = EnFwi(s, exi, pert, wlt, dobs, vmin=1400.0, vmax=5000.0, nita=2, maxdv=200.0, sigfac=0.05,
               niterenkf=1)
    before = en.velocities().cpu().numpy()
    codes = S.random_codes(ENKF_SEED, s.ns, skip=0)
    enc = (wlt[:, None] * codes[None, :].astype(np.float32)).astype(np.float32)
    hona = torch.zeros((4, s.ng * s.nt), device="cuda")
    en.fm.ess_forward_members(torch.from_numpy(enc).cuda(), torch.from_numpy(before).cuda(), hona)
    encobs = np.zeros((s.nt, s.ng), np.float32)
    for i in range(s.ns):
        encobs = (encobs + dobs[i] * np.float32(codes[i])).astype(np.float32)
    z = np.random.default_rng(5).standard_normal((4, s.nt * s.ng))
    t4, sigma, _ = E.gain_matrix(hona.cpu().numpy(), encobs.T.reshape(-1), z, 0.05)
    want = E.analyze_update(before.reshape(4, -1), t4, s.dx, s.dt).reshape(before.shape)
    en.analyze(torch.from_numpy(z).cuda())
    got = en.velocities().cpu().numpy()
    assert en.enkf.sigma == sigma
    assert (np.abs(got - want) / np.abs(want)).max() < 1e-5
