"""Gradients and per-iteration arithmetic on the GPU against the reference."""
import numpy as np
import pytest

from tests.conftest import golden, rel_l2
from tests.gpu_helpers import small_method, t

pytestmark = pytest.mark.gpu


def test_calgradient_fwi_bit_exact(cuda):
    torch = cuda
    s, m, g, _ = small_method(torch)
    gr = torch.zeros(g["grad_shot1"].shape, device="cuda")
    m.calgradient_fwi(t(torch, g["wlt"]), t(torch, g["vsrc"]), gr, 1)
    np.testing.assert_array_equal(gr.cpu().numpy(), g["grad_shot1"])
    m.scaleGradient(gr)
    m.maskGradient(gr)
    np.testing.assert_array_equal(gr.cpu().numpy(), g["grad_shot1_scaled"])


def test_calgradient_ess_bit_exact(cuda):
    torch = cuda
    s, m, g, _ = small_method(torch)
    enc = (g["wlt"][:, None] * g["ess_codes"][None, :].astype(np.float32)).astype(np.float32)
    gr = torch.zeros(g["grad_ess"].shape, device="cuda")
    m.calgradient_ess(t(torch, enc), t(torch, g["vsrc"]), gr)
    np.testing.assert_array_equal(gr.cpu().numpy(), g["grad_ess"])


@pytest.mark.parametrize("tuning", [None, (1, 248, 7, 3, 1), (1, 376, 64, 7, 0), (1, 120, 9, 3, 0),
                                    (5, 120, 64, 3, 0), (5, 120, 7, 7, 0), (5, 120, 1, 3, 0)])
def test_gradient_batch_matches_reference_loop(cuda, tuning):
    # the per-shot loop of FwiFramework::epoch: gradient bit-exact, the
    # objective summed in FP64 (the reference sums in float); with the
    # default and other stencil launch shapes
    torch = cuda
    s, m, g, _ = small_method(torch)
    if tuning is not None:
        m.set_tuning(*tuning)
    gr = torch.zeros(g["grad_sum"].shape, device="cuda")
    obj = m.gradient_batch(t(torch, g["wlt"]), t(torch, g["dobs"]), [0, 1, 2], gr)
    np.testing.assert_array_equal(gr.cpu().numpy(), g["grad_sum"])
    assert abs(obj.sum() - float(g["obj"])) / float(g["obj"]) < 1e-5


def test_gradient_host_entry_matches_device(cuda):
    torch = cuda
    s, m, g, _ = small_method(torch)
    gh, obj = m.gradient_host(g["exvel_init"], g["wlt"], g["dobs"][[2, 0]], [2, 0])
    gd = torch.zeros(g["grad_sum"].shape, device="cuda")
    obj2 = m.gradient_batch(t(torch, g["wlt"]), t(torch, g["dobs"]), [2, 0], gd)
    np.testing.assert_array_equal(gh, gd.cpu().numpy())
    np.testing.assert_array_equal(obj, obj2)


def test_fast_gradient_within_tolerance_and_f64(cuda, fdo):
    import swfwi_b200 as S
    torch = cuda
    s, m, g, vel = small_method(torch, arith=S.ARITH_FAST)
    gr = torch.zeros(g["grad_shot1"].shape, device="cuda")
    m.calgradient_fwi(t(torch, g["wlt"]), t(torch, g["vsrc"]), gr, 1)
    fast = gr.cpu().numpy()
    assert rel_l2(fast, g["grad_shot1"]) < 1e-4
    g64 = torch.zeros(g["grad_shot1"].shape, dtype=torch.float64, device="cuda")
    m.calgradient_fwi_f64(vel, t(torch, g["wlt"], torch.float64), t(torch, g["vsrc"], torch.float64), g64, 1)
    g64 = g64.cpu().numpy()
    bx0 = s.nb + 6
    nzpad = s.nz + s.nb + 12
    src = (s.sxbeg + 1 * s.jsx + bx0) * nzpad + s.szbeg + 6
    rec = (np.arange(s.ng) + bx0) * nzpad + s.gzbeg + 6
    cpu64 = fdo.gradient_f64(g["exvel_init"].astype(np.float64), bx0, s.nt, s.dt, g["wlt"].astype(np.float64),
                             src, rec, g["vsrc"].astype(np.float64))
    assert rel_l2(g64, cpu64) < 1e-9
    print(f"gradient rel-L2 vs FP64: REF {rel_l2(g['grad_shot1'], g64):.2e}  FAST {rel_l2(fast, g64):.2e}")


@pytest.mark.parametrize("fmt,bound", [(1, 1e-4), (2, 1e-4)])
def test_16bit_strips_gradient_error_vs_f64(cuda, fmt, bound):
    # scaled FP16 / BF16 boundary strips: the gradient's error against the
    # FP64 run of the same scheme, beside the FP32-strip gradient's
    import swfwi_b200 as S
    torch = cuda
    s, m, g, vel = small_method(torch)
    g64 = torch.zeros(g["grad_shot1"].shape, dtype=torch.float64, device="cuda")
    m.calgradient_fwi_f64(vel, t(torch, g["wlt"], torch.float64), t(torch, g["vsrc"], torch.float64), g64, 1)
    g64 = g64.cpu().numpy()
    m.set_strip_format(fmt)
    gr = torch.zeros(g["grad_shot1"].shape, device="cuda")
    m.calgradient_fwi(t(torch, g["wlt"]), t(torch, g["vsrc"]), gr, 1)
    q = gr.cpu().numpy()
    e32, eq = rel_l2(g["grad_shot1"], g64), rel_l2(q, g64)
    print(f"gradient rel-L2 vs FP64: F32 strips {e32:.2e}  {('F16', 'BF16')[fmt - 1]} strips {eq:.2e}")
    assert np.isfinite(q).all() and eq < bound, eq
    # back to FP32 strips: bit-exact again
    m.set_strip_format(S.STRIP_F32)
    gr.zero_()
    m.calgradient_fwi(t(torch, g["wlt"]), t(torch, g["vsrc"]), gr, 1)
    np.testing.assert_array_equal(gr.cpu().numpy(), g["grad_shot1"])


def test_16bit_strips_batched_gradient(cuda):
    # the batched gradient loop with FP16 strips stays within the FP16
    # bound of the exact (FP32-strip) result
    import swfwi_b200 as S
    torch = cuda
    s, m, g, _ = small_method(torch)
    m.set_strip_format(S.STRIP_F16)
    gr = torch.zeros(g["grad_sum"].shape, device="cuda")
    obj = m.gradient_batch(t(torch, g["wlt"]), t(torch, g["dobs"]), [0, 1, 2], gr)
    assert rel_l2(gr.cpu().numpy(), g["grad_sum"]) < 1e-4
    assert abs(obj.sum() - float(g["obj"])) / float(g["obj"]) < 1e-5


def test_uneven_spreads_match_per_shot_reference(cuda, ref):
    # per-shot receiver spreads (not expressible in the reference's one
    # common line): each shot checked against a reference model built with
    # that shot's own receiver line
    import swfwi_b200 as S
    from swfwi_b200 import survey as sv
    torch = cuda
    s = sv.small(nx=60, nz=40, nt=160, ns=3)
    s.spreads = sv.uneven_spreads(s, seed=4, lo=20, hi=50)
    v = sv.layered_model(s.nx, s.nz, seed=5)
    vi = sv.smooth(v, 3).astype(np.float32)
    off, gx, gz = s.spreads
    ngmax = int(np.max(np.diff(off)))
    wlt = ref.ricker(s.nt, s.fm, s.dt)
    m = S.Damp4t10d.from_survey(s)
    ext = m.expandDomain(v)
    exi = m.expandDomain(vi)
    dobs = np.zeros((s.ns, s.nt, ngmax), np.float32)
    want_g = np.zeros_like(ext)
    want_obj = 0.0
    for shot in range(s.ns):
        n = int(off[shot + 1] - off[shot])
        ss = s.scaled(ng=n, gxbeg=int(gx[off[shot]]), sxbeg=s.sxbeg + shot * s.jsx, ns=1, spreads=None)
        M = ref.model(ss)
        M.bind_velocity(ext)
        dobs[shot, :, :n] = M.fwi_forward(wlt, 0)
        M.bind_velocity(exi)
        gs, o = M.fwi_gradient(wlt, dobs[shot:shot + 1, :, :n])
        want_g = (want_g + gs).astype(np.float32)
        want_obj += o
    vel = t(torch, exi)
    m.bindVelocity(vel)
    gr = torch.zeros(ext.shape, device="cuda")
    obj = m.gradient_batch(t(torch, wlt), t(torch, dobs), [0, 1, 2], gr)
    np.testing.assert_array_equal(gr.cpu().numpy(), want_g)
    assert abs(obj.sum() - want_obj) / want_obj < 1e-5


def test_cg_and_velocity_update_match_reference(cuda, ref):
    import swfwi_b200 as S
    torch = cuda
    s, m, g, vel = small_method(torch)
    M = ref.model(s)
    M.bind_velocity(g["exvel_init"])
    rng = np.random.default_rng(2)
    g0 = rng.standard_normal(g["grad_sum"].shape).astype(np.float32)
    g1 = g["grad_sum"]
    d = rng.standard_normal(g1.shape).astype(np.float32)
    pre_r, dir_r = ref.update_grad(g0, g1, d, 1)
    pre, dd = t(torch, g0).clone(), t(torch, d).clone()
    S.update_grad(pre, t(torch, g1), dd, 1)
    np.testing.assert_array_equal(pre.cpu().numpy(), pre_r)
    assert rel_l2(dd.cpu().numpy(), dir_r) < 1e-6
    a2, a3 = S.cal_max_alpha(vel, t(torch, g1), s.dt, s.dx, s.maxdv)
    ra2, ra3 = M.cal_max_alpha(g1, s.maxdv)
    assert (a2, a3) == (ra2, ra3)
    nv = torch.zeros_like(vel)
    S.update_vel(nv, vel, t(torch, g1), a2, 1500.0, 4700.0, s.dx, s.dt)
    np.testing.assert_array_equal(nv.cpu().numpy(), M.update_vel(g["exvel_init"], g1, a2, 1500.0, 4700.0))
    m.refillBoundary(nv)
    np.testing.assert_array_equal(nv.cpu().numpy(),
                                  M.refill_boundary(M.update_vel(g["exvel_init"], g1, a2, 1500.0, 4700.0)))
