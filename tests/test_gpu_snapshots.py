"""Checkpoint-snapshot reconstruction of the source field in the gradients'
backward sweep (FP32 / FP16 / BF16 snapshots with per-field scaling): the
gradient against the FP64 run of the same scheme and against the strips'
back-propagation, and its independence of the snapshot interval."""
import numpy as np
import pytest

from tests.conftest import rel_l2
from tests.gpu_helpers import small_method, t

pytestmark = pytest.mark.gpu


def _interior(a, s):
    # the gradient's unmasked region (maskGradient): outside it the strips'
    # back-propagation is not the forward field (undamped steps over the
    # sponge), so the two reconstructions are compared inside it
    b = s.nb + 6
    return a[b:a.shape[0] - b, 6:a.shape[1] - b]


def _grad(torch, m, g, shot=1):
    gr = torch.zeros(g["grad_shot1"].shape, device="cuda")
    m.calgradient_fwi(t(torch, g["wlt"]), t(torch, g["vsrc"]), gr, shot)
    return gr.cpu().numpy()


def _grad64(torch, m, g, vel, shot=1):
    g64 = torch.zeros(g["grad_shot1"].shape, dtype=torch.float64, device="cuda")
    m.calgradient_fwi_f64(vel, t(torch, g["wlt"], torch.float64), t(torch, g["vsrc"], torch.float64), g64, shot)
    return g64.cpu().numpy()


def test_f64_snapshots_match_f64_strips(cuda):
    # in FP64 both reconstructions are exact up to rounding: the forward
    # field re-run from snapshots and the field back-propagated with strips
    # image the same gradient (the strips' source terms vanish in the
    # imaging window); intervals that give many segments, two, and one
    import swfwi_b200 as S
    torch = cuda
    s, m, g, vel = small_method(torch)
    strips = _interior(_grad64(torch, m, g, vel), s)
    for every in (7, 64, 1000):
        m.set_reconstruction(S.RECON_SNAPSHOTS, every, S.STRIP_F32)
        snap = _interior(_grad64(torch, m, g, vel), s)
        assert rel_l2(snap, strips) < 1e-11, (every, rel_l2(snap, strips))
    m.set_reconstruction(S.RECON_STRIPS)


@pytest.mark.parametrize("arith", [0, 1])
def test_f32_snapshots_independent_of_interval_and_closer_to_f64(cuda, arith):
    # FP32 snapshots restore the forward's own fields, so the re-run is the
    # forward bit for bit: the gradient does not depend on the interval, and
    # it is at least as close to FP64 as the strips' back-propagation
    import swfwi_b200 as S
    torch = cuda
    s, m, g, vel = small_method(torch, arith=arith)
    g64 = _interior(_grad64(torch, m, g, vel), s)
    strips_full = _grad(torch, m, g)
    strips = _interior(strips_full, s)
    outs = []
    for every in (7, 64, 1000):
        m.set_reconstruction(S.RECON_SNAPSHOTS, every, S.STRIP_F32)
        outs.append(_interior(_grad(torch, m, g), s))
    for o in outs[1:]:
        np.testing.assert_array_equal(o, outs[0])
    e_strips, e_snap = rel_l2(strips, g64), rel_l2(outs[0], g64)
    print(f"\ngradient rel-L2 vs FP64 ({('REF', 'FAST')[arith]}): strips {e_strips:.2e}  F32 snapshots {e_snap:.2e}")
    assert e_snap < 1e-5 and e_snap <= 1.5 * e_strips
    assert rel_l2(outs[0], strips) < 1e-4
    # back to strips: the same bits as before (the reference's, in REF)
    m.set_reconstruction(S.RECON_STRIPS)
    again = _grad(torch, m, g)
    np.testing.assert_array_equal(again, strips_full)
    if arith == 0:
        np.testing.assert_array_equal(again, g["grad_shot1"])


@pytest.mark.parametrize("fmt,bound", [(1, 2e-3), (2, 2e-2)])
def test_16bit_snapshots_gradient_error_vs_f64(cuda, fmt, bound):
    import swfwi_b200 as S
    torch = cuda
    s, m, g, vel = small_method(torch)
    g64 = _interior(_grad64(torch, m, g, vel), s)
    m.set_reconstruction(S.RECON_SNAPSHOTS, 16, fmt)
    q = _interior(_grad(torch, m, g), s)
    e = rel_l2(q, g64)
    print(f"\ngradient rel-L2 vs FP64, {('F16', 'BF16')[fmt - 1]} snapshots every 16 steps: {e:.2e}")
    assert np.isfinite(q).all() and e < bound, e


def test_batched_gradient_with_snapshots(cuda):
    # the batched gradient loop (all shots in one sweep; scaled and masked)
    # with FP32 snapshots: within FP32 tolerance of the reference's strips
    # result, and the same bits for any interval
    import swfwi_b200 as S
    torch = cuda
    s, m, g, _ = small_method(torch)
    res = []
    for every in (5, 50):
        m.set_reconstruction(S.RECON_SNAPSHOTS, every, S.STRIP_F32)
        gr = torch.zeros(g["grad_sum"].shape, device="cuda")
        obj = m.gradient_batch(t(torch, g["wlt"]), t(torch, g["dobs"]), [0, 1, 2], gr)
        res.append(gr.cpu().numpy())
        assert rel_l2(res[-1], g["grad_sum"]) < 1e-4
        assert abs(obj.sum() - float(g["obj"])) / float(g["obj"]) < 1e-5
    np.testing.assert_array_equal(res[0], res[1])


def test_reconstruction_arguments_checked(cuda):
    import swfwi_b200 as S
    torch = cuda
    s, m, g, vel = small_method(torch)
    with pytest.raises(S.SwfwiError):
        m.set_reconstruction(7, 16, S.STRIP_F32)
    with pytest.raises(S.SwfwiError):
        m.set_reconstruction(S.RECON_SNAPSHOTS, 1, S.STRIP_F32)
    with pytest.raises(S.SwfwiError):
        m.set_reconstruction(S.RECON_SNAPSHOTS, 16, 9)
