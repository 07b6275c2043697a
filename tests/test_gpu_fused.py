"""The fused backward time loop (source subtraction and imaging in the
source back-step, residual injection in the receiver step) against the
separate-launch path and the compiled reference, over geometries that
exercise each way a line meets the rows."""
import numpy as np
import pytest

from tests.conftest import golden
from tests.gpu_helpers import small_method, t

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("arith", [0, 1])
def test_fused_and_separate_paths_identical(cuda, arith):
    # same kernels' arithmetic either way: bit-identical seismograms, and
    # gradients in REF; in FAST the separate path images every shot into
    # one image (summed before the scale), so its gradient matches to
    # rounding
    from tests.conftest import rel_l2
    torch = cuda
    out = []
    for fuse in (True, False):
        s, m, g, _ = small_method(torch, arith=arith)
        m.set_fusion(fuse)
        d = torch.zeros((s.ns, s.nt, s.ng), device="cuda")
        m.forward_batch(t(torch, g["wlt"]), d, [0, 1, 2])
        gr = torch.zeros(g["grad_sum"].shape, device="cuda")
        obj = m.gradient_batch(t(torch, g["wlt"]), t(torch, g["dobs"]), [0, 1, 2], gr)
        out.append((d.cpu().numpy(), gr.cpu().numpy(), obj))
    np.testing.assert_array_equal(out[0][0], out[1][0])
    if arith == 0:
        np.testing.assert_array_equal(out[0][1], out[1][1])
    else:
        assert rel_l2(out[1][1], out[0][1]) < 1e-6
    np.testing.assert_array_equal(out[0][2], out[1][2])
    if arith == 0:
        np.testing.assert_array_equal(out[0][0], golden("small_survey")["dcal"])


@pytest.mark.parametrize("geom", [
    dict(jgx=2, ng=30),                                    # receivers on every other row
    dict(jgx=0, jgz=1, gxbeg=33, gzbeg=2, ng=30),          # a vertical receiver line (a well)
    dict(jsz=3, jsx=7, szbeg=2, sxbeg=5, ns=3, jgx=1),     # sources on a diagonal
])
def test_fused_geometries_match_reference(cuda, ref, geom):
    import swfwi_b200 as S
    from swfwi_b200 import survey as sv
    torch = cuda
    s = sv.small(nx=60, nz=40, nt=160, ns=3).scaled(**geom)
    if "ng" not in geom:
        s = s.scaled(ng=min(s.ng, 60))
    v = sv.layered_model(s.nx, s.nz, seed=12)
    M = ref.model(s)
    ex = M.expand_domain(v)
    wlt = ref.ricker(s.nt, s.fm, s.dt)
    m = S.Damp4t10d.from_survey(s)
    m.set_fusion(True)
    vel = t(torch, ex)
    m.bindVelocity(vel)
    d = torch.zeros((s.ns, s.nt, s.ng), device="cuda")
    m.forward_batch(t(torch, wlt), d, list(range(s.ns)))
    got = d.cpu().numpy()
    for shot in range(s.ns):
        np.testing.assert_array_equal(got[shot], M.fwi_forward(wlt, shot))
    # the encoded supershot: all sources of the line in one field
    codes = np.array([1, -1, 1][: s.ns], np.int32)
    enc = (wlt[:, None] * codes[None, :].astype(np.float32)).astype(np.float32)
    de = torch.zeros((s.nt, s.ng), device="cuda")
    m.EssForwardModeling(t(torch, enc), de)
    np.testing.assert_array_equal(de.cpu().numpy(), M.ess_forward(enc))
    # gradients through the fused backward (lines the fused steps can inject
    # on) and the separate one: the same bits
    vi = sv.smooth(v, 3.0).astype(np.float32)
    veli = t(torch, m.expandDomain(vi))
    m.bindVelocity(veli)
    grads = []
    for fuse in (True, False):
        m.set_fusion(fuse)
        gr = torch.zeros(ex.shape, device="cuda")
        obj = m.gradient_batch(t(torch, wlt), d, list(range(s.ns)), gr)
        grads.append((gr.cpu().numpy(), obj))
    np.testing.assert_array_equal(grads[0][0], grads[1][0])
    np.testing.assert_array_equal(grads[0][1], grads[1][1])
    assert np.abs(grads[0][0]).max() > 0


def test_fused_ess_gradient_bit_exact(cuda):
    torch = cuda
    s, m, g, _ = small_method(torch)
    m.set_fusion(True)
    enc = (g["wlt"][:, None] * g["ess_codes"][None, :].astype(np.float32)).astype(np.float32)
    gr = torch.zeros(g["grad_ess"].shape, device="cuda")
    m.calgradient_ess(t(torch, enc), t(torch, g["vsrc"]), gr)
    np.testing.assert_array_equal(gr.cpu().numpy(), g["grad_ess"])


def test_fused_strips_gradient_bit_exact(cuda):
    # the gradient's forward sweep saves FP32 strips in the fused step
    torch = cuda
    s, m, g, _ = small_method(torch)
    m.set_fusion(True)
    gr = torch.zeros(g["grad_shot1"].shape, device="cuda")
    m.calgradient_fwi(t(torch, g["wlt"]), t(torch, g["vsrc"]), gr, 1)
    np.testing.assert_array_equal(gr.cpu().numpy(), g["grad_shot1"])
