"""The learned preconditioner's CUDA kernels against the CPU oracle
(torch FP32 on the CPU with BF16 rounding at the same points).

Two kinds of inputs:
* exact: integer images and weights/biases on a 2^-6 grid, so that the
  FP32 sums of the forward pass do not depend on their order; the output
  must match to 1e-4 relative L2 (an indexing error shows as O(1); a sum
  that is not exact moves one BF16 rounding, 1e-6 here);
* random: seeded normal images and He-uniform weights.  The two sides sum
  in different orders, and a BF16 rounding that falls the other way moves
  one stored value by 2^-8 of itself and everything downstream of it; the
  output is held to 1e-2 and the parameter gradient to 5e-2 relative L2.
"""
import numpy as np
import pytest

from tests.conftest import rel_l2
from tests.test_precond_oracle import seeded_params

pytestmark = pytest.mark.gpu


def make_net(widths=(16, 32, 64, 64), seed=0):
    from swfwi_b200.precond import Preconditioner
    net = Preconditioner(widths)
    p = seeded_params(widths, seed)
    net.set_params(p)
    return net, p


def exact_params(widths=(16, 32, 64, 64), seed=0):
    from oracle.precond_oracle import layer_table
    layers, n = layer_table(widths)
    rng = np.random.default_rng(seed)
    p = np.zeros(n, np.float32)
    for ci, co, wo, bo in layers[:-1]:
        p[wo:wo + co * 9 * ci] = rng.integers(-3, 4, co * 9 * ci) / 64.0
        p[bo:bo + co] = rng.integers(-2, 5, co) / 64.0
    ci, _, wo, bo = layers[-1]
    p[wo:wo + ci] = rng.integers(-3, 4, ci) / 16.0
    p[bo] = 1 / 16.0
    return p


@pytest.mark.parametrize("N,H,W", [(1, 16, 24), (2, 24, 72), (1, 40, 136), (3, 8, 200)])
def test_exact_arithmetic_forward_matches_oracle(cuda, N, H, W):
    from oracle.precond_oracle import NetOracle
    from swfwi_b200.precond import Preconditioner
    torch = cuda
    p = exact_params(seed=N + H)
    net = Preconditioner()
    net.set_params(p)
    rng = np.random.default_rng(W)
    x = rng.integers(-3, 4, (N, H, W, 3)).astype(np.float32)
    t = rng.standard_normal((N, H, W)).astype(np.float32)
    y = net.forward(torch.from_numpy(x).cuda()).cpu().numpy()
    o = NetOracle(p, bf16=True)
    y_ref = o.forward(x)
    e = rel_l2(y, y_ref)
    net.backward(torch.from_numpy(t).cuda())
    _, g_ref = o.backward(t)
    eg = rel_l2(net.grads(), g_ref)
    print(f"exact inputs: output rel-L2 {e:.2e}, gradient rel-L2 {eg:.2e}")
    assert np.abs(y_ref).max() > 0
    assert e < 1e-4, e
    assert eg < 5e-2, eg


@pytest.mark.parametrize("N,H,W", [(1, 16, 24), (2, 24, 72), (1, 40, 136)])
def test_forward_and_gradient_match_oracle(cuda, N, H, W):
    from oracle.precond_oracle import NetOracle
    torch = cuda
    net, p = make_net()
    rng = np.random.default_rng(N * 1000 + H)
    x = rng.standard_normal((N, H, W, 3)).astype(np.float32)
    t = rng.standard_normal((N, H, W)).astype(np.float32)
    y = net.forward(torch.from_numpy(x).cuda())
    loss = net.backward(torch.from_numpy(t).cuda())
    g = net.grads()
    o = NetOracle(p, bf16=True)
    y_ref = o.forward(x)
    loss_ref, g_ref = o.backward(t)
    ey = rel_l2(y.cpu().numpy(), y_ref)
    eg = rel_l2(g, g_ref)
    print(f"output rel-L2 {ey:.2e}, gradient rel-L2 {eg:.2e}")
    assert ey < 1e-2, ey
    assert abs(loss - loss_ref) < 1e-2 * loss_ref
    assert eg < 5e-2, eg
    for l, (ci, co, wo, bo) in enumerate(o.layers):
        end = bo + co
        assert rel_l2(g[wo:end], g_ref[wo:end]) < 1e-1, l


def test_narrow_widths_match_oracle(cuda):
    from oracle.precond_oracle import NetOracle
    torch = cuda
    widths = (16, 16, 32, 16)
    net, p = make_net(widths, seed=3)
    rng = np.random.default_rng(5)
    x = rng.standard_normal((1, 16, 32, 3)).astype(np.float32)
    t = rng.standard_normal((1, 16, 32)).astype(np.float32)
    y = net.forward(torch.from_numpy(x).cuda())
    net.backward(torch.from_numpy(t).cuda())
    o = NetOracle(p, widths, bf16=True)
    assert rel_l2(y.cpu().numpy(), o.forward(x)) < 1e-2
    _, g_ref = o.backward(t)
    assert rel_l2(net.grads(), g_ref) < 5e-2


def test_adam_step_matches_formula(cuda):
    torch = cuda
    net, p = make_net()
    rng = np.random.default_rng(7)
    x = torch.from_numpy(rng.standard_normal((1, 16, 16, 3)).astype(np.float32)).cuda()
    t = torch.from_numpy(rng.standard_normal((1, 16, 16)).astype(np.float32)).cuda()
    net.forward(x)
    net.backward(t)
    g = net.grads()
    net.adam_step(1e-3)
    # first Adam step: m = 0.1 g, v = 0.001 g^2, lr_t = lr sqrt(1-0.999)/(1-0.9)
    lr_t = 1e-3 * np.sqrt(1 - 0.999) / (1 - 0.9)
    m = 0.1 * g
    v = 0.001 * g * g
    want = p - lr_t * m / (np.sqrt(v) + 1e-8)
    np.testing.assert_allclose(net.params(), want, rtol=1e-5, atol=1e-7)


def test_training_reduces_loss(cuda):
    torch = cuda
    net, _ = make_net()
    rng = np.random.default_rng(9)
    x = torch.from_numpy(rng.standard_normal((4, 32, 48, 3)).astype(np.float32)).cuda()
    # a smooth target the network can fit: a blurred copy of channel 0
    t = torch.nn.functional.avg_pool2d(x[..., 0][:, None], 5, 1, 2)[:, 0].contiguous() * 3
    losses = [net.train_step(x, t, 3e-3) for _ in range(60)]
    assert np.all(np.isfinite(losses))
    assert losses[-1] < 0.3 * losses[0], (losses[0], losses[-1])


def test_features_target_scatter(cuda):
    import swfwi_b200 as S
    from swfwi_b200.precond import image_shape
    from tests.gpu_helpers import small_method
    torch = cuda
    s, m, g, vel = small_method(torch)
    net, _ = make_net()
    nxpad, nzpad = m.dims()[:2]
    rng = np.random.default_rng(11)
    grad = rng.standard_normal((nxpad, nzpad)).astype(np.float32)
    il = np.abs(rng.standard_normal((nxpad, nzpad))).astype(np.float32) * 1e3
    H, W = image_shape(m)
    x3 = net.features(m, torch.from_numpy(grad).cuda(), vel, torch.from_numpy(il).cuda()).cpu().numpy()
    bx0, bz0 = s.nb + 6, 6
    nx, nz = s.nx, s.nz
    assert (H, W) == ((nx + 7) // 8 * 8, (nz + 7) // 8 * 8)
    gi = grad[bx0:bx0 + nx, bz0:bz0 + nz].astype(np.float64)
    vi = g["exvel_init"][bx0:bx0 + nx, bz0:bz0 + nz].astype(np.float64)
    ii = il[bx0:bx0 + nx, bz0:bz0 + nz].astype(np.float64)
    np.testing.assert_allclose(x3[:nx, :nz, 0], gi / np.sqrt((gi ** 2).mean()), rtol=1e-5, atol=1e-6)
    np.testing.assert_allclose(x3[:nx, :nz, 1], (vi - vi.mean()) / vi.std(), rtol=1e-4, atol=1e-4)
    np.testing.assert_allclose(x3[:nx, :nz, 2], (np.log10(ii / ii.max() + 1e-6) + 3) / 3, rtol=1e-4, atol=1e-5)
    assert np.all(x3[nx:] == 0) and np.all(x3[:, nz:] == 0)
    t = net.target(m, torch.from_numpy(grad).cuda()).cpu().numpy()
    np.testing.assert_allclose(t[:nx, :nz], gi / np.sqrt((gi ** 2).mean()), rtol=1e-5, atol=1e-6)
    d = net.propose(m, torch.from_numpy(grad).cuda(), vel, torch.from_numpy(il).cuda()).cpu().numpy()
    y = net.forward(torch.from_numpy(x3[None].copy()).cuda()).cpu().numpy()[0]
    np.testing.assert_array_equal(d[bx0:bx0 + nx, bz0:bz0 + nz], y[:nx, :nz])
    mask = np.ones_like(d, bool)
    mask[bx0:bx0 + nx, bz0:bz0 + nz] = False
    assert np.all(d[mask] == 0)
    with pytest.raises(S.SwfwiError):
        net.forward(torch.zeros((1, 12, 16, 3), device="cuda"))     # H not a multiple of 8


def test_learned_epoch_falls_back_and_keeps_decrease(cuda):
    """An untrained network attached to plain FWI: every epoch either takes
    a confirmed decrease along the network or the plain step; the objective
    never rises above the initial one."""
    import swfwi_b200 as S
    from swfwi_b200.precond import Preconditioner
    from tests.gpu_helpers import small_method
    torch = cuda
    s, m, g, vel = small_method(torch)
    fw = S.FwiFramework(m, g["exvel_init"], s.vmin, s.vmax, s.nita, s.maxdv, g["wlt"], g["dobs"])
    net = Preconditioner()
    fw.setPreconditioner(net)
    for it in range(3):
        fw.epoch(it)
        last, tried, acc = fw.learnedStats()
        assert tried == it + 1
        assert np.isfinite(fw.getUpdateObj())
    assert fw.getUpdateObj() < fw.getInitObj()
    il = fw.illumination()
    assert il.shape == g["exvel_init"].shape and il.max() > 0
    grad = fw.gradient()
    assert np.isfinite(grad).all() and np.abs(grad).max() > 0
    ess = S.EssFwiFramework(m, g["exvel_init"], s.vmin, s.vmax, s.nita, s.maxdv, g["wlt"], g["dobs"])
    with pytest.raises(S.SwfwiError):
        ess.setPreconditioner(net)


def test_training_is_bit_reproducible(cuda):
    # gradients are summed in a fixed order (no atomics): two trainings from
    # the same start on the same data give the same weights bit for bit
    torch = cuda
    rng = np.random.default_rng(21)
    x = torch.from_numpy(rng.standard_normal((3, 24, 40, 3)).astype(np.float32)).cuda()
    t = torch.from_numpy(rng.standard_normal((3, 24, 40)).astype(np.float32)).cuda()
    finals = []
    for _ in range(2):
        net, _ = make_net()
        for _ in range(5):
            net.train_step(x, t, 1e-3)
        finals.append(net.params())
    np.testing.assert_array_equal(finals[0], finals[1])
