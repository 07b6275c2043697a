"""Forward modelling, sources, receivers, strips and the data-side
operations on the GPU against the reference."""
import numpy as np
import pytest

from tests.conftest import golden, rel_l2
from tests.golden.make_golden import small_survey
from tests.gpu_helpers import small_method, t

pytestmark = pytest.mark.gpu


def test_forward_modeling_bit_exact(cuda):
    torch = cuda
    s, m, g, _ = small_method(torch)
    wlt = t(torch, g["wlt"])
    for shot in range(s.ns):
        d = torch.zeros((s.nt, s.ng), device="cuda")
        m.FwiForwardModeling(wlt, d, shot)
        np.testing.assert_array_equal(d.cpu().numpy(), g["dcal"][shot])


def test_forward_batch_bit_exact(cuda):
    torch = cuda
    s, m, g, _ = small_method(torch)
    d = torch.zeros((s.ns, s.nt, s.ng), device="cuda")
    m.forward_batch(t(torch, g["wlt"]), d, [2, 0, 1])
    np.testing.assert_array_equal(d.cpu().numpy(), g["dcal"][[2, 0, 1]])


def test_step_by_step_api_composes_forward(cuda):
    # FwiForwardModeling written out with the propagator's own calls
    # (damp4t10d.cpp:272-289): addSource, stepForward, swap, recordSeis.
    torch = cuda
    s, m, g, _ = small_method(torch)
    nxpad, nzpad = m.dims()[:2]
    wlt = t(torch, g["wlt"])
    p0 = torch.zeros((nxpad, nzpad), device="cuda")
    p1 = torch.zeros((nxpad, nzpad), device="cuda")
    d = torch.zeros((s.nt, s.ng), device="cuda")
    for it in range(s.nt):
        m.addSource(p1, wlt[it:], 1)
        m.stepForward(p0, p1)
        p0, p1 = p1, p0
        m.recordSeis(d[it], p0)
    np.testing.assert_array_equal(d.cpu().numpy(), g["dcal"][1])


def test_fast_forward_within_tolerance(cuda, fdo):
    import swfwi_b200 as S
    torch = cuda
    s, m, g, vel = small_method(torch, arith=S.ARITH_FAST)
    d = torch.zeros((s.nt, s.ng), device="cuda")
    m.FwiForwardModeling(t(torch, g["wlt"]), d, 1)
    err_ref = rel_l2(d.cpu().numpy(), g["dcal"][1])
    assert err_ref < 1e-5, err_ref
    # FP64 GPU oracle run of the same scheme
    d64 = torch.zeros((s.nt, s.ng), dtype=torch.float64, device="cuda")
    m.FwiForwardModeling_f64(vel, t(torch, g["wlt"], torch.float64), d64, 1)
    d64 = d64.cpu().numpy()
    bx0 = s.nb + 6
    nzpad = s.nz + s.nb + 12
    src = (s.sxbeg + 1 * s.jsx + bx0) * nzpad + s.szbeg + 6
    rec = (np.arange(s.ng) + bx0) * nzpad + s.gzbeg + 6
    cpu64 = fdo.forward_f64(g["exvel_init"].astype(np.float64), bx0, s.nt, g["wlt"].astype(np.float64), src, rec)
    assert rel_l2(d64, cpu64) < 1e-12
    print(f"seismogram rel-L2 vs FP64: REF {rel_l2(g['dcal'][1], d64):.2e}  FAST {rel_l2(d.cpu().numpy(), d64):.2e}")


@pytest.mark.parametrize("kern,bz,rows,depth", [(1, 376, 64, 3), (1, 248, 9, 7), (5, 120, 48, 3),
                                                (5, 120, 31, 7), (6, 120, 0, 3), (6, 120, 1, 3), (6, 120, 2, 3),
                                                (6, 120, 33, 3), (6, 120, 200, 3)])
def test_fast_forward_every_kernel_within_tolerance(cuda, kern, bz, rows, depth):
    # FAST arithmetic in every stencil kernel: seismogram within 1e-5
    # relative L2 of the reference's
    import swfwi_b200 as S
    torch = cuda
    s, m, g, vel = small_method(torch, arith=S.ARITH_FAST)
    m.set_tuning(kern, bz, rows, depth, 0)
    d = torch.zeros((s.nt, s.ng), device="cuda")
    m.FwiForwardModeling(t(torch, g["wlt"]), d, 1)
    err = rel_l2(d.cpu().numpy(), g["dcal"][1])
    assert err < 1e-5, err


def test_remove_direct_arrival_exact(cuda):
    torch = cuda
    s, m, g, _ = small_method(torch)
    for shot in range(s.ns):
        d = t(torch, g["dcal"][shot]).clone()
        m.fwiRemoveDirectArrival(d, shot)
        np.testing.assert_array_equal(d.cpu().numpy(), g["muted"][shot])
    d = t(torch, g["dcal"][0]).clone()
    m.removeDirectArrival(d)
    np.testing.assert_array_equal(d.cpu().numpy(), g["muted_ess"])


def test_trans_vsrc_exact(cuda):
    import swfwi_b200 as S
    torch = cuda
    g = golden("small_survey")
    out = torch.zeros(g["res"].shape, device="cuda")
    S.trans_vsrc(out, t(torch, g["res"]))
    np.testing.assert_array_equal(out.cpu().numpy(), g["vsrc"])


def test_ess_forward_bit_exact(cuda):
    torch = cuda
    s, m, g, _ = small_method(torch)
    enc = (g["wlt"][:, None] * g["ess_codes"][None, :].astype(np.float32)).astype(np.float32)
    d = torch.zeros((s.nt, s.ng), device="cuda")
    m.EssForwardModeling(t(torch, enc), d)
    np.testing.assert_array_equal(d.cpu().numpy(), g["ess_dcal"])


def test_boundary_strips_exact_and_round_trip(cuda):
    torch = cuda
    s, m, g, _ = small_method(torch)
    nxpad, nzpad = m.dims()[:2]
    field = torch.arange(nxpad * nzpad, dtype=torch.float32, device="cuda").reshape(nxpad, nzpad)
    b = m.initBndryVector(3)
    m.writeBndry(b, field, 2)
    bs = m.bndrySize()
    np.testing.assert_array_equal(b[2 * bs:].cpu().numpy(), g["bndr"])
    assert torch.count_nonzero(b[: 2 * bs]) == 0
    other = torch.zeros_like(field)
    m.readBndry(b, other, 2)
    mask = other != 0
    assert torch.equal(other[mask], field[mask]) and int(mask.sum()) >= bs - 1


def test_gpu_vs_reference_cfg0_grid(cuda, ref):
    # the 151 x 461 grid of the plain-FWI workload, 300 steps, one shot
    import swfwi_b200 as S
    from swfwi_b200 import survey as sv
    torch = cuda
    s = sv.config("fwi").scaled(nt=300)
    v = sv.layered_model(s.nx, s.nz, seed=1)
    M = ref.model(s)
    ex = M.expand_domain(v)
    wlt = ref.ricker(s.nt, s.fm, s.dt)
    want = M.fwi_forward(wlt, 7)
    m = S.Damp4t10d.from_survey(s)
    np.testing.assert_array_equal(m.expandDomain(v), ex)
    vel = t(torch, ex)
    m.bindVelocity(vel)
    d = torch.zeros((s.nt, s.ng), device="cuda")
    m.FwiForwardModeling(t(torch, wlt), d, 7)
    np.testing.assert_array_equal(d.cpu().numpy(), want)


def test_linearity_full_batched_grid(cuda):
    # size-independent property on the 301 x 921 grid: doubling the source
    # doubles every recorded sample (exact for normal floats; subnormal
    # amplitudes round on a fixed grid, so only to ~1e-7 overall)
    import swfwi_b200 as S
    from swfwi_b200 import survey as sv
    torch = cuda
    s = sv.config("encoded").scaled(nt=400)
    v = sv.layered_model(s.nx, s.nz, seed=3)
    m = S.Damp4t10d.from_survey(s)
    vel = t(torch, m.expandDomain(v))
    m.bindVelocity(vel)
    w = t(torch, S.ricker_wavelet(s.nt, s.fm, s.dt))
    d1 = torch.zeros((2, s.nt, s.ng), device="cuda")
    d2 = torch.zeros_like(d1)
    m.forward_batch(w, d1, [0, 95])
    m.forward_batch(w * 2, d2, [0, 95])
    err = float((d2 - d1 * 2).norm() / (d1 * 2).norm())
    assert err < 1e-6, err
    assert float(d1.abs().max()) > 0


def test_errors_reported(cuda):
    import swfwi_b200 as S
    torch = cuda
    s, m, g, _ = small_method(torch)
    d = torch.zeros((s.nt, s.ng), device="cuda")
    with pytest.raises(S.SwfwiError) as e:
        m.FwiForwardModeling(t(torch, g["wlt"]), d, s.ns)   # shot id out of range
    assert e.value.status == 1
    s2, _, _ = small_survey()
    m2 = S.Damp4t10d.from_survey(s2)
    with pytest.raises(S.SwfwiError) as e:
        m2.FwiForwardModeling(t(torch, g["wlt"]), d, 0)     # no velocity bound
    assert e.value.status == 6
    bad = s2.scaled(gxbeg=s2.nx - 3)                        # receivers beyond the grid
    with pytest.raises(S.SwfwiError):
        S.Damp4t10d.from_survey(bad)


@pytest.mark.parametrize("kern,bz,rows,depth,order", [
    (1, 120, 1, 3, 1), (1, 248, 9, 7, 0), (1, 376, 64, 7, 0), (1, 376, 3, 3, 1), (1, 120, 200, 7, 0),
    (1, 376, 16, 3, 0), (1, 248, 33, 3, 1),
    (5, 120, 1, 3, 0), (5, 120, 9, 7, 0), (5, 120, 64, 3, 0), (5, 120, 33, 7, 0), (5, 120, 200, 3, 0),
    (5, 120, 11, 3, 0), (5, 120, 12, 7, 0), (5, 120, 8, 3, 0), (5, 120, 16, 7, 0),
    (5, 120, 0, 3, 0), (5, 120, 0, 7, 0), (1, 376, 0, 3, 0), (6, 120, 0, 3, 0), (6, 120, 5, 3, 0)])
def test_stream_launch_shapes_bit_exact(cuda, kern, bz, rows, depth, order):
    # every band depth / chunk length of the streaming stencil gives the
    # reference's seismogram bit for bit
    torch = cuda
    s, m, g, _ = small_method(torch)
    m.set_tuning(kern, bz, rows, depth, order)
    d = torch.zeros((s.nt, s.ng), device="cuda")
    m.FwiForwardModeling(t(torch, g["wlt"]), d, 2)
    np.testing.assert_array_equal(d.cpu().numpy(), g["dcal"][2])


@pytest.mark.parametrize("kern,bz,depth", [(1, 120, 7), (1, 248, 3), (1, 376, 3), (1, 376, 7),
                                           (5, 120, 3), (5, 120, 7), (6, 120, 3)])
def test_stream_matches_reference_large_grid(cuda, ref, kern, bz, depth):
    # 921 x 301 (993 x 343 padded, pitch 344): several bands, a short last
    # band, many chunks
    import swfwi_b200 as S
    from swfwi_b200 import survey as sv
    torch = cuda
    s = sv.config("encoded").scaled(nt=120, ns=4, sxbeg=100, jsx=200)
    v = sv.layered_model(s.nx, s.nz, seed=8)
    M = ref.model(s)
    ex = M.expand_domain(v)
    wlt = ref.ricker(s.nt, s.fm, s.dt)
    m = S.Damp4t10d.from_survey(s)
    m.set_tuning(kern, bz, 50, depth, 1)
    vel = t(torch, ex)
    m.bindVelocity(vel)
    d = torch.zeros((s.nt, s.ng), device="cuda")
    m.FwiForwardModeling(t(torch, wlt), d, 3)
    np.testing.assert_array_equal(d.cpu().numpy(), M.fwi_forward(wlt, 3))


def test_graph_loops_bit_exact_and_timed(cuda):
    # the same batched forward and gradient with the time loops replayed as
    # CUDA graphs (second and later calls) and launched one by one
    import time
    import swfwi_b200 as S
    from swfwi_b200 import survey as sv
    torch = cuda
    s = sv.config("fwi").scaled(nt=600, ns=6, sxbeg=40, jsx=70)
    v = sv.layered_model(s.nx, s.nz, seed=5)
    out = {}
    for graphs in (False, True):
        m = S.Damp4t10d.from_survey(s, arith=S.ARITH_FAST)
        m.set_graphs(graphs)
        vel = t(torch, m.expandDomain(v))
        m.bindVelocity(vel)
        w = t(torch, S.ricker_wavelet(s.nt, s.fm, s.dt))
        d = torch.zeros((s.ns, s.nt, s.ng), device="cuda")
        ids = list(range(s.ns))
        m.forward_batch(w, d, ids)          # first use: direct launches
        grad = torch.zeros_like(vel)
        m.gradient_batch(w, d * 1.01, ids, grad)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(3):
            m.forward_batch(w, d, ids)
            m.gradient_batch(w, d * 1.01, ids, grad)
        torch.cuda.synchronize()
        out[graphs] = (d.cpu().numpy(), grad.cpu().numpy(), (time.perf_counter() - t0) / 3)
    np.testing.assert_array_equal(out[True][0], out[False][0])
    np.testing.assert_array_equal(out[True][1], out[False][1])
    print(f"forward + gradient, 6 shots of 533 x 193, nt 600: launches {out[False][2] * 1e3:.1f} ms, "
          f"graphs {out[True][2] * 1e3:.1f} ms")


def test_graph_replay_reads_current_data(cuda):
    # replayed loops (same pointers) see new input contents; alternating
    # output buffers select their own cached graphs
    import swfwi_b200 as S
    from swfwi_b200 import survey as sv
    torch = cuda
    s = sv.config("fwi").scaled(nt=300, ns=4, sxbeg=60, jsx=100)
    v = sv.layered_model(s.nx, s.nz, seed=9)
    m = S.Damp4t10d.from_survey(s, arith=S.ARITH_FAST)
    vel = t(torch, m.expandDomain(v))
    m.bindVelocity(vel)
    w = t(torch, S.ricker_wavelet(s.nt, s.fm, s.dt))
    ids = list(range(s.ns))
    ref = torch.zeros((s.ns, s.nt, s.ng), device="cuda")
    m.set_graphs(False)
    m.forward_batch(w, ref, ids)
    m.set_graphs(True)
    outs = [torch.zeros_like(ref) for _ in range(2)]
    for rep in range(3):
        for d in outs:
            d.zero_()
            m.forward_batch(w, d, ids)
            assert torch.equal(d, ref)
    w.mul_(2.0)                              # same pointer, new contents
    m.forward_batch(w, outs[0], ids)
    # doubling is exact for normal floats; subnormals round on a fixed grid
    err = float((outs[0] - ref * 2).norm() / (ref * 2).norm())
    assert err < 1e-6, err


def test_graph_replay_counts_and_times_like_direct_launches(cuda):
    # stencil timing inside replayed loops: the same launch and work counts
    # as direct launches, and every timed launch has a positive time
    import swfwi_b200 as S
    from swfwi_b200 import survey as sv
    torch = cuda
    s = sv.config("fwi").scaled(nt=200, ns=3, sxbeg=60, jsx=100)
    v = sv.layered_model(s.nx, s.nz, seed=4)
    stats = {}
    for graphs in (0, 2):
        m = S.Damp4t10d.from_survey(s, arith=S.ARITH_FAST)
        m.set_graphs(graphs)
        vel = t(torch, m.expandDomain(v))
        m.bindVelocity(vel)
        w = t(torch, S.ricker_wavelet(s.nt, s.fm, s.dt))
        d = torch.zeros((s.ns, s.nt, s.ng), device="cuda")
        grad = torch.zeros_like(vel)
        ids = list(range(s.ns))
        S.stats_enable_step_timing(4)
        for _ in range(2):                  # mode 2: captured at once
            m.gradient_batch(w, d + 1e-3, ids, grad)
        torch.cuda.synchronize()
        S.stats_reset()
        for _ in range(3):                  # replayed (graphs 2)
            m.gradient_batch(w, d + 1e-3, ids, grad)
        torch.cuda.synchronize()
        stats[graphs] = S.stats_read()
        S.stats_enable_step_timing(False)
        del m
    a, b = stats[0], stats[2]
    for k in ("kernel_launches", "step_launches"):
        assert a[k] == b[k], (k, a[k], b[k])
    # every 4th launch: counted across loops when launched directly, from
    # each loop's start inside a graph
    assert abs(a["step_timed_launches"] - b["step_timed_launches"]) <= 3
    assert a["step_point_updates"] == b["step_point_updates"]
    assert b["step_ms"] > 0 and a["step_ms"] > 0
    # per-launch times agree to within the two paths' launch overheads
    ra = a["step_ms"] / a["step_timed_launches"]
    rb = b["step_ms"] / b["step_timed_launches"]
    assert 0.5 < rb / ra < 2.0, (ra, rb)



@pytest.mark.parametrize("rows", [0, 1, 2, 7, 8, 33, 64, 200])
def test_two_row_kernel_bit_identical_to_one_row_kernel(cuda, rows):
    # FAST: kernel 6 (two rows a stage) and kernel 5 give the same
    # seismogram bit for bit, for even and odd task lengths
    import swfwi_b200 as S
    torch = cuda
    s, m, g, vel = small_method(torch, arith=S.ARITH_FAST)
    out = []
    for kern in (5, 6):
        m.set_tuning(kern, 120, rows, 3, 0)
        d = torch.zeros((s.nt, s.ng), device="cuda")
        m.FwiForwardModeling(t(torch, g["wlt"]), d, 1)
        out.append(d.cpu().numpy())
    np.testing.assert_array_equal(out[0], out[1])
