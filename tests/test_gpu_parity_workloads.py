"""Gradient parity on the benchmarked workloads' own grids and acquisitions.

* The batched gradient's workload: 301 x 921 (993 x 343 padded), dx 10 m,
  dt 1 ms, 15 Hz, the benchmark's seeded uneven receiver spreads (seed 11);
  four of its shots (the two shortest and the two longest spreads), time
  axis cut to 900 steps so the backward sweep still reaches its 0.3 s stop
  and the 0.3-0.4 s taper.  Every shot is checked against a reference model
  built with that shot's own receiver line (the reference has one common
  line), in FAST arithmetic (FP32 with FMA, the benchmark's), in REF
  arithmetic (bit for bit), with FP16 and BF16 strips, and against the FP64
  GPU run of the same scheme.
* The plain-FWI workload: 151 x 461, dx 25 m, dt 2 ms, three of its twenty
  shots, 600 steps.

Tolerance: gradients within 1e-4 relative L2 of the reference (FP32);
objectives within 1e-5 in REF arithmetic (summed in FP64 here, in float by
the reference) and 1e-4 in FAST.
"""
import numpy as np
import pytest

from tests.conftest import rel_l2
from tests.gpu_helpers import t

pytestmark = pytest.mark.gpu

GRAD_TOL = 1e-4
OBJ_TOL_FAST = 1e-4
KERNELS = [(1, 376, 64, 3, 0), (5, 120, 0, 3, 0), (5, 120, 48, 7, 0), (6, 120, 0, 3, 0), (6, 120, 77, 3, 0)]


def _batched_case(ref, nt=900, picks=4):
    """Reference gradients for `picks` shots of the batched workload."""
    from swfwi_b200 import survey as sv
    full = sv.config("batched").scaled(nt=nt)
    off, gx, gz = full.spreads
    lens = np.diff(off)
    order = np.argsort(lens, kind="stable")
    ids = sorted(set(order[:picks // 2].tolist() + order[-(picks - picks // 2):].tolist()))
    v = sv.layered_model(full.nx, full.nz, seed=1)
    vi = sv.smooth(v, 15).astype(np.float32)
    wlt = ref.ricker(full.nt, full.fm, full.dt)
    # observed data indexed by shot id, as the batched gradient reads it
    dobs = np.zeros((full.ns, full.nt, full.ngmax), np.float32)
    want_g = None
    want_obj = 0.0
    per_shot = []
    for i in ids:
        n = int(lens[i])
        ss = full.scaled(ng=n, gxbeg=int(gx[off[i]]), sxbeg=int(full.src_x()[i]), ns=1, jsx=1, spreads=None)
        M = ref.model(ss)
        if want_g is None:
            ext, exi = M.expand_domain(v), M.expand_domain(vi)
            want_g = np.zeros_like(ext)
        M.bind_velocity(ext)
        dobs[i, :, :n] = M.fwi_forward(wlt, 0)
        M.bind_velocity(exi)
        gs, o = M.fwi_gradient(wlt, dobs[i:i + 1, :, :n])
        want_g = (want_g + gs).astype(np.float32)
        want_obj += o
        per_shot.append((i, ss, M, n))
    return dict(s=full, ids=ids, ext=ext, exi=exi, wlt=wlt, dobs=dobs, grad=want_g, obj=want_obj,
                per_shot=per_shot)


@pytest.fixture(scope="module")
def batched_case(ref):
    return _batched_case(ref)


def _gpu_gradient(torch, case, arith, tuning=None, strips=None):
    import swfwi_b200 as S
    m = S.Damp4t10d.from_survey(case["s"], arith=arith)
    if tuning is not None:
        m.set_tuning(*tuning)
    if strips is not None:
        m.set_strip_format(strips)
    vel = t(torch, case["exi"])
    m.bindVelocity(vel)
    gr = torch.zeros(case["ext"].shape, device="cuda")
    obj = m.gradient_batch(t(torch, case["wlt"]), t(torch, case["dobs"]), case["ids"], gr)
    return gr.cpu().numpy(), float(obj.sum())


@pytest.mark.parametrize("tuning", KERNELS)
def test_batched_workload_gradient_ref_bit_exact(cuda, batched_case, tuning):
    import swfwi_b200 as S
    g, obj = _gpu_gradient(cuda, batched_case, S.ARITH_REF, tuning)
    np.testing.assert_array_equal(g, batched_case["grad"])
    assert abs(obj - batched_case["obj"]) / batched_case["obj"] < 1e-5


@pytest.mark.parametrize("tuning", KERNELS)
def test_batched_workload_gradient_fast(cuda, batched_case, tuning):
    import swfwi_b200 as S
    g, obj = _gpu_gradient(cuda, batched_case, S.ARITH_FAST, tuning)
    e = rel_l2(g, batched_case["grad"])
    print(f"FAST gradient rel-L2 vs reference, 4 shots of 993 x 343, nt 900, kernel {tuning[0]}: {e:.2e}")
    assert e < GRAD_TOL, e
    # the objective is a sum of squared residuals, differences of nearly
    # equal seismograms: FAST's ~1e-6 seismogram error moves it ~1e-5
    assert abs(obj - batched_case["obj"]) / batched_case["obj"] < OBJ_TOL_FAST


def test_fast_kernels_give_identical_bits(cuda, batched_case):
    # kernels 5 and 6 evaluate every point in kernel 1's operation order
    import swfwi_b200 as S
    a, _ = _gpu_gradient(cuda, batched_case, S.ARITH_FAST, KERNELS[0])
    for kern in KERNELS[1:]:
        b, _ = _gpu_gradient(cuda, batched_case, S.ARITH_FAST, kern)
        np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("fmt", [1, 2])
def test_batched_workload_16bit_strips(cuda, batched_case, fmt):
    import swfwi_b200 as S
    g, obj = _gpu_gradient(cuda, batched_case, S.ARITH_FAST, KERNELS[1], strips=fmt)
    e = rel_l2(g, batched_case["grad"])
    print(f"FAST gradient with {('F16', 'BF16')[fmt - 1]} strips, rel-L2 vs reference: {e:.2e}")
    assert np.isfinite(g).all() and e < GRAD_TOL, e


def test_batched_workload_against_f64(cuda, ref, batched_case):
    # per shot: the FP64 GPU run of the scheme fed the reference's own
    # adjoint source; FAST, REF and the reference itself stated against it
    import swfwi_b200 as S
    torch = cuda
    case = batched_case
    errs = {"ref": [], "fast": [], "cpu": []}
    for i, ss, M, n in (case["per_shot"][0], case["per_shot"][-1]):
        wlt = case["wlt"]
        M.bind_velocity(case["exi"])
        cal = M.remove_direct_arrival(M.fwi_forward(wlt, 0), 0)
        obs = M.remove_direct_arrival(np.ascontiguousarray(case["dobs"][i, :, :n]), 0)
        vsrc = ref.trans_vsrc((obs - cal).astype(np.float32))
        want = M.mask_gradient(M.scale_gradient(M.calgradient_fwi(wlt, vsrc, 0)))
        m64 = S.Damp4t10d.from_survey(ss)
        vel = t(torch, case["exi"])
        m64.bindVelocity(vel)
        g64 = torch.zeros(case["ext"].shape, dtype=torch.float64, device="cuda")
        m64.calgradient_fwi_f64(vel, t(torch, wlt, torch.float64), t(torch, vsrc, torch.float64), g64, 0)
        g64 = g64.cpu().numpy()
        # scaleGradient / maskGradient in FP64 (damp4t10d.cpp:216-226,
        # 309-319): interior depth iz >= 1 times sqrt(iz), iz = 0 kept,
        # zero outside the interior
        bz0, bx0 = 6, ss.nb + 6
        nxpad, nzpad = g64.shape
        iz = np.arange(nzpad - bz0 - bx0, dtype=np.float64)
        sc = np.zeros_like(g64)
        sc[bx0:nxpad - bx0, bz0:nzpad - bx0] = np.where(iz >= 1, np.sqrt(iz), 1.0)[None, :]
        g64 = g64 * sc
        for arith, key in ((S.ARITH_REF, "ref"), (S.ARITH_FAST, "fast")):
            m = S.Damp4t10d.from_survey(ss, arith=arith)
            m.set_tuning(*KERNELS[1])
            m.bindVelocity(vel)
            g = torch.zeros(case["ext"].shape, device="cuda")
            m.calgradient_fwi(t(torch, wlt), t(torch, vsrc), g, 0)
            m.scaleGradient(g)
            m.maskGradient(g)
            errs[key].append(rel_l2(g.cpu().numpy(), g64))
        errs["cpu"].append(rel_l2(want, g64))
    print("gradient rel-L2 vs FP64 GPU run (993 x 343, nt 900): "
          + "  ".join(f"{k} {max(v):.2e}" for k, v in errs.items()))
    for k, v in errs.items():
        assert max(v) < GRAD_TOL, (k, v)


def test_plain_fwi_workload_gradient(cuda, ref):
    # three shots of the 151 x 461 plain-FWI workload, common receiver line
    import swfwi_b200 as S
    from swfwi_b200 import survey as sv
    torch = cuda
    full = sv.config("fwi")
    s = full.scaled(nt=600, ns=3, sxbeg=int(full.src_x()[1]), jsx=int(full.src_x()[10] - full.src_x()[1]))
    v = sv.layered_model(s.nx, s.nz, seed=3)
    vi = sv.smooth(v, 15).astype(np.float32)
    M = ref.model(s)
    ext, exi = M.expand_domain(v), M.expand_domain(vi)
    wlt = ref.ricker(s.nt, s.fm, s.dt)
    M.bind_velocity(ext)
    dobs = np.stack([M.fwi_forward(wlt, i) for i in range(s.ns)]).astype(np.float32)
    M.bind_velocity(exi)
    want, want_obj = M.fwi_gradient(wlt, dobs)
    for arith in (S.ARITH_REF, S.ARITH_FAST):
        m = S.Damp4t10d.from_survey(s, arith=arith)
        m.set_tuning(*KERNELS[1])
        vel = t(torch, exi)
        m.bindVelocity(vel)
        gr = torch.zeros(ext.shape, device="cuda")
        obj = m.gradient_batch(t(torch, wlt), t(torch, dobs), [0, 1, 2], gr)
        g = gr.cpu().numpy()
        if arith == S.ARITH_REF:
            np.testing.assert_array_equal(g, want)
        else:
            e = rel_l2(g, want)
            print(f"FAST gradient rel-L2 vs reference, 3 shots of 193 x 533, nt 600: {e:.2e}")
            assert e < GRAD_TOL
        tol = 1e-5 if arith == S.ARITH_REF else OBJ_TOL_FAST
        assert abs(obj.sum() - want_obj) / want_obj < tol
