"""The LSRTM operator (src/unused/prtm2d.cpp) on the GPU.

REF arithmetic against the reference's own outputs (committed fixture):
bit for bit, for two Born calls on one operator (the second continuing from
the receiver fields the first left, as the reference's does), the migration,
and the migration added onto a model.  FAST arithmetic (shots batched, every
shot from zero fields) against the FP64 restatement within 1e-4 relative L2
(the migration: within three times the reference's own float error).
The exact-adjoint mode against the restatement's transpose, and by the
dot-product test (FP32: 1e-5 relative) on a larger survey."""
import numpy as np
import pytest

from oracle.prtm_oracle import PrtmF64
from tests.conftest import golden, rel_l2
from tests.golden.make_golden import PRTM_CASES
from tests.gpu_helpers import t

pytestmark = pytest.mark.gpu

TOL_FAST = 1e-4
TOL_DOT = 1e-5


def _args(case):
    c = dict(PRTM_CASES[case])
    c.pop("nx")
    c.pop("nz")
    return c


def _op(torch, case, arith, vel=None):
    import swfwi_b200 as S
    g = golden("prtm")
    v = t(torch, g[case + "_vel"] if vel is None else vel)
    return S.Prtm2d(v, arith=arith, **_args(case)), g


@pytest.mark.parametrize("case", sorted(PRTM_CASES))
def test_ref_matches_reference_bit_for_bit(cuda, case):
    import swfwi_b200 as S
    torch = cuda
    op, g = _op(torch, case, S.ARITH_REF)
    assert op.batch() == 1
    mod = t(torch, g[case + "_mod"])
    dat = t(torch, g[case + "_dat"])
    b = torch.full_like(dat, 7.0)        # add = 0 must overwrite
    op.lop(False, False, mod, b)
    np.testing.assert_array_equal(b.cpu().numpy(), g[case + "_born1"])
    op.lop(False, False, mod, b)
    np.testing.assert_array_equal(b.cpu().numpy(), g[case + "_born2"])
    m = torch.full_like(mod, -3.0)
    op.lop(True, False, m, dat)
    np.testing.assert_array_equal(m.cpu().numpy(), g[case + "_mig"])
    m = t(torch, g[case + "_base"])
    op.lop(True, True, m, dat)
    np.testing.assert_array_equal(m.cpu().numpy(), g[case + "_mig_add"])
    op.close()


@pytest.mark.parametrize("case", sorted(PRTM_CASES))
def test_fast_born_and_migration(cuda, case):
    import swfwi_b200 as S
    torch = cuda
    op, g = _op(torch, case, S.ARITH_FAST)
    assert op.batch() == PRTM_CASES[case]["ns"]
    o = PrtmF64(g[case + "_vel"], **_args(case))
    mod = t(torch, g[case + "_mod"])
    dat = t(torch, g[case + "_dat"])
    b = torch.zeros_like(dat)
    op.lop(False, False, mod, b)
    assert rel_l2(b.cpu().numpy(), o.born(g[case + "_mod"])) < TOL_FAST
    # the migration reconstructs the source field backwards in time, which
    # FP32 rounding perturbs: against FP64, FAST may be off by three times
    # the reference's own float error (6e-3 on the thin-sponge gather case)
    mig = o.migration(g[case + "_dat"])
    tol = max(TOL_FAST, 3 * rel_l2(g[case + "_mig"], mig))
    m = torch.zeros_like(mod)
    op.lop(True, False, m, dat)
    assert rel_l2(m.cpu().numpy(), mig) < tol
    m = t(torch, g[case + "_base"])
    op.lop(True, True, m, dat)
    assert rel_l2(m.cpu().numpy() - g[case + "_base"], mig) < tol
    op.close()


# exact adjoint against the FP64 transpose, on data the operator makes
# (d = L m): the GPU reconstructs the source field backwards in FP32; with
# the thinnest sponge (gather, nb = 2) that drifts, as the reference's own
# float migration does there (1.6e-4 from FP64 on the same data)
EXACT_TOL = {"line": 1e-4, "gather": 2e-3}


@pytest.mark.parametrize("case", sorted(PRTM_CASES))
@pytest.mark.parametrize("arith", [0, 1])
def test_exact_adjoint_matches_transpose(cuda, case, arith):
    import swfwi_b200 as S
    torch = cuda
    op, g = _op(torch, case, arith)
    op.set_adjoint(S.PRTM_ADJ_EXACT)
    o = PrtmF64(g[case + "_vel"], **_args(case))
    d = o.born(g[case + "_mod"]).astype(np.float32)
    m = torch.zeros(g[case + "_mod"].shape, dtype=torch.float32, device="cuda")
    op.lop(True, False, m, t(torch, d))
    assert rel_l2(m.cpu().numpy(), o.born_transpose(d)) < EXACT_TOL[case]
    op.close()


@pytest.mark.parametrize("csd", [0, 1])
def test_fast_pair_passes_dot_product(cuda, csd):
    import swfwi_b200 as S
    torch = cuda
    rng = np.random.default_rng(40 + csd)
    nx, nz, nt, ns, ng = 160, 120, 600, 6, 20
    vel = t(torch, rng.uniform(1500, 3500, (nx, nz)).astype(np.float32))
    op = S.Prtm2d(vel, dz=10.0, dx=10.0, dt=1e-3, amp=1.0, fm=15.0, nb=30, nt=nt, ns=ns, ng=ng, sxbeg=10, szbeg=2,
                  jsx=25, jsz=0, gxbeg=0 if csd else 5, gzbeg=3, jgx=1 if csd else 3, jgz=0, csdgather=bool(csd),
                  arith=S.ARITH_FAST)
    op.set_adjoint(S.PRTM_ADJ_EXACT)
    m = t(torch, rng.standard_normal((nx, nz)).astype(np.float32))
    d = t(torch, rng.standard_normal((ns, ng, nt)).astype(np.float32))
    lm = torch.zeros_like(d)
    op.lop(False, False, m, lm)
    ltd = torch.zeros_like(m)
    op.lop(True, False, ltd, d)
    a = float(torch.dot(lm.double().ravel(), d.double().ravel()))
    b = float(torch.dot(m.double().ravel(), ltd.double().ravel()))
    assert abs(a - b) <= TOL_DOT * abs(a), (a, b)
    # the reference's migration on the same operator is not the adjoint
    op.set_adjoint(S.PRTM_ADJ_REFERENCE)
    op.lop(True, False, ltd, d)
    c = float(torch.dot(m.double().ravel(), ltd.double().ravel()))
    assert abs(a - c) > 0.3 * max(abs(a), abs(c))
    op.close()


def test_bad_geometry_and_sizes_are_rejected(cuda):
    import swfwi_b200 as S
    torch = cuda
    vel = torch.full((20, 16), 2000.0, device="cuda")
    kw = dict(dz=10.0, dx=10.0, dt=1e-3, amp=1.0, fm=15.0, nb=4, nt=10, ns=2, ng=3, sxbeg=2, szbeg=1, jsx=5, jsz=0,
              gxbeg=0, gzbeg=0, jgx=2, jgz=0)
    for bad in (dict(jsx=-5), dict(sxbeg=19, jsx=1), dict(gzbeg=16), dict(jgx=-1), dict(nb=1)):
        with pytest.raises(S.SwfwiError):
            S.Prtm2d(vel, **{**kw, **bad})
    with pytest.raises(S.SwfwiError):
        # common-shot gathers that walk off the model with the last shot
        S.Prtm2d(vel, **{**kw, "sxbeg": 10, "gxbeg": 8, "jgx": 4, "jsx": 5, "csdgather": True})
    op = S.Prtm2d(vel, **kw)
    with pytest.raises(S.SwfwiError):
        op.lop(False, False, torch.zeros(20, 15, device="cuda"), torch.zeros(2, 3, 10, device="cuda"))
    with pytest.raises(S.SwfwiError):
        op.lop(True, False, torch.zeros(20, 16, device="cuda"), torch.zeros(2, 3, 9, device="cuda"))
    with pytest.raises(S.SwfwiError):
        op.set_adjoint(2)
    op.close()


@pytest.mark.parametrize("arith", [0, 1])
def test_graph_replay_is_bit_identical(cuda, arith):
    # first call eager, second captured, third replayed; and with graphs off
    import swfwi_b200 as S
    torch = cuda
    case = "line"
    outs = []
    for graphs in (True, False):
        op, g = _op(torch, case, arith)
        op.set_graphs(graphs)
        mod = t(torch, g[case + "_mod"])
        dat = t(torch, g[case + "_dat"])
        b = torch.zeros_like(dat)
        m = torch.zeros_like(mod)
        for mode in (S.PRTM_ADJ_REFERENCE, S.PRTM_ADJ_EXACT):
            op.set_adjoint(mode)
            for _ in range(3):
                op.lop(False, False, mod, b)
                outs.append(b.cpu().numpy().copy())
                op.lop(True, False, m, dat)
                outs.append(m.cpu().numpy().copy())
        op.close()
    # REF Born continues from the previous call's receiver fields, so only
    # calls in the same position of the sequence agree
    half = len(outs) // 2
    for a, b in zip(outs[:half], outs[half:]):
        np.testing.assert_array_equal(a, b)


def test_graph_replay_counts_its_kernels(cuda):
    # replayed calls count the kernels their graphs hold, as direct ones do
    import swfwi_b200 as S
    torch = cuda
    counts = []
    for graphs in (False, True):
        op, g = _op(torch, "line", S.ARITH_FAST)
        op.set_graphs(graphs)
        mod = t(torch, g["line_mod"])
        b = torch.zeros(g["line_dat"].shape, dtype=torch.float32, device="cuda")
        op.lop(False, False, mod, b)
        torch.cuda.synchronize()
        S.stats_reset()
        for _ in range(3):           # with graphs: captured, then replayed
            op.lop(False, False, mod, b)
        torch.cuda.synchronize()
        counts.append(S.stats_read()["kernel_launches"])
        op.close()
    assert counts[0] == counts[1] and counts[0] > 0, counts
