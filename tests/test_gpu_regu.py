"""The regularisation factor of the reference's regularised ESS-FWI
(src/unused/ReguFactor.cpp, EssFwiRegu in src/unused/essfwiregu.cpp) on the
GPU: gradient bit for bit against the reference's own code (fixture), the
term within 1e-4 relative of the reference's float sum and 1e-9 of the FP64
restatement, and the regularised epoch's objective bookkeeping."""
import numpy as np
import pytest

from tests.conftest import golden
from tests.gpu_helpers import t

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", ["small", "ragged"])
def test_regu_kernels_match_reference(cuda, case):
    import swfwi_b200 as S
    from oracle.regu_oracle import regu_term
    torch = cuda
    g = golden("regu")
    v = golden("small_survey")["exvel_init"] if case == "small" else g["ragged"]
    lx, lz = float(g["lx_" + case]), float(g["lz_" + case])
    vd = t(torch, v)
    grad = torch.zeros_like(vd)
    S.regu_gradient(vd, lx, lz, grad)
    np.testing.assert_array_equal(grad.cpu().numpy(), g["grad_" + case])
    term = S.regu_term(vd, lx, lz)
    ref = float(g["term_" + case])
    assert abs(term - ref) <= 1e-4 * ref, (term, ref)
    assert abs(term - regu_term(v, lx, lz)) <= 1e-9 * ref


def test_regu_gradient_accumulates(cuda):
    import swfwi_b200 as S
    torch = cuda
    g = golden("regu")
    v = golden("small_survey")["exvel_init"]
    rng = np.random.default_rng(4)
    g0 = rng.standard_normal(v.shape).astype(np.float32)
    acc = t(torch, g0).clone()
    S.regu_gradient(t(torch, v), 0.3, 0.7, acc, accumulate=True)
    np.testing.assert_array_equal(acc.cpu().numpy(), (g0 + g["grad_small"]).astype(np.float32))


def test_regularised_epoch_objective(cuda):
    import swfwi_b200 as S
    from tests.golden.make_golden import small_survey
    torch = cuda
    g = golden("small_survey")
    s, _, _ = small_survey()
    res = {}
    for lam in (0.0, 0.05):
        m = S.Damp4t10d.from_survey(s)
        fw = S.EssFwiFramework(m, g["exvel_init"], 1500.0, 4700.0, s.nita, s.maxdv, g["wlt"], g["dobs"])
        fw.setRegularization(lam, lam)
        fw.epoch(0)
        fw.epoch(1)
        res[lam] = (fw.getInitObj(), fw.getUpdateObj(), fw.velocity())
        del fw
    term = S.regu_term(t(torch, g["exvel_init"]), 0.05, 0.05)
    # obj1 = data misfit + float(term) (essfwiregu.cpp:716-720)
    assert abs((res[0.05][0] - res[0.0][0]) - term) <= 1e-5 * res[0.05][0]
    assert np.isfinite(res[0.05][1]) and res[0.05][1] < res[0.05][0]
    assert not np.array_equal(res[0.05][2], res[0.0][2])
    plain = S.FwiFramework(S.Damp4t10d.from_survey(s), g["exvel_init"], 1500.0, 4700.0, s.nita, s.maxdv,
                           g["wlt"], g["dobs"])
    with pytest.raises(S.SwfwiError):      # plain FWI has no regularised epoch
        S._check(S.lib().swfwi_fwi_set_regularization(plain.h, 0.1, 0.1))
