"""Whole FWI epochs (plain and encoded) on the GPU against the reference."""
import numpy as np
import pytest

from tests.conftest import golden, rel_l2
from tests.golden.make_golden import small_survey

pytestmark = pytest.mark.gpu


def _run(cls, niter):
    import swfwi_b200 as S
    g = golden("small_survey")
    s, _, _ = small_survey()
    m = S.Damp4t10d.from_survey(s)
    fw = cls(m, g["exvel_init"], 1500.0, 4700.0, s.nita, s.maxdv, g["wlt"], g["dobs"])
    objs = []
    for it in range(niter):
        fw.epoch(it)
        objs.append((fw.getInitObj(), fw.getUpdateObj()))
    return fw, np.array(objs)


def test_plain_fwi_epochs_match_reference(cuda):
    import swfwi_b200 as S
    e = golden("small_epochs")
    fw, objs = _run(S.FwiFramework, 2)
    v = fw.velocity()
    # FP64 objective sums move the step length by float rounding only
    assert rel_l2(v, e["fwi_vel"]) < 1e-5, rel_l2(v, e["fwi_vel"])
    np.testing.assert_allclose(objs[0, 0], e["fwi_objs"][0, 0], rtol=1e-5)
    np.testing.assert_allclose(objs[:, 1], e["fwi_objs"][:, 2], rtol=1e-3)
    a, o = fw.lastLineSearch()
    np.testing.assert_allclose(a[3], e["fwi_objs"][1, 1], rtol=1e-3)


def test_ess_fwi_epochs_match_reference(cuda):
    import swfwi_b200 as S
    e = golden("small_epochs")
    fw, objs = _run(S.EssFwiFramework, 2)
    v = fw.velocity()
    assert rel_l2(v, e["ess_vel"]) < 1e-5, rel_l2(v, e["ess_vel"])
    np.testing.assert_allclose(objs, e["ess_objs"], rtol=1e-4)
