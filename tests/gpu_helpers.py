"""Helpers for the GPU tests: a propagator on the small golden survey."""
import numpy as np

from tests.conftest import golden
from tests.golden.make_golden import small_survey


def small_method(torch, arith=0):
    import swfwi_b200 as S
    g = golden("small_survey")
    s, _, _ = small_survey()
    m = S.Damp4t10d.from_survey(s, arith=arith)
    vel = torch.from_numpy(g["exvel_init"]).cuda()
    m.bindVelocity(vel)
    return s, m, g, vel


def t(torch, a, dtype=None):
    a = np.ascontiguousarray(a)
    x = torch.from_numpy(a).cuda()
    return x if dtype is None else x.to(dtype)
