"""The LSRTM operator's oracle (src/unused/prtm2d.cpp): the FP64
restatement's Born branch against the reference's own output (committed
fixture, generated by compiling prtm2d.cpp in place), its exact transpose by
the dot-product test, and the two properties of the reference's operator
that the GPU's REF mode reproduces and its exact-adjoint mode repairs: its
migration is not the adjoint of its Born branch, and its Born branch carries
the receiver fields from one shot (and one call) to the next."""
import numpy as np
import pytest

from oracle.prtm_oracle import PrtmF64
from tests.conftest import golden, rel_l2
from tests.golden.make_golden import PRTM_CASES


def _args(case):
    c = dict(PRTM_CASES[case])
    c.pop("nx")
    c.pop("nz")
    return c


@pytest.mark.parametrize("case", sorted(PRTM_CASES))
def test_f64_born_matches_reference_first_shot(case):
    # the first shot of the reference's first Born call starts from zero
    # fields, as every shot of the restatement does
    g = golden("prtm")
    o = PrtmF64(g[case + "_vel"], **_args(case))
    d = o.born(g[case + "_mod"])
    assert rel_l2(d[0], g[case + "_born1"][0]) < 1e-5


@pytest.mark.parametrize("csd", [0, 1])
def test_f64_transpose_passes_dot_product(csd):
    rng = np.random.default_rng(5 + csd)
    vel = rng.uniform(1500, 3000, (30, 22)).astype(np.float32)
    o = PrtmF64(vel, dz=9.0, dx=11.0, dt=1e-3, amp=1.0, fm=22.0, nb=6, nt=90, ns=2, ng=7, sxbeg=4, szbeg=1,
                jsx=9, jsz=1, gxbeg=1, gzbeg=2, jgx=3, jgz=1, csdgather=bool(csd))
    m = rng.standard_normal((30, 22))
    d = rng.standard_normal((2, 7, 90))
    a = np.vdot(o.born(m), d)
    b = np.vdot(m, o.born_transpose(d))
    assert abs(a - b) <= 1e-11 * abs(a)


@pytest.mark.parametrize("case", sorted(PRTM_CASES))
def test_reference_migration_is_not_the_adjoint(case):
    # <L m, d> against <m, L' d> with the reference's own pair (one call
    # each from zero fields, which is linear in m): off by order one
    g = golden("prtm")
    a = np.vdot(g[case + "_born1"].astype(np.float64), g[case + "_dat"])
    b = np.vdot(g[case + "_mod"].astype(np.float64), g[case + "_mig"])
    assert abs(a - b) > 0.3 * max(abs(a), abs(b))


@pytest.mark.parametrize("case", sorted(PRTM_CASES))
def test_reference_born_carries_receiver_fields(case):
    g = golden("prtm")
    o = PrtmF64(g[case + "_vel"], **_args(case))
    d = o.born(g[case + "_mod"])
    # later shots differ from their zero-start Born data; a second call
    # differs from the first
    assert rel_l2(d[1], g[case + "_born1"][1]) > 0.05
    assert rel_l2(g[case + "_born2"], g[case + "_born1"]) > 0.05


@pytest.mark.parametrize("case", sorted(PRTM_CASES))
def test_f64_migration_matches_reference(case):
    # the reference's float reconstruction drifts from FP64 on the
    # thin-sponge gather case (6.4e-3); on the line case it is 2.4e-6
    g = golden("prtm")
    o = PrtmF64(g[case + "_vel"], **_args(case))
    assert rel_l2(g[case + "_mig"], o.migration(g[case + "_dat"])) < (1e-2 if case == "gather" else 1e-5)
