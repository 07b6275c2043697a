"""The oracle pinned against the golden fixtures (no GPU)."""
import numpy as np
import pytest

from tests.conftest import golden, rel_l2
from tests.golden.make_golden import pthread_inputs, sha, small_survey, wrap_inputs


def test_reference_reproduces_wrap_case(ref):
    # src/test/fd/wrap.cpp: one damped call, 533 x 193, nb = 36
    g = golden("wrap_533x193")
    prev, curr, vel, nb = wrap_inputs()
    ref.step(prev, curr, vel, nb)
    assert sha(prev) == str(g["sha256"])


def test_restatement_reproduces_wrap_case(fdo):
    g = golden("wrap_533x193")
    prev, curr, vel, nb = wrap_inputs()
    fdo.step_ref(prev, curr, vel, nb, damped=True)
    assert sha(prev) == str(g["sha256"])
    np.testing.assert_array_equal(prev.ravel()[::101], g["sub"])


def test_restatement_reproduces_pthread_case(fdo):
    # src/test/pthread-sim-fd/fd4t10s-zjh.cpp: 20 x 20, two undamped steps;
    # the reference compares sums, this compares every element
    g = golden("pthread_20x20")
    p0, p1, vel = pthread_inputs()
    for k in range(2):
        fdo.step_ref(p0, p1, vel, 1, damped=False)
        np.testing.assert_array_equal(p0, g["p0_steps"][k])
        p0, p1 = p1, p0


@pytest.mark.parametrize("nx,nz,nb", [(40, 30, 12), (97, 61, 20), (64, 200, 36)])
@pytest.mark.parametrize("damped", [True, False])
def test_restatement_bit_exact_random(ref, fdo, nx, nz, nb, damped):
    rng = np.random.default_rng(nx * 1000 + nz)
    curr = rng.standard_normal((nx, nz)).astype(np.float32)
    prev = rng.standard_normal((nx, nz)).astype(np.float32)
    vt = rng.uniform(5.0, 60.0, (nx, nz)).astype(np.float32)
    a, b = prev.copy(), prev.copy()
    ref.step(a, curr, vt, nb if damped else None)
    fdo.step_ref(b, curr, vt, nb, damped)
    np.testing.assert_array_equal(a.view(np.int32), b.view(np.int32))


def test_reference_reproduces_small_survey(ref):
    g = golden("small_survey")
    s, vtrue, vinit = small_survey()
    M = ref.model(s)
    np.testing.assert_array_equal(M.expand_domain(vtrue), g["exvel_true"])
    np.testing.assert_array_equal(M.expand_domain(vinit), g["exvel_init"])
    wlt = ref.ricker(s.nt, s.fm, s.dt)
    np.testing.assert_array_equal(wlt, g["wlt"])
    np.testing.assert_array_equal(M.fwi_forward(wlt, 1), g["dcal"][1])
    np.testing.assert_array_equal(M.calgradient_fwi(wlt, g["vsrc"], 1), g["grad_shot1"])


def test_parabola_known_answer(ref):
    g = golden("parabola")
    xv, yv = ref.parabola_vertex(*[float(x) for x in g["inputs"]])
    assert np.float32(xv) == g["xv"] and np.float32(yv) == g["yv"]
    # the vertex lies between the trial steps for this convex triple
    assert 0 < xv < float(g["inputs"][4])


def test_f64_oracle_forward_close(fdo):
    # FP64 restatement vs the reference's FP32 seismogram on the small survey
    g = golden("small_survey")
    s, _, _ = small_survey()
    bx0 = s.nb + 6
    nzpad = s.nz + s.nb + 12
    src = (s.sxbeg + 1 * s.jsx + bx0) * nzpad + s.szbeg + 6
    rec = (np.arange(s.ng) + bx0) * nzpad + s.gzbeg + 6
    d64 = fdo.forward_f64(g["exvel_init"].astype(np.float64), bx0, s.nt, g["wlt"].astype(np.float64), src, rec)
    err = rel_l2(g["dcal"][1], d64)
    assert err < 1e-5, err


def test_f64_oracle_gradient_close(fdo):
    g = golden("small_survey")
    s, _, _ = small_survey()
    bx0 = s.nb + 6
    nzpad = s.nz + s.nb + 12
    src = (s.sxbeg + 1 * s.jsx + bx0) * nzpad + s.szbeg + 6
    rec = (np.arange(s.ng) + bx0) * nzpad + s.gzbeg + 6
    g64 = fdo.gradient_f64(g["exvel_init"].astype(np.float64), bx0, s.nt, s.dt, g["wlt"].astype(np.float64),
                           src, rec, g["vsrc"].astype(np.float64))
    err = rel_l2(g["grad_shot1"], g64)
    assert err < 1e-4, err
