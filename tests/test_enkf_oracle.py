"""The EnKF analysis oracle on the CPU: clipPosition pinned to the
reference's compiled Matrix.cpp, and the cross-product form of the gain that
the GPU path uses checked against the SVD form the reference computes."""
import numpy as np
import pytest

from oracle import enkf_oracle as E


def test_clip_position_matches_compiled_reference(ref):
    rng = np.random.default_rng(0)
    for _ in range(500):
        n = int(rng.integers(2, 70))
        s = np.sort(np.abs(rng.standard_normal(n)) * 10 ** rng.uniform(-3, 3, n))[::-1]
        if rng.random() < 0.3:
            s[int(rng.integers(1, n)):] *= 10 ** rng.uniform(-8, -2)
        assert ref.clip_position(s) == E.clip_position(s)


def test_a_plus_b_matches_compiled_reference(ref):
    rng = np.random.default_rng(1)
    a, b = rng.standard_normal(300), rng.standard_normal(300)
    np.testing.assert_array_equal(ref.a_plus_b(a, b), a + b)


def _case(n=16, rows=3000, seed=2):
    rng = np.random.default_rng(seed)
    base = rng.standard_normal(rows).astype(np.float32)
    hona = (base[None, :] + 0.3 * rng.standard_normal((n, rows))).astype(np.float32)
    dobs = (base + 0.1 * rng.standard_normal(rows)).astype(np.float32)
    z = rng.standard_normal((n, rows))
    return hona, dobs, z


@pytest.mark.parametrize("n", [4, 16, 64])
def test_cross_product_form_equals_svd_form(n):
    hona, dobs, z = _case(n=n)
    t4, sigma, clip = E.gain_matrix(hona, dobs, z, 0.05)
    t4g, clipg = E.gain_matrix_gram(hona, dobs, z, sigma)
    assert clip == clipg
    assert np.linalg.norm(t4g - t4) / np.linalg.norm(t4) < 1e-9


def test_sigma_is_first_float_maximum():
    hap = np.array([[0.5, -2.0000001], [2.0, 0.1]])   # |-2.0000001| and 2.0 tie in float
    assert E.max_abs_hap(hap) == 2.0000001
