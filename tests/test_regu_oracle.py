"""The regularisation factor's restatement (oracle/regu_oracle.py) against
the reference's own ReguFactor (src/unused/ReguFactor.cpp) through the
committed fixture, and against the compiled reference where it is built.
The gradient matches bit for bit; the term within 1e-4 relative (the
reference sums in float in loop order, the restatement in float64)."""
import numpy as np
import pytest

from oracle.regu_oracle import regu_gradient, regu_term
from tests.conftest import golden


def test_restatement_matches_fixture():
    g = golden("regu")
    s = golden("small_survey")
    v = s["exvel_init"]
    np.testing.assert_array_equal(regu_gradient(v, g["lx_small"], g["lz_small"]), g["grad_small"])
    assert abs(regu_term(v, g["lx_small"], g["lz_small"]) - float(g["term_small"])) <= 1e-4 * float(g["term_small"])
    w = g["ragged"]
    np.testing.assert_array_equal(regu_gradient(w, g["lx_ragged"], g["lz_ragged"]), g["grad_ragged"])
    assert abs(regu_term(w, g["lx_ragged"], g["lz_ragged"]) - float(g["term_ragged"])) <= 1e-4 * float(g["term_ragged"])


def test_gradient_keeps_the_reference_overwrite():
    # the reference's z loop writes into the x-term array: every element
    # above the last depth holds its z term only; the last depth holds the
    # x term (or 0 on the last row)
    rng = np.random.default_rng(3)
    p = rng.uniform(1, 2, (6, 5)).astype(np.float32)
    g = regu_gradient(p, 0.5, 0.0)
    assert np.all(g[:, :-1] == 0)
    assert np.all(g[:-1, -1] != 0) and g[-1, -1] == 0


@pytest.mark.parametrize("shape", [(1, 4), (4, 1), (2, 3), (9, 17)])
def test_restatement_matches_compiled_reference(ref, shape):
    rng = np.random.default_rng(shape[0] * 100 + shape[1])
    v = rng.uniform(0.5, 2.0, shape).astype(np.float32)
    t, g = ref.regu(v, 0.4, 1.3)
    np.testing.assert_array_equal(regu_gradient(v, 0.4, 1.3), g)
    assert abs(regu_term(v, 0.4, 1.3) - t) <= 1e-4 * max(abs(t), 1e-30)
