"""Host-side pieces of the learned-preconditioner workload (no GPU): the
seeded anomaly models, the demo acquisition and the time-to-error rule."""
import numpy as np

from swfwi_b200 import precond as P


def test_anomaly_models_are_seeded_and_in_range():
    a, bg = P.anomaly_model(240, 80, 7)
    b, bg2 = P.anomaly_model(240, 80, 7)
    c, _ = P.anomaly_model(240, 80, 8)
    assert a.dtype == np.float32 and a.shape == (240, 80)
    np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(bg, bg2)
    assert not np.array_equal(a, c)
    # background: a linear depth gradient, the same for every x
    assert np.allclose(bg, bg[:1, :]) and np.all(np.diff(bg[0]) > 0)
    assert 1600 <= bg[0, 0] <= 2000 and 3500 <= bg[0, -1] <= 4300
    # anomalies of at most +-350 m/s each (4-8 of them)
    d = a - bg
    assert np.abs(d).max() > 100 and np.abs(d).max() <= 8 * 350


def test_demo_survey_fits_its_grid():
    s = P.demo_survey()
    xs = s.src_x()
    assert xs.min() >= 0 and xs.max() < s.nx and len(xs) == s.ns
    assert s.ng == s.nx and s.szbeg < s.nz and s.gzbeg < s.nz
    # 25 m cells at 2 ms: Courant number of the fastest model below 0.5
    assert 4700.0 * s.dt / s.dx < 0.5


def test_time_to_error_takes_the_first_crossing():
    hist = [(0.0, 0.013, None, False), (0.2, 0.012, 1.0, True), (0.4, 0.0095, 0.8, True),
            (0.6, 0.0099, 0.7, False), (0.8, 0.009, 0.6, True)]
    assert P.time_to_error(hist, 0.0099) == 0.4
    assert P.time_to_error(hist, 0.013) == 0.0
    assert P.time_to_error(hist, 0.001) is None
