"""Host-side pieces of the EnFWI driver on the CPU: the velocity transforms
and the slowness norms in the reference's float order."""
import numpy as np

from oracle import enkf_oracle as E
from swfwi_b200 import enfwi


def test_velocity_transforms_match_oracle():
    rng = np.random.default_rng(0)
    v = rng.uniform(1500, 4700, 1000).astype(np.float32)
    t = enfwi.vel_trans(v, 20.0, 0.002)
    np.testing.assert_array_equal(t, E.vel_trans(v, 20.0, 0.002))
    np.testing.assert_array_equal(enfwi.vel_recover(t, 20.0, 0.002), E.vel_recover(t, 20.0, 0.002))


def test_slowness_norms_loop_order():
    # slownessL1L2Norm written out as the reference's double loop
    rng = np.random.default_rng(1)
    nx, nz, nb, dx, dt = 30, 20, 4, 20.0, 0.002
    pad = (nx + 2 * nb + 12) * (nz + nb + 12)
    acc = enfwi.vel_trans(rng.uniform(2000, 3000, pad), dx, dt)
    cur = enfwi.vel_trans(rng.uniform(2000, 3000, pad), dx, dt)
    a = enfwi.vel_recover(acc[: nx * nz], dx, dt)
    c = enfwi.vel_recover(cur[: nx * nz], dx, dt)
    n1 = n2 = s1 = s2 = np.float32(0)
    for ix in range(nb, nx - nb):
        for iz in range(0, nz - nb):
            o = ix * nz + iz
            av, cv = np.float32(1) / a[o], np.float32(1) / c[o]
            d = np.float32(abs(av - cv))
            n2 = np.float32(n2 + d * d)
            s2 = np.float32(s2 + av * av)
            n1 = np.float32(n1 + d)
            s1 = np.float32(s1 + av)
    l1, l2 = enfwi.slowness_l1l2(acc, cur, nx, nz, nb, dx, dt)
    assert l1 == float(n1 / s1) and l2 == float(n2 / s2)
