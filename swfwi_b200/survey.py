"""Seeded synthetic surveys of the sizes swfwi's FWI workloads run on.

No public dataset is involved: the reference's job flows use a Marmousi
model that is not part of this project.  These generators stand in for it:

* ``layered_model``: six dipping interfaces with seeded depths and dips,
  layer velocities sorted between 1500 and 4700 m/s, plus a uniform random
  field smoothed with a Gaussian of sigma 5 grid points and rescaled to
  +-150 m/s.
* ``smooth``: the initial model, the true model smoothed with sigma 15.
* ``Survey``: grid, time axis, sponge width and an acquisition of regular
  source/receiver lines (the reference's ShotPosition), optionally with
  per-shot receiver spreads of seeded lengths.

Arrays are [nx][nz] float32 with z fastest, as the reference stores them.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


def _gauss_kernel(sigma: float) -> np.ndarray:
    r = max(1, int(np.ceil(4 * sigma)))
    x = np.arange(-r, r + 1, dtype=np.float64)
    k = np.exp(-0.5 * (x / sigma) ** 2)
    return k / k.sum()


def smooth(a: np.ndarray, sigma: float) -> np.ndarray:
    """Separable Gaussian smoothing with edge replication."""
    if sigma <= 0:
        return a.copy()
    k = _gauss_kernel(sigma)
    r = len(k) // 2
    out = np.asarray(a, dtype=np.float64)
    for ax in (0, 1):
        pad = [(0, 0), (0, 0)]
        pad[ax] = (r, r)
        p = np.pad(out, pad, mode="edge")
        acc = np.zeros_like(out)
        for i, w in enumerate(k):
            sl = [slice(None), slice(None)]
            sl[ax] = slice(i, i + out.shape[ax])
            acc += w * p[tuple(sl)]
        out = acc
    return out


def layered_model(nx: int, nz: int, seed: int = 2024, vmin: float = 1500.0, vmax: float = 4700.0,
                  n_interfaces: int = 6, pert: float = 150.0, sigma: float = 5.0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    z = np.arange(nz, dtype=np.float64)[None, :]
    x = np.arange(nx, dtype=np.float64)[:, None]
    depths = np.sort(rng.uniform(0.12, 0.92, n_interfaces)) * nz
    dips = rng.uniform(-0.12, 0.12, n_interfaces) * (nz / max(nx, 1))
    vel = np.sort(rng.uniform(vmin, vmax, n_interfaces + 1))
    vel[0], vel[-1] = vmin + 0.0, vmax - 0.0
    v = np.full((nx, nz), vel[0])
    for k in range(n_interfaces):
        iface = depths[k] + dips[k] * (x - nx / 2.0)
        v = np.where(z >= iface, vel[k + 1], v)
    u = smooth(rng.uniform(-1.0, 1.0, (nx, nz)), sigma)
    u *= pert / max(np.abs(u).max(), 1e-12)
    return np.clip(v + u, vmin, vmax).astype(np.float32)


@dataclass
class Survey:
    """Grid, time axis and acquisition (the reference's Params/ShotPosition)."""
    nz: int
    nx: int
    dx: float
    dt: float
    nt: int
    fm: float
    nb: int
    ns: int
    sxbeg: int
    jsx: int
    ng: int
    gxbeg: int = 0
    jgx: int = 1
    szbeg: int = 6
    jsz: int = 0
    gzbeg: int = 6
    jgz: int = 0
    amp: float = 1.0
    vmin: float = 1500.0
    vmax: float = 4700.0
    maxdv: float = 200.0
    nita: int = 5
    name: str = ""
    # optional per-shot receiver spreads: offsets [ns+1], gx, gz (unpadded)
    spreads: tuple | None = field(default=None, repr=False)

    @property
    def nxpad(self) -> int:
        return self.nx + 2 * self.nb + 12

    @property
    def nzpad(self) -> int:
        return self.nz + self.nb + 12

    @property
    def ngmax(self) -> int:
        if self.spreads is None:
            return self.ng
        off = self.spreads[0]
        return int(np.max(np.diff(off)))

    def src_x(self):
        return self.sxbeg + np.arange(self.ns) * self.jsx

    def scaled(self, **kw) -> "Survey":
        d = dict(self.__dict__)
        d.update(kw)
        return Survey(**d)


def uneven_spreads(s: Survey, seed: int, lo: int = 200, hi: int | None = None):
    """Per-shot receiver spreads of seeded lengths in [lo, hi], centred on
    each source and clipped to the grid (all at depth gzbeg)."""
    hi = s.nx if hi is None else hi
    rng = np.random.default_rng(seed)
    offs = [0]
    gx, gz = [], []
    for sx in s.src_x():
        n = int(rng.integers(lo, hi + 1))
        a = int(sx) - n // 2
        a = min(max(a, 0), s.nx - n)
        xs = np.arange(a, a + n)
        gx.extend(xs.tolist())
        gz.extend([s.gzbeg] * n)
        offs.append(len(gx))
    return (np.asarray(offs, np.int32), np.asarray(gx, np.int32), np.asarray(gz, np.int32))


def config(name: str) -> Survey:
    """The five workload shapes: fwi (plain, 151x461, 20 shots),
    batched (301x921, 96 shots, uneven spreads), encoded (301x921, 96
    shots encoded into one supershot), enkf (201x461, 16 shots per member),
    learned (1000x3000, 120 shots)."""
    if name == "fwi":
        return Survey(name=name, nz=151, nx=461, dx=25.0, dt=0.002, nt=2000, fm=10.0, nb=30,
                      ns=20, sxbeg=11, jsx=23, ng=461)
    if name in ("batched", "encoded"):
        s = Survey(name=name, nz=301, nx=921, dx=10.0, dt=0.001, nt=4000, fm=15.0, nb=30,
                   ns=96, sxbeg=33, jsx=9, ng=921)
        if name == "batched":
            s.spreads = uneven_spreads(s, seed=11)
        return s
    if name == "enkf":
        return Survey(name=name, nz=201, nx=461, dx=20.0, dt=0.002, nt=3000, fm=10.0, nb=30,
                      ns=16, sxbeg=14, jsx=29, ng=461)
    if name == "learned":
        return Survey(name=name, nz=1000, nx=3000, dx=5.0, dt=0.0005, nt=8000, fm=12.0, nb=30,
                      ns=120, sxbeg=12, jsx=25, ng=3000)
    raise KeyError(name)


def small(nz=40, nx=50, nt=200, ns=3, nb=10, dx=25.0, dt=0.002, fm=10.0) -> Survey:
    """A tiny survey the CPU oracle finishes in a second."""
    jsx = max(1, (nx - 2) // ns)
    return Survey(name="small", nz=nz, nx=nx, dx=dx, dt=dt, nt=nt, fm=fm, nb=nb, ns=ns,
                  sxbeg=1 + jsx // 2, jsx=jsx, ng=nx, szbeg=2, gzbeg=2)


def gaussian_random_field(nx: int, nz: int, dx: float, corr_len: float, std: float, seed: int) -> np.ndarray:
    """Seeded Gaussian random field [nx][nz] (float32): white noise smoothed
    with a Gaussian of the correlation length, rescaled to `std` (the
    ensemble members' perturbations of the EnKF workload: 200 m, 100 m/s)."""
    rng = np.random.default_rng(seed)
    f = smooth(rng.standard_normal((nx, nz)), corr_len / dx)
    f = f - f.mean()
    return (f * (std / max(f.std(), 1e-30))).astype(np.float32)
