"""Generates the golden fixtures in this folder by running the reference's
own CPU code (swfwi sources compiled in place by ``oracle/Makefile`` into
``oracle/_ref``).  Run where the reference tree exists:

    make -C oracle && python tests/golden/make_golden.py

The reference ships no stored outputs; its only checks are the cases
reproduced here:
  * src/test/fd/wrap.cpp:19-46 - one damped call on a 533 x 193 grid,
    nb = 36, vel = 1500, curr = rand()/RAND_MAX (glibc rand, seed 1);
  * src/test/pthread-sim-fd/fd4t10s-zjh.cpp:394-444 - a 20 x 20 grid,
    p0 then p1 filled with rand() % 10, vel = 1500, two undamped steps with
    a swap (the reference compares per-step sums; we keep the fields);
  * src/tool/main-test.cpp:37-60 - the parabolaVertex triple.
Plus small end-to-end cases on a seeded 50 x 40 survey: forward modelling,
direct-arrival mute, the time derivative, per-shot and encoded gradients,
the per-shot gradient loop, and two epochs of plain and encoded FWI; the
regularisation factor (``--regu``) and the LSRTM operator (``--prtm``,
src/unused/prtm2d.cpp) on seeded inputs.
"""
from __future__ import annotations

import ctypes
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from swfwi_b200 import survey as sv  # noqa: E402


def libc_rand_seq(n: int) -> np.ndarray:
    """glibc rand() from its default seed (1), as the reference's tests draw."""
    libc = ctypes.CDLL("libc.so.6")
    libc.srand(1)
    return np.array([libc.rand() for _ in range(n)], dtype=np.int64)


RAND_MAX = 2147483647


def wrap_inputs():
    nx, nz, nb = 533, 193, 36
    r = libc_rand_seq(nx * nz)
    curr = (r * 1.0 / RAND_MAX).astype(np.float32).reshape(nx, nz)
    prev = np.zeros((nx, nz), np.float32)
    vel = np.full((nx, nz), 1500.0, np.float32)
    return prev, curr, vel, nb


def pthread_inputs():
    nx = nz = 20
    r = libc_rand_seq(2 * nx * nz)
    p0 = (r[: nx * nz] % 10).astype(np.float32).reshape(nx, nz)
    p1 = (r[nx * nz:] % 10).astype(np.float32).reshape(nx, nz)
    vel = np.full((nx, nz), 1500.0, np.float32)
    return p0, p1, vel


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def small_survey():
    s = sv.small()
    vtrue = sv.layered_model(s.nx, s.nz, seed=7)
    vinit = sv.smooth(vtrue, 3.0).astype(np.float32)
    return s, vtrue, vinit


def main():
    R = oracle.RefLib()
    out = {}

    prev, curr, vel, nb = wrap_inputs()
    R.step(prev, curr, vel, nb)
    np.savez_compressed(os.path.join(HERE, "wrap_533x193.npz"), sha256=sha(prev), sub=prev.ravel()[::101],
                        sum=np.float32(np.add.accumulate(prev.ravel(), dtype=np.float32)[-1]))

    p0, p1, vel = pthread_inputs()
    steps = []
    for _ in range(2):
        R.step(p0, p1, vel, None)
        steps.append(p0.copy())
        p0, p1 = p1, p0
    np.savez_compressed(os.path.join(HERE, "pthread_20x20.npz"), p0_steps=np.stack(steps))

    tri = (0.0, 6.84734e+06, 6.17151e-05, 5.49986e+06, 0.00012343, 5.26678e+06, 0.00012343)
    xv, yv = R.parabola_vertex(*tri)
    np.savez_compressed(os.path.join(HERE, "parabola.npz"), inputs=np.array(tri, np.float32),
                        xv=np.float32(xv), yv=np.float32(yv))

    codes = {f"seed{seed}": np.stack([R.random_codes(seed, 96, skip=k) for k in range(3)])
             for seed in (1, 2)}
    wl = {f"{name}": R.ricker(c.nt, c.fm, c.dt, 1.0)
          for name, c in (("fwi", sv.config("fwi")), ("batched", sv.config("batched")))}
    np.savez_compressed(os.path.join(HERE, "codes_ricker.npz"), **codes, **wl)

    s, vtrue, vinit = small_survey()
    M = R.model(s)
    ext = M.expand_domain(vtrue)
    exi = M.expand_domain(vinit)
    wlt = R.ricker(s.nt, s.fm, s.dt, 1.0)
    M.bind_velocity(ext)
    dobs = np.stack([M.fwi_forward(wlt, i) for i in range(s.ns)])
    M.bind_velocity(exi)
    dcal = np.stack([M.fwi_forward(wlt, i) for i in range(s.ns)])
    muted = np.stack([M.remove_direct_arrival(dcal[i], i) for i in range(s.ns)])
    muted_ess = M.remove_direct_arrival(dcal[0], -1)
    res = (muted[1] - M.remove_direct_arrival(dobs[1], 1)).astype(np.float32)
    vsrc = R.trans_vsrc(res)
    g1 = M.calgradient_fwi(wlt, vsrc, 1)
    g1s = M.mask_gradient(M.scale_gradient(g1))
    g2, obj = M.fwi_gradient(wlt, dobs)
    ecodes = R.random_codes(1, s.ns)
    encsrc = (wlt[:, None] * ecodes[None, :].astype(np.float32)).astype(np.float32)
    ess_dcal = M.ess_forward(encsrc)
    gess = M.calgradient_ess(encsrc, vsrc)
    bndr = M.write_bndry(dcal_field := np.arange(M.nxpad * M.nzpad, dtype=np.float32).reshape(M.nxpad, M.nzpad))
    np.savez_compressed(os.path.join(HERE, "small_survey.npz"), vtrue=vtrue, vinit=vinit, exvel_true=ext,
                        exvel_init=exi, wlt=wlt, dobs=dobs, dcal=dcal, muted=muted, muted_ess=muted_ess,
                        res=res, vsrc=vsrc, grad_shot1=g1, grad_shot1_scaled=g1s, grad_sum=g2,
                        obj=np.float32(obj), ess_codes=ecodes, ess_dcal=ess_dcal, grad_ess=gess, bndr=bndr)

    # two epochs of each framework from the initial model
    M2 = R.model(s)
    M2.expand_domain(vinit)
    vf, objs_f = M2.fwi_run(wlt, dobs, 2, s.nita, s.maxdv, 1500.0, 4700.0)
    M3 = R.model(s)
    M3.expand_domain(vinit)
    ve, objs_e = M3.ess_fwi_run(wlt, dobs, 2, s.nita, s.maxdv, 1500.0, 4700.0)
    np.savez_compressed(os.path.join(HERE, "small_epochs.npz"), fwi_vel=vf, fwi_objs=objs_f, ess_vel=ve,
                        ess_objs=objs_e)
    regu_fixture(R)
    print("fixtures written to", HERE)


def regu_fixture(R=None):
    """ReguFactor (src/unused/ReguFactor.cpp) on the small survey's padded
    initial model and on a seeded ragged grid: term and gradient."""
    R = R or oracle.RefLib()
    g = np.load(os.path.join(HERE, "small_survey.npz"))
    v = g["exvel_init"]
    t1, g1 = R.regu(v, 0.3, 0.7)
    rng = np.random.default_rng(17)
    w = rng.uniform(0.2, 3.0, (13, 7)).astype(np.float32)
    t2, g2 = R.regu(w, 1.5, 0.25)
    np.savez_compressed(os.path.join(HERE, "regu.npz"), term_small=np.float32(t1), grad_small=g1,
                        lx_small=np.float32(0.3), lz_small=np.float32(0.7), ragged=w, term_ragged=np.float32(t2),
                        grad_ragged=g2, lx_ragged=np.float32(1.5), lz_ragged=np.float32(0.25))


PRTM_CASES = {
    # one line of surface shots, receivers every other cell
    "line": dict(nx=48, nz=36, dz=10.0, dx=10.0, dt=1e-3, amp=1.0, fm=20.0, nb=10, nt=160, ns=3, ng=23,
                 sxbeg=6, szbeg=2, jsx=16, jsz=0, gxbeg=2, gzbeg=1, jgx=2, jgz=0, csdgather=0),
    # common-shot gathers along a slanted shot line, all receivers of a shot
    # in one cell, the thinnest sponge the scheme allows
    "gather": dict(nx=33, nz=29, dz=8.0, dx=12.0, dt=8e-4, amp=2.0, fm=25.0, nb=2, nt=120, ns=2, ng=5,
                   sxbeg=20, szbeg=3, jsx=4, jsz=2, gxbeg=10, gzbeg=24, jgx=0, jgz=0, csdgather=1),
}


def prtm_fixture():
    """The reference's LSRTM operator (src/unused/prtm2d.cpp, compiled in
    place) on seeded inputs: two Born calls on one operator (the second
    continues from the receiver fields the first left), the migration of
    seeded data, and the migration added onto a seeded model."""
    out = {}
    for name, c in PRTM_CASES.items():
        rng = np.random.default_rng(sum(map(ord, name)))
        nx, nz = c["nx"], c["nz"]
        vel = rng.uniform(1800.0, 2600.0, (nx, nz)).astype(np.float32)
        mod = rng.standard_normal((nx, nz)).astype(np.float32)
        dat = rng.standard_normal((c["ns"], c["ng"], c["nt"])).astype(np.float32)
        base = rng.standard_normal((nx, nz)).astype(np.float32)
        kw = {k: v for k, v in c.items() if k not in ("nx", "nz")}
        op = oracle.PrtmRef(vel, **kw)
        b1 = np.zeros_like(dat)
        op.lop(0, 0, mod, b1)
        b2 = np.zeros_like(dat)
        op.lop(0, 0, mod, b2)
        m1 = np.zeros_like(mod)
        op.lop(1, 0, m1, dat)
        m2 = base.copy()
        op.lop(1, 1, m2, dat)
        op.close()
        out.update({f"{name}_vel": vel, f"{name}_mod": mod, f"{name}_dat": dat, f"{name}_base": base,
                    f"{name}_born1": b1, f"{name}_born2": b2, f"{name}_mig": m1, f"{name}_mig_add": m2})
    np.savez_compressed(os.path.join(HERE, "prtm.npz"), **out)


if __name__ == "__main__":
    import sys
    if "--regu" in sys.argv:
        regu_fixture()
    elif "--prtm" in sys.argv:
        prtm_fixture()
    else:
        main()
