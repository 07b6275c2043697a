"""Batched shot generation: the reference's fm-damp tool
(src/tool/main-fm-damp.cpp:202-282) on the GPU.

Reads a velocity RSF (n1 = nz, n2 = nx, d2 = dx), models every shot of a
regular source line with a Ricker wavelet of amplitude `amp` (addSource ->
stepForward -> swap -> recordSeis per step, one batch over all shots) and
writes the shots RSF (n1 = nt, n2 = ng, n3 = ns, on disk [is][ig][it]) with
the header keys main-fm-damp.cpp:144-173 writes.

    python -m swfwi_b200.fm_damp vinit=vel.rsf shots=shots.rsf dt=0.001 nt=4000 \
        ns=96 ng=921 jsx=9 sxbeg=30 szbeg=0 gxbeg=0 gzbeg=0 fm=15 amp=1 nb=30
"""
from __future__ import annotations

import sys

import numpy as np

from . import ARITH_REF, Damp4t10d, ShotPosition, ricker_wavelet, rsf


def fm_damp(vinit: str, shots: str, *, dt: float, nt: int, ns: int, ng: int, jsx: int, sxbeg: int,
            szbeg: int, gxbeg: int, gzbeg: int, amp: float = 1000.0, fm: float = 10.0, nb: int = 30,
            jsz: int = 0, jgx: int = 1, jgz: int = 0, arith: int = ARITH_REF) -> np.ndarray:
    """Models all shots; writes them to `shots` and returns dobs [ns][nt][ng]."""
    import torch
    vel = rsf.read(vinit)                                   # [nx][nz]
    nx, nz = vel.shape
    dx = float(rsf.dims(vinit)[1][1])
    # Params::check (main-fm-damp.cpp:147-160)
    if not (sxbeg >= 0 and szbeg >= 0 and sxbeg + (ns - 1) * jsx < nx and szbeg + (ns - 1) * jsz < nz):
        raise ValueError("sources exceed the computing zone")
    if not (gxbeg >= 0 and gzbeg >= 0 and gxbeg + (ng - 1) * jgx < nx and gzbeg + (ng - 1) * jgz < nz):
        raise ValueError("geophones exceed the computing zone")
    m = Damp4t10d(ShotPosition(szbeg, sxbeg, jsz, jsx, ns, nz), ShotPosition(gzbeg, gxbeg, jgz, jgx, ng, nz),
                  dt, dx, fm, nb, nt, arith=arith)
    exvel = torch.from_numpy(m.expandDomain(vel)).cuda()
    m.bindVelocity(exvel)
    wlt = torch.from_numpy(ricker_wavelet(nt, fm, dt, amp)).cuda()
    dobs = torch.zeros((ns, nt, ng), dtype=torch.float32, device="cuda")
    m.forward_batch(wlt, dobs, np.arange(ns, dtype=np.int32))
    out = dobs.cpu().numpy()
    extra = {"amp": amp, "fm": fm, "ng": ng, "szbeg": szbeg, "sxbeg": sxbeg, "gzbeg": gzbeg, "gxbeg": gxbeg,
             "jsx": jsx, "jsz": jsz, "jgx": jgx, "jgz": jgz, "nb": nb,
             "vmin": float(vel.min()), "vmax": float(vel.max())}
    rsf.write_shots(shots, out, dt, jgx * dx, extra)
    return out


def main(argv: list[str]) -> int:
    kv = dict(a.split("=", 1) for a in argv if "=" in a)
    ints = ("nt", "ns", "ng", "jsx", "sxbeg", "szbeg", "gxbeg", "gzbeg", "nb", "jsz", "jgx", "jgz")
    floats = ("dt", "amp", "fm")
    args = {k: int(v) for k, v in kv.items() if k in ints}
    args.update({k: float(v) for k, v in kv.items() if k in floats})
    fm_damp(kv["vinit"], kv["shots"], **args)
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv[1:]))
