"""Restatement of the reference's regularisation factor (test infrastructure).

Only tests, the smoke check and the benchmark's CPU legs use this module, as
the checker of the library's CUDA kernels; nothing in the product calls it.
It follows src/unused/ReguFactor.cpp (class ReguFactor):

* getWx2 (:30-47): sum over ix < nx-1, iz < nz of (p[ix+1][iz] - p[ix][iz])^2,
  getWz2 (:49-65): sum over ix < nx, iz < nz-1 of (p[ix][iz+1] - p[ix][iz])^2,
  getReguTerm (:19-27): lx * Wx2 + lz * Wz2.  Each difference and square is
  formed in float as in the reference's loop body; the reference then sums
  in float in loop order, this restatement in float64 (the sums are compared
  within a tolerance, like the objective).
* getReguGradient (:67-108), element by element in float, exactly as the
  loops leave it: the x loop writes 2 lx (p - p[x+1]) at ix = 0 and
  2 lx (2p - p[x+1] - p[x-1]) for 0 < ix < nx-1; the z loop then writes into
  the SAME array, 2 lz (p - p[z+1]) at iz = 0 and 2 lz (2p - p[z+1] - p[z-1])
  for 0 < iz < nz-1, so every element with iz < nz-1 holds its z term; the
  second array stays zero and the final sum adds nothing.
"""
from __future__ import annotations

import numpy as np


def regu_term(p: np.ndarray, lx: float, lz: float) -> float:
    # each difference and its square in float, as the reference's loop body;
    # the sum in float64
    p = np.asarray(p, np.float32)
    rx = (p[1:, :] - p[:-1, :]).astype(np.float32)
    rz = (p[:, 1:] - p[:, :-1]).astype(np.float32)
    wx2 = float((rx * rx).astype(np.float32).astype(np.float64).sum())
    wz2 = float((rz * rz).astype(np.float32).astype(np.float64).sum())
    return float(np.float32(lx)) * wx2 + float(np.float32(lz)) * wz2


def regu_gradient(p: np.ndarray, lx: float, lz: float) -> np.ndarray:
    p = np.asarray(p, np.float32)
    nx, nz = p.shape
    f = np.float32
    two = f(2)
    out = np.zeros_like(p)
    cx, cz = two * f(lx), two * f(lz)
    # x loop (ix < nx-1)
    if nx > 1:
        out[0, :] = cx * (p[0, :] - p[1, :])
        if nx > 2:
            out[1:nx - 1, :] = cx * ((two * p[1:nx - 1, :] - p[2:, :]) - p[:nx - 2, :])
    # z loop (iz < nz-1) overwrites the same array
    if nz > 1:
        out[:, 0] = cz * (p[:, 0] - p[:, 1])
        if nz > 2:
            out[:, 1:nz - 1] = cz * ((two * p[:, 1:nz - 1] - p[:, 2:]) - p[:, :nz - 2])
    return (out + f(0)).astype(np.float32)
