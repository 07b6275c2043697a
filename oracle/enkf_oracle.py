"""EnKF analysis oracle: test infrastructure only.

A numpy FP64 restatement of swfwi's serial ensemble Kalman analysis
(src/enfwi), used to check the GPU path.  The reference's EnKF sources need
MPI and Fortran LAPACK/BLAS, which are absent, so they are not compiled:
this file follows them step by step instead, and uses numpy's SVD and
matrix products as the solver (the reference calls LAPACK dgesvd and BLAS
dgemm; neither is pinned to a version, so parity here is against the
restated algorithm).  The observation-perturbation draws (Boost mt19937 +
normal_distribution in the reference) are passed in, so the oracle and the
GPU path consume identical draws; those draws themselves are unpinned.

Only tests/ may import this module.
"""
from __future__ import annotations

import numpy as np


def clip_position(s: np.ndarray) -> int:
    """clipPosition (src/enfwi/Matrix.cpp:170-185): the number of leading
    singular values kept.  relativeError is a float literal held in a double."""
    rel = float(np.float32(0.001))
    n = len(s)
    total = 0.0
    pos = 0
    while pos < n - 1:
        total += abs(float(s[pos]))
        if rel / (1 - rel) * total > (n - pos + 1) * float(s[pos + 1]):
            break
        pos += 1
    return pos + 1


def init_gamma(p: np.ndarray) -> np.ndarray:
    """initGamma (enkfanalyze.cpp:501-521): subtract each data row's mean
    over the members.  p is [N][rows] (member-major, the reference's
    column-major Matrix with one column per member); the row sum runs over
    members in order, in double."""
    n = p.shape[0]
    s = np.zeros(p.shape[1])
    for i in range(n):
        s = s + p[i]
    return p - s / n


def max_abs_hap(hap: np.ndarray) -> float:
    """initPerturbation's std::max_element(..., abs_less<float>)
    (enkfanalyze.cpp:621-635, common.h abs_less): elements compared by the
    float value of |x|, first maximum in column-major (member-major) order;
    the result is the double |x| of that element."""
    flat = hap.reshape(-1)
    key = np.abs(flat.astype(np.float32))
    idx = int(np.argmax(key))          # argmax returns the first maximum
    return abs(float(flat[idx]))


def gain_matrix(hona: np.ndarray, dobs: np.ndarray, z: np.ndarray, sigfac: float,
                sigma: float | None = None):
    """calGainMatrix (enkfanalyze.cpp:185-341), serial.

    hona [N][rows] float32: each member's modelled encoded data (rows in the
    reference's trace-major order); dobs [rows] float32: the encoded observed
    data (every column of D); z [N][rows]: standard-normal draws, the
    perturbation being sigma * z (normal_distribution(0, sigma)); sigma
    None: max|HA'| * sigfac as on the first call.  Returns (t4 as a numpy
    matrix indexed [row, col], sigma, clip)."""
    ha = hona.astype(np.float64)
    d = dobs.astype(np.float64)
    hap = init_gamma(ha)                                   # HA_Perturb
    if sigma is None:
        sigma = max_abs_hap(hap) * float(np.float32(sigfac))   # initPerturbSigma
    pert = sigma * z.astype(np.float64)
    dmat = d[None, :] + pert                               # D + perturbation
    gamma = init_gamma(pert)
    band = hap + gamma                                     # A_plus_B
    # LAPACKE_dgesvd_col_major('S','S', rows, N, band): band as rows x N
    u, s, _ = np.linalg.svd(band.T, full_matrices=False)
    clip = clip_position(s)
    ssqinv = np.zeros((len(s), len(s)))
    for i in range(clip):
        ssqinv[i, i] = (1 / s[i]) * (1 / s[i])
    t0 = (dmat - ha).T                                     # D - HA, rows x N
    t1 = u.T @ t0                                          # U' (D - HA)
    t2 = hap @ u                                           # HA'^T U  (hap is N x rows)
    t3 = t2 @ ssqinv
    t4 = t3 @ t1
    return t4, sigma, clip


def create_a_mean(vels: np.ndarray) -> np.ndarray:
    """createAMean (enkfanalyze.cpp:568-580): float sequential sum over
    members, divided by N in float."""
    s = np.zeros(vels.shape[1], np.float32)
    for j in range(vels.shape[0]):
        s = (s + vels[j]).astype(np.float32)
    return (s / np.float32(vels.shape[0])).astype(np.float32)


def vel_recover(v, dx, dt):
    """velRecover (src/common/common.h:22-25), float."""
    v = np.asarray(v, np.float32)
    dx, dt = np.float32(dx), np.float32(dt)
    t = (dx * dx) / ((dt * dt) * v)
    return np.sqrt(t.astype(np.float32)).astype(np.float32)


def vel_trans(v, dx, dt):
    """velTrans (src/common/common.h:27-30), float."""
    v = np.asarray(v, np.float32)
    dx, dt = np.float32(dx), np.float32(dt)
    return ((dx * dx) / (((dt * dt) * v) * v)).astype(np.float32)


def analyze_update(vels: np.ndarray, t4: np.ndarray, dx: float, dt: float) -> np.ndarray:
    """The update of EnkfAnalyze::analyze (enkfanalyze.cpp:57-111): vels
    [N][model] float32 transformed members -> updated members."""
    mean = create_a_mean(vels)
    ap = vels.astype(np.float64) - mean.astype(np.float64)[None, :]   # initAPerturb, minus<double>
    t5 = ap.T @ t4                                                      # model x N
    out = np.empty_like(vels)
    for i in range(vels.shape[0]):
        phys = vel_recover(vels[i], dx, dt)
        upd = (phys.astype(np.float64) + t5[:, i]).astype(np.float32)   # plus<double> -> float
        out[i] = vel_trans(upd, dx, dt)
    return out


def gain_matrix_gram(hona, dobs, z, sigma):
    """The same gain through the N x N cross products (band^T band
    eigenpairs), the form the GPU path uses; for checking that the two forms
    agree."""
    ha = hona.astype(np.float64)
    hap = init_gamma(ha)
    pert = sigma * z.astype(np.float64)
    band = hap + init_gamma(pert)
    t0 = dobs.astype(np.float64)[None, :] + pert - ha
    x1, x2, x3 = band @ band.T, hap @ band.T, band @ t0.T
    w, v = np.linalg.eigh(x1)
    order = np.argsort(w)[::-1]
    s = np.sqrt(np.maximum(w[order], 0))
    v = v[:, order]
    clip = clip_position(s)
    d = np.zeros(len(s))
    d[:clip] = 1 / s[:clip] ** 4
    return x2 @ v @ np.diag(d) @ v.T @ x3, clip
