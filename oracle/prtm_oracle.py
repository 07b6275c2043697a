"""The oracle (test infrastructure only): an FP64 numpy restatement of
prtm2d_lop of src/unused/prtm2d.cpp (:354-437): the Born branch (:408-434)
with every shot starting from zero fields, its exact transpose, and the
reference's migration branch (:371-407).

The reference's own migration (:371-407) is not the adjoint of its Born
branch; the transpose here is derived step by step from the Born loop and
checked by a dot-product test, so that the GPU's exact-adjoint mode has a
CPU reference.  Small grids only (whole fields per time step in numpy).

Layout as the reference's: fields [nxpad][nzpad], model [nx][nz], data
[ns][ng][nt]; the model sits at [nb, nb + n) in both axes.
"""
from __future__ import annotations

import math

import numpy as np


class PrtmF64:
    """prtm2d_init's set-up (:241-338) in FP64 (the wavelet and the sponge
    taper are computed as the reference computes them, in float)."""

    def __init__(self, vel, dz, dx, dt, amp, fm, nb, nt, ns, ng, sxbeg, szbeg, jsx, jsz, gxbeg, gzbeg, jgx, jgz,
                 csdgather=False):
        vel = np.asarray(vel, np.float32)
        self.nx, self.nz = vel.shape
        self.nb, self.nt, self.ns, self.ng = nb, nt, ns, ng
        nx, nz = self.nx, self.nz
        self.nxpad, self.nzpad = nx + 2 * nb, nz + 2 * nb
        t = np.float32(1.0 / np.float32(dz * dz))
        c11, c12 = 4.0 * float(t) / 3.0, -float(t) / 12.0
        t = np.float32(1.0 / np.float32(dx * dx))
        c21, c22 = 4.0 * float(t) / 3.0, -float(t) / 12.0
        self.c = (-2.0 * (c11 + c12 + c21 + c22), c11, c12, c21, c22)
        vp = np.pad(vel.astype(np.float64), nb, mode="edge")
        self.vv = (vp * dt) ** 2
        w = np.array([math.exp(-(0.015 * (nb - 1 - ib)) ** 2) for ib in range(nb)])
        iz = np.arange(self.nzpad)
        ix = np.arange(self.nxpad)
        ibz = np.minimum(iz, self.nzpad - 1 - iz)
        ibx = np.minimum(ix, self.nxpad - 1 - ix)
        wz = np.where(ibz < nb, w[np.minimum(ibz, nb - 1)], 1.0)
        wx = np.where(ibx < nb, w[np.minimum(ibx, nb - 1)], 1.0)
        self.W = wx[:, None] * wz[None, :]
        self.P = np.zeros((self.nxpad, self.nzpad))
        self.P[2:-2, 2:-2] = 1.0
        tt = np.pi * fm * (np.arange(nt) * dt - 1.0 / fm)
        tt = tt * tt
        self.wlt = amp * (1.0 - 2.0 * tt) * np.exp(-tt)
        distx = sxbeg - gxbeg
        self.src = [(sxbeg + s * jsx + nb, szbeg + s * jsz + nb) for s in range(ns)]
        self.rec = []
        for s in range(ns):
            gx0 = sxbeg + s * jsx - distx if csdgather else gxbeg
            self.rec.append((np.array([gx0 + g * jgx + nb for g in range(ng)]),
                             np.array([gzbeg + g * jgz + nb for g in range(ng)])))

    def _lap(self, u):
        """c0 u + c11 (u[z-1] + u[z+1]) + ... on the whole grid, zero outside"""
        c0, c11, c12, c21, c22 = self.c
        q = np.pad(u, 2)
        return (c0 * u + c11 * (q[2:-2, 1:-3] + q[2:-2, 3:-1]) + c12 * (q[2:-2, :-4] + q[2:-2, 4:])
                + c21 * (q[1:-3, 2:-2] + q[3:-1, 2:-2]) + c22 * (q[:-4, 2:-2] + q[4:, 2:-2]))

    def _step(self, u0, u1, adj):
        """step_forward (:82-120) in place on [2, n-2)"""
        s = self._lap(self.vv * u1) if adj else self.vv * self._lap(u1)
        u0[2:-2, 2:-2] = (2.0 * u1 - u0 + s)[2:-2, 2:-2]

    def _source_fields(self, s):
        """sp0 at the start of every Born time step of shot s"""
        S0 = np.zeros((self.nxpad, self.nzpad))
        S1 = np.zeros_like(S0)
        out = []
        sx, sz = self.src[s]
        for it in range(self.nt):
            out.append(S0.copy())
            S1[sx, sz] += self.wlt[it]
            self._step(S0, S1, False)
            S0 *= self.W
            S1 *= self.W
            S0, S1 = S1, S0
        return out

    def born(self, mod):
        """Born branch (:410-434), every shot from zero receiver fields"""
        nb, nx, nz = self.nb, self.nx, self.nz
        mod = np.asarray(mod, np.float64)
        dat = np.zeros((self.ns, self.ng, self.nt))
        for s in range(self.ns):
            S = self._source_fields(s)
            G0 = np.zeros((self.nxpad, self.nzpad))
            G1 = np.zeros_like(G0)
            rx, rz = self.rec[s]
            for it in range(self.nt):
                G1[nb:nb + nx, nb:nb + nz] += S[it][nb:nb + nx, nb:nb + nz] * mod
                G0, G1 = G1, G0
                G0 *= self.W
                G1 *= self.W
                self._step(G0, G1, True)
                dat[s, :, it] = G1[rx, rz]
        return dat

    def born_transpose(self, dat):
        """The exact transpose of ``born``.  With a^, b^ the adjoints of the
        receiver fields after a step and x = P a^:
          b^ += R' d_it;  a^_prev = W (2 x + V D x + b^);
          b^_prev = W ((1 - P) a^ - x);  mod^ += S_it b^_prev."""
        nb, nx, nz = self.nb, self.nx, self.nz
        dat = np.asarray(dat, np.float64)
        mod = np.zeros((nx, nz))
        for s in range(self.ns):
            S = self._source_fields(s)
            A = np.zeros((self.nxpad, self.nzpad))
            B = np.zeros_like(A)
            rx, rz = self.rec[s]
            for it in range(self.nt - 1, -1, -1):
                np.add.at(B, (rx, rz), dat[s, :, it])
                x = self.P * A
                An = self.W * (2.0 * x + self.vv * self._lap(x) + B)
                B = self.W * ((1.0 - self.P) * A - x)
                mod += (S[it] * B)[nb:nb + nx, nb:nb + nz]
                A = An
        return mod

    def migration(self, dat):
        """The reference's migration branch (:371-407) in FP64: the source
        field forward with its 2-cell ring saved, then reconstructed backwards
        while the receiver field is back-propagated and imaged."""
        nb, nx, nz = self.nb, self.nx, self.nz
        dat = np.asarray(dat, np.float64)
        mod = np.zeros((nx, nz))
        ring = [(slice(nb, nb + nx), slice(nb - 2, nb)), (slice(nb, nb + nx), slice(nb + nz, nb + nz + 2)),
                (slice(nb - 2, nb), slice(nb, nb + nz)), (slice(nb + nx, nb + nx + 2), slice(nb, nb + nz))]
        for s in range(self.ns):
            sx, sz = self.src[s]
            rx, rz = self.rec[s]
            S0 = np.zeros((self.nxpad, self.nzpad))
            S1 = np.zeros_like(S0)
            saved = []
            for it in range(self.nt):
                S1[sx, sz] += self.wlt[it]
                self._step(S0, S1, False)
                S0 *= self.W
                S1 *= self.W
                S0, S1 = S1, S0
                saved.append([S0[r].copy() for r in ring])
            G0 = np.zeros_like(S0)
            G1 = np.zeros_like(S0)
            for it in range(self.nt - 1, -1, -1):
                for r, v in zip(ring, saved[it]):
                    S0[r] = v
                S0, S1 = S1, S0
                self._step(S0, S1, False)
                S1[sx, sz] -= self.wlt[it]
                np.add.at(G1, (rx, rz), dat[s, :, it])
                self._step(G0, G1, False)
                G0 *= self.W
                G1 *= self.W
                G0, G1 = G1, G0
                mod += (S0 * G1)[nb:nb + nx, nb:nb + nz]
        return mod
