"""Ensemble-Kalman FWI: the reference's enfwi-damp driver
(src/tool/main-enfwi-damp.cpp:406-631) on the GPU.

N velocity members, each the initial model plus a perturbation
(createVelDB, main-enfwi-damp.cpp:180-205: v = velTrans(velRecover(v0) +
p)), each with its own encoded-source FWI (EssFwiFramework).  An EnKF
analysis of the encoded observed data (EnkfAnalyze::pAnalyze) moves all
members at the start and every `niterenkf` iterations; after every
iteration the members' mean model is scored with the encoded objective of
calobj (main-enfwi-damp.cpp:262-283: seed-1 codes, direct arrival muted
from both data).  Per-member data misfit and slowness L1/L2 norms against a
true model are logged at each analysis (slownessL1L2Norm,
main-enfwi-damp.cpp:368-402, including its use of the unpadded sizes to
walk the padded arrays).
"""
from __future__ import annotations

import numpy as np

from . import (ARITH_FAST, Damp4t10d, EnkfAnalyze, EssFwiFramework, cal_objective, encode_obs,
               encode_source, random_codes)

ENKF_SEED = 2      # EnkfAnalyze::ENKF_SEED (enkfanalyze.h:44)
CALOBJ_SEED = 1    # calobj's RandomCodes(1)


def vel_recover(v, dx, dt):
    """velRecover (src/common/common.h:22-25) in float."""
    v = np.asarray(v, np.float32)
    dx, dt = np.float32(dx), np.float32(dt)
    return np.sqrt(((dx * dx) / ((dt * dt) * v)).astype(np.float32)).astype(np.float32)


def vel_trans(v, dx, dt):
    """velTrans (src/common/common.h:27-30) in float."""
    v = np.asarray(v, np.float32)
    dx, dt = np.float32(dx), np.float32(dt)
    return ((dx * dx) / (((dt * dt) * v) * v)).astype(np.float32)


def slowness_l1l2(accurate, curr, nx: int, nz: int, nb: int, dx: float, dt: float):
    """slownessL1L2Norm: accurate/curr are the padded transformed models;
    the reference takes their first nx*nz values with the unpadded sizes as
    strides; float sums in loop order."""
    a = vel_recover(np.ravel(accurate)[: nx * nz], dx, dt).reshape(nx, nz)
    c = vel_recover(np.ravel(curr)[: nx * nz], dx, dt).reshape(nx, nz)
    sa = (np.float32(1.0) / a[nb:nx - nb, : nz - nb]).astype(np.float32).ravel()
    sc = (np.float32(1.0) / c[nb:nx - nb, : nz - nb]).astype(np.float32).ravel()
    d = np.abs((sa - sc).astype(np.float32))
    norm1 = np.cumsum(d, dtype=np.float32)[-1]
    norm2 = np.cumsum((d * d).astype(np.float32), dtype=np.float32)[-1]
    s1 = np.cumsum(sa, dtype=np.float32)[-1]
    s2 = np.cumsum((sa * sa).astype(np.float32), dtype=np.float32)[-1]
    return float(norm1 / s1), float(norm2 / s2)


class EnFwi:
    """survey: the acquisition (swfwi_b200.survey.Survey); exvel: the padded
    transformed initial model; perturbations [N][nxpad][nzpad] in m/s;
    wlt [nt] and dobs [ns][nt][ng] host float32; exvel_true (optional): the
    padded transformed true model for the slowness norms."""

    def __init__(self, survey, exvel, perturbations, wlt, dobs, vmin: float, vmax: float, nita: int,
                 maxdv: float, sigfac: float, niterenkf: int, exvel_true=None, arith: int = ARITH_FAST):
        import torch
        self.s = survey
        self.niterenkf = niterenkf
        self.exvel_true = exvel_true
        self.arith = arith
        v0 = vel_recover(exvel, survey.dx, survey.dt)
        self.methods, self.members = [], []
        for p in perturbations:
            m = Damp4t10d.from_survey(survey, arith=arith)
            v = vel_trans((np.asarray(p, np.float32) + v0).astype(np.float32), survey.dx, survey.dt)
            self.methods.append(m)
            self.members.append(EssFwiFramework(m, v, vmin, vmax, nita, maxdv, wlt, dobs))
        self.n = len(self.members)
        self.fm = Damp4t10d.from_survey(survey, arith=arith)      # analysis and mean-model scoring
        self.wlt = torch.from_numpy(np.ascontiguousarray(wlt, np.float32)).cuda()
        self.dobs = torch.from_numpy(np.ascontiguousarray(dobs, np.float32)).cuda()
        self.enkf = EnkfAnalyze(self.fm, self.wlt, self.dobs, sigfac)
        self.analyses = 0
        self.absobj, self.norobj, self.logs = [], [], []

    def velocities(self):
        import torch
        return torch.from_numpy(np.stack([fw.velocity() for fw in self.members])).cuda()

    def analyze(self, z=None):
        """pAnalyze: every member moved in place."""
        codes = random_codes(ENKF_SEED, self.s.ns, skip=self.analyses)
        vels = self.velocities()
        t4, clip = self.enkf.analyze(vels, codes, z)
        host = vels.cpu().numpy()
        for fw, v in zip(self.members, host):
            fw.setVelocity(v)
        self.analyses += 1
        return t4, clip

    def mean_objective(self) -> float:
        """calobj of the members' mean model."""
        import torch
        vels = self.velocities()
        mean = self.enkf.createAMean(vels)
        nxpad, nzpad, ns, ng, nt = self.fm.dims()
        self.fm.bindVelocity(mean)
        self._mean = mean
        c = torch.from_numpy(random_codes(CALOBJ_SEED, ns)).cuda()
        encsrc = torch.empty((nt, ns), dtype=torch.float32, device="cuda")
        encode_source(encsrc, self.wlt, c)
        encobs = torch.empty((nt, ng), dtype=torch.float32, device="cuda")
        encode_obs(encobs, self.dobs, c)
        dcal = torch.zeros((nt, ng), dtype=torch.float32, device="cuda")
        self.fm.EssForwardModeling(encsrc, dcal)
        self.fm.removeDirectArrival(encobs)
        self.fm.removeDirectArrival(dcal)
        return float(cal_objective((encobs - dcal).contiguous()))

    def _score(self):
        obj = self.mean_objective()
        self.absobj.append(obj)
        self.norobj.append(obj / self.absobj[0])

    def _log(self, it: int):
        for i, fw in enumerate(self.members):
            row = {"iter": it, "member": i, "data_rss": fw.getUpdateObj()}
            if self.exvel_true is not None:
                row["slowness_l1"], row["slowness_l2"] = slowness_l1l2(
                    self.exvel_true, fw.velocity(), self.s.nx, self.s.nz, self.s.nb, self.s.dx, self.s.dt)
            self.logs.append(row)

    def run(self, niter: int, z_draws=None):
        """The driver's loop; z_draws(i) may supply the i-th analysis's
        observation-perturbation draws (default: drawn on the device)."""
        draw = z_draws or (lambda i: None)
        self.analyze(draw(0))
        self._score()
        for it in range(niter):
            for fw in self.members:
                fw.epoch(it)
            if it % self.niterenkf == 0:
                self._log(it)
                self.analyze(draw(self.analyses))
            self._score()
        return self.absobj, self.norobj
