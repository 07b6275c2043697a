"""Autotuner for the streaming stencil's launch shape.

The streaming step (``stream.cuh``) has knobs that do not change its
results: which kernel (register-queue warps, each a self-contained TMA
pipeline, one or two rows a stage; or warp-specialised CTAs with a copy
warp), output depths per
CTA, rows per task (0: the register-queue kernel's automatic length, one
wave of tasks), rows in flight ahead of the compute and the launch
order (shots slowest or fastest).  ``tune`` times short batched forward runs of a survey for each
candidate with the library's CUDA-event step timing and returns the fastest;
``apply`` sets it on a propagator.
"""
from __future__ import annotations

import itertools

import numpy as np

DEFAULT = {"kernel": 6, "band_depth": 120, "rows_per_cta": 0, "rows_in_flight": 3,
           "shots_slowest": False}


def candidates(nz: int):
    """The register-queue kernel's task lengths and prefetch depths, the
    warp-specialised kernel's band depths, chunk lengths, prefetch depths
    and launch orders."""
    for rows in (0, 64, 96, 128):
        yield {"kernel": 6, "band_depth": 120, "rows_per_cta": rows, "rows_in_flight": 3, "shots_slowest": False}
    for rows, depth in itertools.product((0, 32, 48, 64), (3, 7)):
        yield {"kernel": 5, "band_depth": 120, "rows_per_cta": rows, "rows_in_flight": depth,
               "shots_slowest": False}
    for bz, rows, depth, order in itertools.product((248, 376), (48, 64), (3, 7), (False, True)):
        yield {"kernel": 1, "band_depth": bz, "rows_per_cta": rows, "rows_in_flight": depth,
               "shots_slowest": order}


def valid(cfg: dict) -> bool:
    """The launch shapes swfwi_damp4t10d_set_tuning accepts."""
    if cfg["kernel"] in (5, 6):
        ok_bz = cfg["band_depth"] == 120
    elif cfg["kernel"] == 1:
        ok_bz = cfg["band_depth"] in (120, 248, 376)
    else:
        return False
    return ok_bz and cfg["rows_in_flight"] in (3, 7) and cfg["rows_per_cta"] >= 0


def time_config(method, wlt, dcal, ids, cfg, repeats=2) -> float:
    """Mean stencil launch time (microseconds) of a short batched forward."""
    import swfwi_b200 as S
    method.set_fusion(False)          # time the launch shape itself
    method.set_tuning(**cfg)
    method.forward_batch(wlt, dcal, ids)      # warm-up
    S.stats_reset()
    S.stats_enable_step_timing(True)
    for _ in range(repeats):
        method.forward_batch(wlt, dcal, ids)
    st = S.stats_read()
    S.stats_enable_step_timing(False)
    return st["step_ms"] * 1e3 / max(st["step_launches"], 1)


def tune(survey, vel_padded: np.ndarray, arith: int, nt_probe: int = 24, shots: int | None = None,
         configs=None, verbose: bool = False):
    """Times every candidate on `shots` shots (default: all) of the survey
    over nt_probe steps; returns (best config, table)."""
    import torch
    import swfwi_b200 as S
    s = survey.scaled(nt=nt_probe)
    m = S.Damp4t10d.from_survey(s, arith=arith)
    vel = torch.from_numpy(np.ascontiguousarray(vel_padded, np.float32)).cuda()
    m.bindVelocity(vel)
    wlt = torch.from_numpy(S.ricker_wavelet(s.nt, s.fm, s.dt)).cuda()
    n = s.ns if shots is None else min(shots, s.ns)
    ids = np.arange(n, dtype=np.int32)
    dcal = torch.zeros((n, s.nt, m.getng()), device="cuda")
    table = []
    for cfg in (configs or list(candidates(s.nzpad))):
        us = time_config(m, wlt, dcal, ids, cfg)
        table.append((us, cfg))
        if verbose:
            print(f"{us:9.1f} us  {cfg}")
    table.sort(key=lambda r: r[0])
    # within 1 % of the fastest (timing noise), prefer the automatic task
    # length: it sizes the tasks for whatever grid the propagator runs next
    near = [cfg for us, cfg in table if us <= 1.01 * table[0][0] and cfg.get("rows_per_cta", 1) == 0]
    return (near[0] if near else table[0][1]), table


def apply(method, cfg: dict) -> None:
    method.set_tuning(**cfg)
