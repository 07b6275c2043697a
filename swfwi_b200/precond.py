"""Learned preconditioner for plain FWI.

A small convolutional encoder-decoder (``include/swfwi_gpu.h``,
``swfwi_precond_*``; kernels in ``csrc/precond.cu``) maps three images of
the model interior -- the raw gradient of an FWI epoch, the current
(transformed) velocity and the source illumination of that epoch's forward
sweep -- to an update direction.  It is trained only on what plain FWI
itself produces: for every epoch k of a plain run on a seeded synthetic
model, the input is (gradient_k, velocity_k, illumination_k) and the target
is the update plain FWI still has to make, velocity_final - velocity_k, at
unit RMS.

Attached to a plain ``FwiFramework`` (``setPreconditioner``), each epoch
first searches along the network's direction with the plain step-length
search and keeps that step only when the search confirms an objective
decrease; otherwise it takes the plain CG step.  Plain FWI thus stays both
the fallback and the arbiter of every learned step.

The network has no counterpart in the reference (src/fwi/fwiframework.cpp
is the plain method it sits beside).
"""
from __future__ import annotations

import ctypes as C
import time

import numpy as np

from . import Damp4t10d, FwiFramework, _check, _fp, _ptr, _stream, lib

DEFAULT_WIDTHS = (16, 32, 64, 64)


def image_shape(method: Damp4t10d) -> tuple[int, int]:
    """Network image of a propagator's interior: rows along x, columns along
    depth, both rounded up to a multiple of 8."""
    nxpad, nzpad = method.dims()[:2]
    nx, nz = nxpad - 2 * method.nb - 12, nzpad - method.nb - 12
    return (nx + 7) // 8 * 8, (nz + 7) // 8 * 8


class Preconditioner:
    """The network (BF16 weights and activations, FP32 accumulation and
    master weights, Adam).  Tensors are torch CUDA float32 tensors."""

    def __init__(self, widths=DEFAULT_WIDTHS):
        w = (C.c_int * 4)(*[int(v) for v in widths])
        h = C.c_void_p()
        _check(lib().swfwi_precond_create(C.byref(h), w))
        self.h = h
        self.widths = tuple(int(v) for v in widths)

    def __del__(self):
        try:
            if getattr(self, "h", None):
                lib().swfwi_precond_destroy(self.h)
                self.h = None
        except Exception:
            pass

    @property
    def num_params(self) -> int:
        n = C.c_longlong()
        _check(lib().swfwi_precond_num_params(self.h, C.byref(n)))
        return n.value

    def layers(self):
        """[(cin, cout, w_off, b_off)] for the 14 3x3 convs and the 1x1 output."""
        out = []
        for l in range(15):
            ci, co, wo, bo = C.c_int(), C.c_int(), C.c_longlong(), C.c_longlong()
            _check(lib().swfwi_precond_layer(self.h, l, C.byref(ci), C.byref(co), C.byref(wo), C.byref(bo)))
            out.append((ci.value, co.value, wo.value, bo.value))
        return out

    def params(self) -> np.ndarray:
        p = np.zeros(self.num_params, np.float32)
        _check(lib().swfwi_precond_get_params(self.h, p.ctypes.data_as(_fp)))
        return p

    def set_params(self, p: np.ndarray) -> None:
        p = np.ascontiguousarray(p, np.float32)
        if p.size != self.num_params:
            raise ValueError(f"expected {self.num_params} parameters, got {p.size}")
        _check(lib().swfwi_precond_set_params(self.h, p.ctypes.data_as(_fp)))

    def grads(self) -> np.ndarray:
        g = np.zeros(self.num_params, np.float32)
        _check(lib().swfwi_precond_get_grads(self.h, g.ctypes.data_as(_fp)))
        return g

    def save(self, path: str) -> None:
        np.savez(path, params=self.params(), widths=np.asarray(self.widths))

    @classmethod
    def load(cls, path: str) -> "Preconditioner":
        z = np.load(path)
        net = cls(tuple(int(v) for v in z["widths"]))
        net.set_params(z["params"])
        return net

    # ---- raw network ----
    def forward(self, x, y=None, stream=None):
        """x [N][H][W][3] -> y [N][H][W]."""
        import torch
        N, H, W, c = x.shape
        assert c == 3 and x.is_contiguous() and x.dtype == torch.float32
        if y is None:
            y = torch.empty((N, H, W), dtype=torch.float32, device=x.device)
        _check(lib().swfwi_precond_forward(self.h, _ptr(x), _ptr(y), N, H, W, _stream(stream)))
        return y

    def backward(self, t, stream=None) -> float:
        loss = C.c_double()
        _check(lib().swfwi_precond_backward(self.h, _ptr(t), C.byref(loss), _stream(stream)))
        return loss.value

    def adam_step(self, lr: float, stream=None) -> None:
        _check(lib().swfwi_precond_adam_step(self.h, lr, _stream(stream)))

    def train_step(self, x, t, lr: float, stream=None) -> float:
        N, H, W, _ = x.shape
        loss = C.c_double()
        _check(lib().swfwi_precond_train_step(self.h, _ptr(x), _ptr(t), N, H, W, lr, C.byref(loss),
                                              _stream(stream)))
        return loss.value

    # ---- model grid <-> image ----
    def features(self, method: Damp4t10d, grad, vel, illum=None, stream=None):
        import torch
        H, W = image_shape(method)
        x3 = torch.empty((H, W, 3), dtype=torch.float32, device=grad.device)
        _check(lib().swfwi_precond_features(self.h, method.h, _ptr(grad), _ptr(vel),
                                            _ptr(illum) if illum is not None else None, _ptr(x3),
                                            _stream(stream)))
        return x3

    def target(self, method: Damp4t10d, dv, stream=None):
        import torch
        H, W = image_shape(method)
        t = torch.empty((H, W), dtype=torch.float32, device=dv.device)
        _check(lib().swfwi_precond_target(self.h, method.h, _ptr(dv), _ptr(t), _stream(stream)))
        return t

    def propose(self, method: Damp4t10d, grad, vel, illum=None, stream=None):
        import torch
        d = torch.empty_like(grad)
        _check(lib().swfwi_precond_propose(self.h, method.h, _ptr(grad), _ptr(vel),
                                           _ptr(illum) if illum is not None else None, _ptr(d),
                                           _stream(stream)))
        return d


# --------------------------------------------------------------------------
# Plain runs, training pairs, training, and the learned-vs-plain comparison
# --------------------------------------------------------------------------
def model_error(fw: FwiFramework, v_true_interior: np.ndarray) -> float:
    """Relative L2 error of the interior velocity (m/s)."""
    v = fw.writeVel().astype(np.float64)
    t = np.asarray(v_true_interior, np.float64)
    return float(np.linalg.norm(v - t) / np.linalg.norm(t))


def run_fwi(method: Damp4t10d, exvel0: np.ndarray, wlt: np.ndarray, dobs: np.ndarray, survey, iters: int,
            v_true_interior: np.ndarray | None = None, net: Preconditioner | None = None,
            collect: bool = False, target_error: float | None = None, min_decrease: float = 0.0,
            patience: int = 0):
    """Plain FWI (net None) or learned-preconditioned FWI for `iters` epochs.

    Returns a dict: history [(seconds since start, model error, objective,
    learned step taken)], and with collect=True the per-epoch (velocity,
    gradient, illumination) host arrays and the final velocity.  Stops early
    once the model error reaches target_error."""
    import torch
    fw = FwiFramework(method, exvel0, survey.vmin, survey.vmax, survey.nita, survey.maxdv, wlt, dobs)
    if net is not None:
        fw.setPreconditioner(net)
        fw.setLearnedMinDecrease(min_decrease)
        fw.setLearnedPatience(patience)
    if collect:
        fw.collectIllumination(True)
    hist, samples = [], []
    err0 = model_error(fw, v_true_interior) if v_true_interior is not None else None
    hist.append((0.0, err0, None, False))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    paused = 0.0
    for it in range(iters):
        if collect:
            v_before = fw.velocity()
        fw.epoch(it)
        torch.cuda.synchronize()
        t_now = time.perf_counter() - t0 - paused
        p0 = time.perf_counter()
        learned = fw.learnedStats()[0] if net is not None else False
        err = model_error(fw, v_true_interior) if v_true_interior is not None else None
        if collect:
            samples.append((v_before, fw.gradient(), fw.illumination()))
        paused += time.perf_counter() - p0     # bookkeeping is not FWI time
        hist.append((t_now, err, fw.getUpdateObj(), learned))
        if target_error is not None and err is not None and err <= target_error:
            break
    out = {"history": hist, "final": fw.velocity(), "stats": fw.learnedStats() if net is not None else None}
    if collect:
        out["samples"] = samples
    return out


def training_pairs(net: Preconditioner, method: Damp4t10d, run: dict, skip_last: int = 3,
                   horizon: int | None = None):
    """(inputs [S][H][W][3], targets [S][H][W]) on the device from one
    collected plain run: input = features of (gradient_k, velocity_k,
    illumination_k), target = velocity_{k+horizon} - velocity_k (horizon
    None: the run's final velocity) at unit RMS."""
    import torch
    final = torch.from_numpy(run["final"]).cuda()
    xs, ts = [], []
    samples = run["samples"]
    for k, (v, g, il) in enumerate(samples[: max(1, len(samples) - skip_last)]):
        vd = torch.from_numpy(v).cuda()
        gd = torch.from_numpy(g).cuda()
        ild = torch.from_numpy(il).cuda()
        if horizon is None or k + horizon >= len(samples):
            ahead = final
        else:
            ahead = torch.from_numpy(samples[k + horizon][0]).cuda()
        xs.append(net.features(method, gd, vd, ild))
        ts.append(net.target(method, (ahead - vd).contiguous()))
    torch.cuda.synchronize()
    return torch.stack(xs), torch.stack(ts)


def train(net: Preconditioner, X, T, epochs: int = 40, batch: int = 8, lr: float = 1e-3, seed: int = 0,
          flip: bool = True, verbose: bool = False):
    """Adam on minibatches of (X, T); flip=True adds the mirror image along
    x (the acquisition is left-right symmetric).  Returns the mean loss of
    each epoch."""
    import torch
    g = torch.Generator().manual_seed(seed)
    S = X.shape[0]
    losses = []
    for ep in range(epochs):
        perm = torch.randperm(S, generator=g).tolist()
        tot, nb = 0.0, 0
        for b0 in range(0, S, batch):
            idx = perm[b0:b0 + batch]
            x = X[idx]
            t = T[idx]
            if flip and (ep % 2 == 1):
                x = torch.flip(x, dims=[1])
                t = torch.flip(t, dims=[1])
            tot += net.train_step(x.contiguous(), t.contiguous(), lr)
            nb += 1
        losses.append(tot / max(nb, 1))
        if verbose:
            print(f"epoch {ep:3d} loss {losses[-1]:.4f}")
    return losses


def time_to_error(history, target: float):
    """Seconds until the model error first reaches `target` (None if never)."""
    for t, e, _, _ in history:
        if e is not None and e <= target:
            return t
    return None


def demo_survey(nz: int = 80, nx: int = 240, nt: int = 1000, ns: int = 12):
    """The learned-preconditioner workload's recipe on a grid one run can
    afford: 25 m cells, 2 ms steps, 10 Hz Ricker, 30-point sponge, shots
    evenly spaced at the surface, receivers at every surface point."""
    from .survey import Survey
    jsx = nx // ns
    return Survey(name="learned-demo", nz=nz, nx=nx, dx=25.0, dt=0.002, nt=nt, fm=10.0, nb=30,
                  ns=ns, sxbeg=jsx // 2, jsx=jsx, ng=nx)


def anomaly_model(nx: int, nz: int, seed: int):
    """(true, background) [nx][nz] float32: a linear depth gradient (top
    1600-2000 m/s, bottom 3500-4300 m/s) plus 4-8 Gaussian anomalies of
    +-150-350 m/s with radii of 6-14 points across and 4-10 in depth, all
    seeded."""
    rng = np.random.default_rng(seed)
    x = np.arange(nx, dtype=np.float64)[:, None]
    z = np.arange(nz, dtype=np.float64)[None, :]
    top, bot = rng.uniform(1600, 2000), rng.uniform(3500, 4300)
    bg = (top + (bot - top) * z / max(nz - 1, 1)) * np.ones((nx, 1))
    v = bg.copy()
    for _ in range(int(rng.integers(4, 9))):
        cx, cz = rng.uniform(0.1, 0.9) * nx, rng.uniform(0.2, 0.85) * nz
        rx, rz = rng.uniform(6, 14), rng.uniform(4, 10)
        amp = rng.choice([-1.0, 1.0]) * rng.uniform(150, 350)
        v += amp * np.exp(-(((x - cx) / rx) ** 2 + ((z - cz) / rz) ** 2))
    return v.astype(np.float32), bg.astype(np.float32)


def synthetic_case(survey, seed: int, recipe: str = "anomaly", smooth_sigma: float = 10.0, arith: int = 1):
    """(method, initial padded model, true interior velocity, wavelet, dobs)
    for one seeded model; dobs modelled on the GPU.  recipe "anomaly":
    anomaly_model, starting from its background; "anomaly-smooth": the same
    truth, starting from it smoothed with smooth_sigma; "layered": the
    layered+random model, starting from it smoothed with smooth_sigma."""
    import torch
    from . import ricker_wavelet
    from .survey import layered_model, smooth
    if recipe == "layered":
        vtrue = layered_model(survey.nx, survey.nz, seed=seed)
        vinit = smooth(vtrue, smooth_sigma).astype(np.float32)
    elif recipe == "anomaly":
        vtrue, vinit = anomaly_model(survey.nx, survey.nz, seed)
    elif recipe == "anomaly-smooth":
        vtrue, _ = anomaly_model(survey.nx, survey.nz, seed)
        vinit = smooth(vtrue, smooth_sigma).astype(np.float32)
    else:
        raise ValueError(recipe)
    m = Damp4t10d.from_survey(survey, arith=arith)
    ex_true = m.expandDomain(vtrue)
    ex_init = m.expandDomain(vinit)
    wlt = ricker_wavelet(survey.nt, survey.fm, survey.dt)
    vt = torch.from_numpy(ex_true).cuda()
    m.bindVelocity(vt)
    d = torch.zeros((survey.ns, survey.nt, survey.ng), device="cuda")
    m.forward_batch(torch.from_numpy(wlt).cuda(), d, list(range(survey.ns)))
    dobs = d.cpu().numpy()
    return m, ex_init, vtrue, wlt, dobs


def train_from_plain(survey, train_seeds, iters: int, epochs: int, lr: float = 1e-3, batch: int = 16,
                     widths=DEFAULT_WIDTHS, recipe: str = "anomaly", verbose: bool = False,
                     horizon: int | None = None):
    """Collect training pairs from plain FWI runs (iters epochs each) on the
    seeded models and train a network on them (targets `horizon` plain
    epochs ahead, or the run's end).  Returns (net, stats)."""
    import torch
    net = Preconditioner(widths)
    X, T = [], []
    t_collect = time.perf_counter()
    for sd in train_seeds:
        m, ex0, vtrue, wlt, dobs = synthetic_case(survey, sd, recipe)
        run = run_fwi(m, ex0, wlt, dobs, survey, iters, vtrue, collect=True)
        x, t = training_pairs(net, m, run, horizon=horizon)
        X.append(x)
        T.append(t)
        if verbose:
            print(f"model {sd}: plain error {run['history'][0][1]:.4f} -> {run['history'][-1][1]:.4f}")
        del m
    X = torch.cat(X).contiguous()
    T = torch.cat(T).contiguous()
    t_collect = time.perf_counter() - t_collect
    torch.cuda.synchronize()
    t_train = time.perf_counter()
    losses = train(net, X, T, epochs=epochs, batch=batch, lr=lr, verbose=verbose)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t_train
    return net, {"samples": int(X.shape[0]), "params": net.num_params, "collect_s": t_collect,
                 "train_s": t_train, "loss_first": losses[0], "loss_last": losses[-1]}


def compare(survey, net: Preconditioner, test_seed: int, iters: int, recipe: str = "anomaly",
            min_decrease: float = 0.0, plain=None, patience: int = 0):
    """Plain and learned FWI on one held-out model: the lowest model error
    the plain run reaches in `iters` epochs is the target; returns the seconds
    each method needs to reach it with both histories (pass `plain` to reuse
    a plain run of the same model)."""
    m, ex0, vtrue, wlt, dobs = synthetic_case(survey, test_seed, recipe)
    if plain is None:
        plain = run_fwi(m, ex0, wlt, dobs, survey, iters, vtrue)
    # the best model error plain FWI reaches in its budget (its error need
    # not fall monotonically)
    target = min(h[1] for h in plain["history"][1:])
    learned = run_fwi(m, ex0, wlt, dobs, survey, iters, vtrue, net=net, target_error=target,
                      min_decrease=min_decrease, patience=patience)
    return {"target_error": target, "initial_error": plain["history"][0][1],
            "plain_s": time_to_error(plain["history"], target),
            "learned_s": time_to_error(learned["history"], target),
            "plain_history": plain["history"], "learned_history": learned["history"],
            "learned_stats": learned["stats"], "plain": plain}


def learned_vs_plain(survey=None, train_seeds=range(100, 108), test_seed: int = 200, iters: int = 25,
                     epochs: int = 60, lr: float = 1e-3, batch: int = 8, widths=DEFAULT_WIDTHS,
                     recipe: str = "anomaly", min_decrease: float = 0.0, verbose: bool = False):
    """Train on plain runs over seeded models, then run plain and learned
    FWI on a held-out model.  Returns the measurements: both histories, the
    lowest model error the plain run reaches (the target), the seconds each
    method needs to reach it, training time and loss."""
    survey = survey or demo_survey()
    net, st = train_from_plain(survey, train_seeds, iters, epochs, lr, batch, widths, recipe, verbose)
    r = compare(survey, net, test_seed, iters, recipe, min_decrease)
    return {"survey": survey, "net": net, **st, **r}
