"""swfwi_b200: swfwi's 2D acoustic FWI path on NVIDIA B200 (sm_100a).

The product is the shared library ``libswfwi_b200.so`` (C ABI in
``include/swfwi_gpu.h``).  This module is a thin ctypes mirror of the
reference's C++ interface for tests, benchmarks and Python callers:

* ``fd4t10s_damp_zjh_2d_vtrans`` / ``fd4t10s_zjh_2d_vtrans``: the drop-in
  stencil steps (src/modeling/fd4t10s-*.h).
* ``ShotPosition``, ``Damp4t10d``: the propagator (src/modeling/damp4t10d.h),
  method names as in the reference.
* ``FwiFramework``, ``EssFwiFramework``: the inversion drivers
  (src/fwi/fwiframework.h, src/essfwi/essfwiframework.h).

Device arrays are torch CUDA tensors (torch is used for device memory and
streams only; every computation runs in the library's kernels).  There is
no CPU fallback: loading fails loudly when the library is missing.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libswfwi_b200.so")

ARITH_REF, ARITH_FAST, ARITH_F64 = 0, 1, 2
STRIP_F32, STRIP_F16, STRIP_BF16 = 0, 1, 2
RECON_STRIPS, RECON_SNAPSHOTS = 0, 1


class SwfwiError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"swfwi status {status}: {msg}")
        self.status = status


class Stats(C.Structure):
    _fields_ = [("kernel_launches", C.c_longlong), ("step_launches", C.c_longlong),
                ("step_ms", C.c_double), ("step_point_updates", C.c_double), ("step_bytes", C.c_double),
                ("step_timed_launches", C.c_longlong)]


class _ShotPos(C.Structure):
    _fields_ = [(n, C.c_int) for n in ("szbeg", "sxbeg", "jsz", "jsx", "ns", "nz")]


_lib = None
_vp, _fp, _dp, _ip = C.c_void_p, C.POINTER(C.c_float), C.POINTER(C.c_double), C.POINTER(C.c_int)

_SIGS = {
    "swfwi_fd4t10s_damp_zjh_2d_vtrans": [_vp, _vp, _vp, _vp, C.c_int, C.c_int, C.c_int, _vp],
    "swfwi_fd4t10s_zjh_2d_vtrans": [_vp, _vp, _vp, _vp, C.c_int, C.c_int, _vp],
    "swfwi_fd4t10s_step_batch": [_vp, _vp, _vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                 C.c_longlong, _vp],
    "swfwi_fd4t10s_step_f64": [_vp, _vp, _vp, C.c_int, C.c_int, C.c_int, C.c_int, _vp],
    "swfwi_damp4t10d_create": [C.POINTER(_vp), C.POINTER(_ShotPos), C.POINTER(_ShotPos), C.c_float,
                               C.c_float, C.c_float, C.c_int, C.c_int],
    "swfwi_damp4t10d_destroy": [_vp],
    "swfwi_damp4t10d_set_stream": [_vp, _vp],
    "swfwi_damp4t10d_set_arith": [_vp, C.c_int],
    "swfwi_damp4t10d_set_strip_format": [_vp, C.c_int],
    "swfwi_damp4t10d_set_reconstruction": [_vp, C.c_int, C.c_int, C.c_int],
    "swfwi_damp4t10d_set_tuning": [_vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int],
    "swfwi_damp4t10d_set_receivers_per_shot": [_vp, _ip, _ip, _ip],
    "swfwi_damp4t10d_dims": [_vp, _ip, _ip, _ip, _ip, _ip],
    "swfwi_damp4t10d_expand_domain": [_vp, _fp, C.c_int, C.c_int, _fp],
    "swfwi_damp4t10d_set_model_size": [_vp, C.c_int, C.c_int],
    "swfwi_damp4t10d_bind_velocity": [_vp, _vp],
    "swfwi_damp4t10d_step_forward": [_vp, _vp, _vp],
    "swfwi_damp4t10d_step_backward": [_vp, _vp, _vp],
    "swfwi_damp4t10d_add_source": [_vp, _vp, _vp, C.c_int],
    "swfwi_damp4t10d_sub_source": [_vp, _vp, _vp, C.c_int],
    "swfwi_damp4t10d_add_receiver_source": [_vp, _vp, _vp],
    "swfwi_damp4t10d_record_seis": [_vp, _vp, _vp],
    "swfwi_damp4t10d_bndry_size": [_vp, _ip],
    "swfwi_damp4t10d_write_bndry": [_vp, _vp, _vp, C.c_int],
    "swfwi_damp4t10d_read_bndry": [_vp, _vp, _vp, C.c_int],
    "swfwi_damp4t10d_mask_gradient": [_vp, _vp],
    "swfwi_damp4t10d_scale_gradient": [_vp, _vp],
    "swfwi_damp4t10d_refill_boundary": [_vp, _vp],
    "swfwi_damp4t10d_remove_direct_arrival": [_vp, _vp, C.c_int],
    "swfwi_damp4t10d_fwi_forward_modeling": [_vp, _vp, _vp, C.c_int],
    "swfwi_damp4t10d_ess_forward_modeling": [_vp, _vp, _vp],
    "swfwi_damp4t10d_forward_batch": [_vp, _vp, _vp, _ip, C.c_int],
    "swfwi_damp4t10d_gradient_batch": [_vp, _vp, _vp, _ip, C.c_int, _vp, _dp],
    "swfwi_gradient_host": [_vp, _fp, _fp, _fp, _ip, C.c_int, _fp, _dp],
    "swfwi_damp4t10d_calgradient_ess": [_vp, _vp, _vp, _vp],
    "swfwi_damp4t10d_calgradient_fwi": [_vp, _vp, _vp, _vp, C.c_int],
    "swfwi_damp4t10d_calgradient_fwi_f64": [_vp, _vp, _vp, _vp, _vp, C.c_int],
    "swfwi_damp4t10d_calgradient_ess_f64": [_vp, _vp, _vp, _vp, _vp],
    "swfwi_damp4t10d_fwi_forward_modeling_f64": [_vp, _vp, _vp, _vp, C.c_int],
    "swfwi_update_grad": [_vp, _vp, _vp, C.c_int, C.c_int, _vp],
    "swfwi_cal_max_alpha": [_vp, _vp, C.c_int, C.c_float, C.c_float, C.c_float, _fp, _fp, _vp],
    "swfwi_update_vel": [_vp, _vp, _vp, C.c_int, C.c_float, C.c_float, C.c_float, C.c_float,
                         C.c_float, _vp],
    "swfwi_trans_vsrc": [_vp, _vp, C.c_int, C.c_int, _vp],
    "swfwi_cal_objective": [_vp, C.c_longlong, _dp, _vp],
    "swfwi_cal_objective_static": [_vp, C.c_longlong, C.c_int, _vp, _vp],
    "swfwi_encode_source": [_vp, _vp, _vp, C.c_int, C.c_int, _vp],
    "swfwi_fwi_set_velocity": [_vp, _fp],
    "swfwi_damp4t10d_set_fusion": [_vp, C.c_int],
    "swfwi_damp4t10d_set_graphs": [_vp, C.c_int],
    "swfwi_rsf_get": [C.c_char_p, C.c_char_p, C.c_char_p, C.c_int],
    "swfwi_rsf_dims": [C.c_char_p, _ip, _ip, _fp, _fp],
    "swfwi_rsf_read": [C.c_char_p, _fp, C.c_longlong, C.c_longlong],
    "swfwi_rsf_write": [C.c_char_p, C.c_char_p, _fp, C.c_int, _ip, _fp, _fp, C.c_char_p],
    "swfwi_rsf_read_shots": [C.c_char_p, _fp, C.c_int, C.c_int, C.c_int],
    "swfwi_rsf_write_shots": [C.c_char_p, C.c_char_p, _fp, C.c_int, C.c_int, C.c_int, C.c_float, C.c_float,
                              C.c_char_p],
    "swfwi_encode_obs": [_vp, _vp, _vp, C.c_longlong, C.c_int, _vp],
    "swfwi_damp4t10d_ess_forward_members": [_vp, _vp, _vp, C.c_int, _vp],
    "swfwi_enkf_gain_matrix": [_vp, _vp, _vp, C.c_longlong, C.c_int, C.c_float, _dp, C.c_ulonglong, _dp,
                               _ip, _vp],
    "swfwi_enkf_update": [_vp, C.c_longlong, C.c_int, _dp, C.c_float, C.c_float, _vp],
    "swfwi_enkf_analyze": [_vp, _vp, _vp, C.c_longlong, C.c_int, C.c_float, _dp, C.c_ulonglong, _vp,
                           C.c_longlong, C.c_float, C.c_float, _dp, _ip, _vp],
    "swfwi_enkf_mean": [_vp, _vp, C.c_longlong, C.c_int, _vp],
    "swfwi_parabola_vertex": [C.c_float] * 7 + [_fp, _fp],
    "swfwi_ricker_wavelet": [_fp, C.c_int, C.c_float, C.c_float, C.c_float],
    "swfwi_random_codes": [C.c_int, C.c_int, C.c_int, _ip],
    "swfwi_fwi_create": [C.POINTER(_vp), _vp, _fp, C.c_float, C.c_float, C.c_int, C.c_float, _fp,
                         _fp, C.c_int],
    "swfwi_fwi_destroy": [_vp],
    "swfwi_fwi_epoch": [_vp, C.c_int],
    "swfwi_fwi_get_update_obj": [_vp, _fp],
    "swfwi_fwi_get_init_obj": [_vp, _fp],
    "swfwi_fwi_get_velocity": [_vp, _fp],
    "swfwi_fwi_write_vel": [_vp, _fp],
    "swfwi_fwi_last_line_search": [_vp, _fp, _fp],
    "swfwi_fwi_last_trials": [_vp, _ip],
    "swfwi_precond_create": [C.POINTER(_vp), _ip],
    "swfwi_precond_destroy": [_vp],
    "swfwi_precond_num_params": [_vp, C.POINTER(C.c_longlong)],
    "swfwi_precond_layer": [_vp, C.c_int, _ip, _ip, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)],
    "swfwi_precond_set_params": [_vp, _fp],
    "swfwi_precond_get_params": [_vp, _fp],
    "swfwi_precond_get_grads": [_vp, _fp],
    "swfwi_precond_forward": [_vp, _vp, _vp, C.c_int, C.c_int, C.c_int, _vp],
    "swfwi_precond_backward": [_vp, _vp, _dp, _vp],
    "swfwi_precond_adam_step": [_vp, C.c_float, _vp],
    "swfwi_precond_train_step": [_vp, _vp, _vp, C.c_int, C.c_int, C.c_int, C.c_float, _dp, _vp],
    "swfwi_precond_features": [_vp, _vp, _vp, _vp, _vp, _vp, _vp],
    "swfwi_precond_target": [_vp, _vp, _vp, _vp, _vp],
    "swfwi_precond_propose": [_vp, _vp, _vp, _vp, _vp, _vp, _vp],
    "swfwi_fwi_set_preconditioner": [_vp, _vp],
    "swfwi_fwi_collect_illumination": [_vp, C.c_int],
    "swfwi_fwi_set_regularization": [_vp, C.c_float, C.c_float],
    "swfwi_regu_term": [_vp, C.c_int, C.c_int, C.c_float, C.c_float, _dp, _vp],
    "swfwi_regu_gradient": [_vp, C.c_int, C.c_int, C.c_float, C.c_float, _vp, C.c_int, _vp],
    "swfwi_prtm2d_create": [C.POINTER(_vp), C.c_int] + [C.c_float] * 5 + [C.c_int] * 15 + [_vp, _vp],
    "swfwi_prtm2d_set_adjoint": [_vp, C.c_int],
    "swfwi_prtm2d_set_graphs": [_vp, C.c_int],
    "swfwi_prtm2d_batch": [_vp, _ip],
    "swfwi_prtm2d_lop": [_vp, C.c_int, C.c_int, C.c_int, C.c_int, _vp, _vp, _vp],
    "swfwi_prtm2d_destroy": [_vp],
    "swfwi_fwi_set_learned_min_decrease": [_vp, C.c_float],
    "swfwi_fwi_set_learned_patience": [_vp, C.c_int],
    "swfwi_fwi_get_gradient": [_vp, _fp],
    "swfwi_fwi_get_illumination": [_vp, _fp],
    "swfwi_fwi_learned_stats": [_vp, _ip, _ip, _ip],
    "swfwi_selftest_bounded_wait": [_vp],
    "swfwi_stats_reset": [],
    "swfwi_stats_enable_step_timing": [C.c_int],
    "swfwi_stats_read": [C.POINTER(Stats)],
    "swfwi_status_string": [C.c_int],
    "swfwi_last_error": [],
    "swfwi_version": [],
}


def lib() -> C.CDLL:
    """The loaded C ABI library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OSError(f"{LIB_PATH} is missing: run `python -m swfwi_b200.build` "
                          "(there is no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        for name, args in _SIGS.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = C.c_int
        L.swfwi_status_string.restype = C.c_char_p
        L.swfwi_last_error.restype = C.c_char_p
        _lib = L
    return _lib


def exported_symbols() -> list[str]:
    return sorted(_SIGS)


def _check(status: int) -> None:
    if status != 0:
        msg = lib().swfwi_last_error().decode(errors="replace")
        raise SwfwiError(status, msg)


def _ptr(t) -> C.c_void_p:
    """Device pointer of a torch CUDA tensor (or an int address)."""
    if t is None:
        return C.c_void_p(0)
    if isinstance(t, int):
        return C.c_void_p(t)
    if not t.is_cuda:
        raise ValueError("expected a CUDA tensor: this library has no CPU path")
    if not t.is_contiguous():
        raise ValueError("expected a contiguous tensor")
    return C.c_void_p(t.data_ptr())


def _stream(stream=None) -> C.c_void_p:
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)


def _host_f32(a):
    a = np.ascontiguousarray(a, dtype=np.float32)
    return a, a.ctypes.data_as(_fp)


# ---------------------------------------------------------------- drop-in
def fd4t10s_damp_zjh_2d_vtrans(prev, curr, vel, nb: int, u2=None, stream=None) -> None:
    """Damped step in place over ``prev`` ([nx][nz] float32 CUDA tensors),
    bit-identical to the reference kernel."""
    nx, nz = prev.shape
    _check(lib().swfwi_fd4t10s_damp_zjh_2d_vtrans(_ptr(prev), _ptr(curr), _ptr(vel), _ptr(u2), nx, nz,
                                                  nb, _stream(stream)))


def fd4t10s_zjh_2d_vtrans(prev, curr, vel, u2=None, stream=None) -> None:
    nx, nz = prev.shape
    _check(lib().swfwi_fd4t10s_zjh_2d_vtrans(_ptr(prev), _ptr(curr), _ptr(vel), _ptr(u2), nx, nz,
                                             _stream(stream)))


def fd4t10s_step_batch(prev, curr, vel, nb: int, damped: bool = True, arith: int = ARITH_REF,
                       stream=None) -> None:
    """Batched step over prev/curr of shape [nshots][nx][nz]."""
    nsh, nx, nz = prev.shape
    _check(lib().swfwi_fd4t10s_step_batch(_ptr(prev), _ptr(curr), _ptr(vel), nx, nz, nb, int(damped),
                                          arith, nsh, nx * nz, _stream(stream)))


def fd4t10s_step_f64(prev, curr, vel, nb: int, damped: bool = True, stream=None) -> None:
    nx, nz = prev.shape
    _check(lib().swfwi_fd4t10s_step_f64(_ptr(prev), _ptr(curr), _ptr(vel), nx, nz, nb, int(damped),
                                        _stream(stream)))


# ---------------------------------------------------------------- stats
def stats_reset() -> None:
    _check(lib().swfwi_stats_reset())


def stats_enable_step_timing(on=True) -> None:
    """False/0: off; True/1: count every stencil launch and time each;
    n >= 2: count every launch, time every n-th."""
    _check(lib().swfwi_stats_enable_step_timing(int(on)))


def stats_read() -> dict:
    st = Stats()
    _check(lib().swfwi_stats_read(C.byref(st)))
    return {k: getattr(st, k) for k, _ in Stats._fields_}


# ---------------------------------------------------------------- helpers
def ricker_wavelet(nt: int, fm: float, dt: float, amp: float = 1.0) -> np.ndarray:
    w = np.zeros(nt, np.float32)
    _check(lib().swfwi_ricker_wavelet(w.ctypes.data_as(_fp), nt, fm, dt, amp))
    return w


def random_codes(seed: int, n: int, skip: int = 0) -> np.ndarray:
    c = np.zeros(n, np.int32)
    _check(lib().swfwi_random_codes(seed, skip, n, c.ctypes.data_as(_ip)))
    return c


def parabola_vertex(x1, y1, x2, y2, x3, y3, max_alpha3):
    a, b = C.c_float(), C.c_float()
    _check(lib().swfwi_parabola_vertex(x1, y1, x2, y2, x3, y3, max_alpha3, C.byref(a), C.byref(b)))
    return a.value, b.value


def update_grad(pre, cur, direction, it: int, stream=None) -> None:
    _check(lib().swfwi_update_grad(_ptr(pre), _ptr(cur), _ptr(direction), cur.numel(), it,
                                   _stream(stream)))


def cal_max_alpha(vel, grad, dt, dx, maxdv, stream=None):
    a2, a3 = C.c_float(), C.c_float()
    _check(lib().swfwi_cal_max_alpha(_ptr(vel), _ptr(grad), vel.numel(), dt, dx, maxdv, C.byref(a2),
                                     C.byref(a3), _stream(stream)))
    return a2.value, a3.value


def update_vel(new_vel, vel, grad, steplen, vmin, vmax, dx, dt, stream=None) -> None:
    _check(lib().swfwi_update_vel(_ptr(new_vel), _ptr(vel), _ptr(grad), vel.numel(), steplen, vmin,
                                  vmax, dx, dt, _stream(stream)))


def trans_vsrc(out, inp, stream=None) -> None:
    nt, ng = inp.shape
    _check(lib().swfwi_trans_vsrc(_ptr(out), _ptr(inp), nt, ng, _stream(stream)))


def cal_objective(r, stream=None) -> float:
    o = C.c_double()
    _check(lib().swfwi_cal_objective(_ptr(r), r.numel(), C.byref(o), _stream(stream)))
    return o.value


def encode_source(encsrc, wlt, codes, stream=None) -> None:
    """Encoder::encodeSource: encsrc [nt][ns] = wlt[it] * codes[is] (CUDA)."""
    nt, ns = encsrc.shape
    _check(lib().swfwi_encode_source(_ptr(encsrc), _ptr(wlt), _ptr(codes), nt, ns, _stream(stream)))


def encode_obs(encobs, dobs, codes, stream=None) -> None:
    """Encoder::encodeObsData: encobs [nt][ng] = sum_s codes[s] * dobs[s] (CUDA)."""
    _check(lib().swfwi_encode_obs(_ptr(encobs), _ptr(dobs), _ptr(codes), encobs.numel(), dobs.shape[0],
                                  _stream(stream)))


def enkf_gain_matrix(hona, dobs, z=None, sigfac: float = 0.0, sigma: float = 0.0, seed: int = 1,
                     stream=None):
    """calGainMatrix on the device: hona [n][rows] float32, dobs [rows]
    float32, z [n][rows] float64 or None (device draws).  Returns (t4 as
    numpy [n][n] indexed [row, col], sigma, clip)."""
    n, rows = hona.shape
    t4 = np.zeros((n, n), np.float64)   # filled column-major: t4c[col][row]
    sg = C.c_double(sigma)
    clip = C.c_int(0)
    _check(lib().swfwi_enkf_gain_matrix(_ptr(hona), _ptr(dobs), _ptr(z) if z is not None else None, rows, n,
                                        sigfac, C.byref(sg), seed, t4.ctypes.data_as(_dp), C.byref(clip),
                                        _stream(stream)))
    return t4.T.copy(), sg.value, clip.value


def enkf_update(vels, t4, dx: float, dt: float, stream=None) -> None:
    """analyze's member update in place: vels [n][model] float32 CUDA; t4
    numpy [n][n] indexed [row, col]."""
    n = vels.shape[0]
    t4c = np.ascontiguousarray(np.asarray(t4, np.float64).T)   # column-major for the C ABI
    _check(lib().swfwi_enkf_update(_ptr(vels), vels.numel() // n, n, t4c.ctypes.data_as(_dp), dx, dt,
                                   _stream(stream)))


def enkf_analyze(hona, dobs, vels, dx: float, dt: float, z=None, sigfac: float = 0.0, sigma: float = 0.0,
                 seed: int = 1, stream=None):
    """Gain and member update in one device-side call: vels [n][...] float32
    CUDA moved in place.  Returns (t4 numpy [n][n] indexed [row, col],
    sigma, clip)."""
    n, rows = hona.shape
    t4 = np.zeros((n, n), np.float64)
    sg = C.c_double(sigma)
    clip = C.c_int(0)
    _check(lib().swfwi_enkf_analyze(_ptr(hona), _ptr(dobs), _ptr(z) if z is not None else None, rows, n, sigfac,
                                    C.byref(sg), seed, _ptr(vels), vels.numel() // n, dx, dt,
                                    t4.ctypes.data_as(_dp), C.byref(clip), _stream(stream)))
    return t4.T.copy(), sg.value, clip.value


def enkf_mean(mean, vels, stream=None) -> None:
    n = vels.shape[0]
    _check(lib().swfwi_enkf_mean(_ptr(mean), _ptr(vels), vels.numel() // n, n, _stream(stream)))


class EnkfAnalyze:
    """EnkfAnalyze (src/enfwi/enkfanalyze.h): the ensemble Kalman analysis
    of the encoded observed data, on the GPU.  fm: the propagator (geometry,
    dt, dx); wlt [nt] and dobs [ns][nt][ng]: CUDA tensors; sigfac: the
    perturbation factor.  sigma is fixed at the first analysis, as the
    reference's initPerturbation does."""

    def __init__(self, fm, wlt, dobs, sigfac: float):
        self.fm, self.wlt, self.dobs, self.sigfac = fm, wlt, dobs, sigfac
        self.sigma = 0.0
        self.seed = 1

    def calGainMatrix(self, vels, codes, z=None):
        """vels [N][nxpad][nzpad] CUDA members; codes [ns] +-1 ints.  Returns
        (t4 [N][N] numpy, clip)."""
        hona, d = self._encoded(vels, codes)
        t4, self.sigma, clip = enkf_gain_matrix(hona, d, z, self.sigfac, self.sigma, self.seed)
        self.seed += 1
        return t4, clip

    def _encoded(self, vels, codes):
        import torch
        nxpad, nzpad, ns, ng, nt = self.fm.dims()
        c = torch.as_tensor(np.asarray(codes, np.int32), device=self.wlt.device)
        encsrc = torch.empty((nt, ns), dtype=torch.float32, device=self.wlt.device)
        encode_source(encsrc, self.wlt, c)
        encobs = torch.empty((nt, ng), dtype=torch.float32, device=self.wlt.device)
        encode_obs(encobs, self.dobs, c)
        d = encobs.t().contiguous().reshape(-1)             # matrix_transpose: row ig*nt + it
        hona = torch.empty((vels.shape[0], ng * nt), dtype=torch.float32, device=self.wlt.device)
        self.fm.ess_forward_members(encsrc, vels, hona)
        return hona, d

    def analyze(self, vels, codes, z=None):
        """One analysis: gain, then every member moved in place, the gain
        never leaving the device in between."""
        hona, d = self._encoded(vels, codes)
        t4, self.sigma, clip = enkf_analyze(hona, d, vels, self.fm.dx, self.fm.dt, z, self.sigfac, self.sigma,
                                            self.seed)
        self.seed += 1
        return t4, clip

    def createAMean(self, vels):
        import torch
        mean = torch.empty(vels.shape[1:], dtype=torch.float32, device=vels.device)
        enkf_mean(mean, vels)
        return mean


def regu_term(vel, lx: float, lz: float, stream=None) -> float:
    """ReguFactor::getReguTerm (src/unused/ReguFactor.cpp:19-27) of a CUDA
    model [nx][nz]: lx Wx2 + lz Wz2 (FP64 sums)."""
    nx, nz = vel.shape
    out = C.c_double()
    _check(lib().swfwi_regu_term(_ptr(vel), nx, nz, lx, lz, C.byref(out), _stream(stream)))
    return out.value


def regu_gradient(vel, lx: float, lz: float, grad, accumulate: bool = False, stream=None) -> None:
    """ReguFactor::getReguGradient (:67-108) into (or added to) grad."""
    nx, nz = vel.shape
    _check(lib().swfwi_regu_gradient(_ptr(vel), nx, nz, lx, lz, _ptr(grad), int(accumulate), _stream(stream)))


PRTM_ADJ_REFERENCE, PRTM_ADJ_EXACT = 0, 1


class Prtm2d:
    """The prestack LSRTM linear operator of src/unused/prtm2d.cpp on the GPU:
    the constructor is prtm2d_init (:241-338) with the velocity ``vel`` a
    CUDA [nx][nz] tensor (m/s), ``lop`` is prtm2d_lop (:354-437), ``close``
    prtm2d_close.  Unlike the reference's file-scope state, each object is
    its own operator.

    ``arith=ARITH_REF`` is bit-identical to the compiled reference (shots in
    order; the Born branch continues from the receiver-side fields the
    previous shot or call left, as the reference's does); ``ARITH_FAST``
    batches the shots in FP32 with FMA, every shot starting from zero.
    ``set_adjoint(PRTM_ADJ_EXACT)`` makes ``lop(adj=True)`` the exact
    transpose of the Born branch instead of the reference's migration, which
    is not its adjoint."""

    def __init__(self, vel, dz: float, dx: float, dt: float, amp: float, fm: float, nb: int, nt: int, ns: int,
                 ng: int, sxbeg: int, szbeg: int, jsx: int, jsz: int, gxbeg: int, gzbeg: int, jgx: int, jgz: int,
                 csdgather: bool = False, arith: int = ARITH_REF, stream=None):
        self.h = None
        nx, nz = vel.shape
        self.nx, self.nz, self.nt, self.ns, self.ng = nx, nz, nt, ns, ng
        h = _vp()
        _check(lib().swfwi_prtm2d_create(C.byref(h), arith, dz, dx, dt, amp, fm, nz, nx, nb, nt, ns, ng, sxbeg,
                                         szbeg, jsx, jsz, gxbeg, gzbeg, jgx, jgz, int(csdgather), _ptr(vel),
                                         _stream(stream)))
        self.h = h

    def set_adjoint(self, mode: int) -> None:
        _check(lib().swfwi_prtm2d_set_adjoint(self.h, mode))

    def set_graphs(self, on: bool) -> None:
        """Replay repeated calls (same arrays, direction, mode) as CUDA graphs."""
        _check(lib().swfwi_prtm2d_set_graphs(self.h, int(bool(on))))

    def batch(self) -> int:
        out = C.c_int()
        _check(lib().swfwi_prtm2d_batch(self.h, C.byref(out)))
        return out.value

    def lop(self, adj: bool, add: bool, mod, dat, stream=None) -> None:
        """adj False: dat (+)= L mod; adj True: mod (+)= L' dat.  mod CUDA
        float32 [nx][nz], dat CUDA float32 [ns][ng][nt]."""
        _check(lib().swfwi_prtm2d_lop(self.h, int(bool(adj)), int(bool(add)), mod.numel(), dat.numel(),
                                      _ptr(mod), _ptr(dat), _stream(stream)))

    def close(self) -> None:
        if self.h is not None:
            _check(lib().swfwi_prtm2d_destroy(self.h))
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def cal_objective_static(r, out, stream=None) -> None:
    """Sums of squares of each row of r ([nslots][n] float32, CUDA) into out
    ([nslots] float64, CUDA) without allocating device memory."""
    import torch
    if not (isinstance(r, torch.Tensor) and r.is_cuda and r.dtype == torch.float32 and r.dim() == 2
            and r.is_contiguous()):
        raise SwfwiError(1, "r must be a contiguous 2-D float32 CUDA tensor")
    nslots, n = r.shape
    if not (isinstance(out, torch.Tensor) and out.is_cuda and out.dtype == torch.float64
            and out.is_contiguous() and out.numel() >= nslots):
        raise SwfwiError(1, "out must be a contiguous float64 CUDA tensor of at least nslots elements")
    _check(lib().swfwi_cal_objective_static(_ptr(r), n, nslots, _ptr(out), _stream(stream)))


# ---------------------------------------------------------------- propagator
class ShotPosition:
    """A regular line of points (src/common/shot-position.h)."""

    def __init__(self, szbeg: int, sxbeg: int, jsz: int, jsx: int, ns: int, nz: int):
        self.c = _ShotPos(szbeg, sxbeg, jsz, jsx, ns, nz)
        self.ns = ns

    def getx(self, i: int) -> int:
        return self.c.sxbeg + i * self.c.jsx

    def getz(self, i: int) -> int:
        return self.c.szbeg + i * self.c.jsz


class Damp4t10d:
    """The propagator (src/modeling/damp4t10d.h:18-87) on the GPU.

    Work is ordered on torch's current CUDA stream at construction time
    (``set_stream`` changes it)."""

    def __init__(self, all_src: ShotPosition, all_geo: ShotPosition, dt: float, dx: float, fm: float,
                 nb: int, nt: int, arith: int = ARITH_REF, stream=None):
        h = C.c_void_p()
        _check(lib().swfwi_damp4t10d_create(C.byref(h), C.byref(all_src.c), C.byref(all_geo.c), dt, dx,
                                            fm, nb, nt))
        self.h = h
        self.src, self.geo = all_src, all_geo
        self.dt, self.dx, self.fm, self.nb, self.nt = dt, dx, fm, nb, nt
        self.ns, self.ng = all_src.ns, all_geo.ns
        self._vel = None
        self.set_stream(stream)
        self.set_arith(arith)

    def __del__(self):
        try:
            if getattr(self, "h", None):
                lib().swfwi_damp4t10d_destroy(self.h)
                self.h = None
        except Exception:
            pass

    @classmethod
    def from_survey(cls, s, **kw) -> "Damp4t10d":
        src = ShotPosition(s.szbeg, s.sxbeg, s.jsz, s.jsx, s.ns, s.nz)
        geo = ShotPosition(s.gzbeg, s.gxbeg, s.jgz, s.jgx, s.ng, s.nz)
        m = cls(src, geo, s.dt, s.dx, s.fm, s.nb, s.nt, **kw)
        m.setModelSize(s.nx, s.nz)
        if s.spreads is not None:
            m.setReceiversPerShot(*s.spreads)
        return m

    def set_stream(self, stream=None):
        self.stream = _stream(stream)
        _check(lib().swfwi_damp4t10d_set_stream(self.h, self.stream))

    def set_arith(self, arith: int):
        _check(lib().swfwi_damp4t10d_set_arith(self.h, arith))
        self.arith = arith

    def set_fusion(self, on: bool):
        """Fused backward time loop (source subtraction and imaging in the
        source back-step, residual injection in the receiver step)."""
        _check(lib().swfwi_damp4t10d_set_fusion(self.h, int(bool(on))))

    def set_graphs(self, on):
        """CUDA graphs for the forward/backward time loops: False/0 never,
        True/1 for small (launch-bound) steps, 2 for every step size."""
        _check(lib().swfwi_damp4t10d_set_graphs(self.h, int(on)))

    def set_strip_format(self, fmt: int):
        """Boundary strips of the gradients: STRIP_F32 (exact), STRIP_F16 or
        STRIP_BF16 (scaled 16-bit)."""
        _check(lib().swfwi_damp4t10d_set_strip_format(self.h, fmt))

    def set_reconstruction(self, mode: int, every: int = 64, fmt: int = STRIP_F32):
        """Source-field reconstruction in the gradients' backward sweep:
        RECON_STRIPS (back-propagation with boundary strips, the reference's
        method) or RECON_SNAPSHOTS (checkpoint snapshots of both fields every
        `every` steps in `fmt`, each segment re-run forward in the backward
        sweep)."""
        _check(lib().swfwi_damp4t10d_set_reconstruction(self.h, mode, every, fmt))

    def set_tuning(self, kernel: int = 6, band_depth: int = 120, rows_per_cta: int = 0,
                   rows_in_flight: int = 3, shots_slowest: bool = False):
        """Launch shape of the stencil (results do not change)."""
        _check(lib().swfwi_damp4t10d_set_tuning(self.h, kernel, band_depth, rows_per_cta, rows_in_flight,
                                                int(shots_slowest)))

    def setReceiversPerShot(self, offsets, gx, gz):
        o = np.ascontiguousarray(offsets, np.int32)
        x = np.ascontiguousarray(gx, np.int32)
        z = np.ascontiguousarray(gz, np.int32)
        _check(lib().swfwi_damp4t10d_set_receivers_per_shot(self.h, o.ctypes.data_as(_ip),
                                                            x.ctypes.data_as(_ip), z.ctypes.data_as(_ip)))

    def setModelSize(self, nx: int, nz: int):
        _check(lib().swfwi_damp4t10d_set_model_size(self.h, nx, nz))

    def dims(self):
        v = [C.c_int() for _ in range(5)]
        _check(lib().swfwi_damp4t10d_dims(self.h, *[C.byref(x) for x in v]))
        return tuple(x.value for x in v)   # nxpad, nzpad, ns, ngmax, nt

    def getnx(self):
        return self.dims()[0]

    def getnz(self):
        return self.dims()[1]

    def getng(self):
        return self.dims()[3]

    def expandDomain(self, vel: np.ndarray) -> np.ndarray:
        """Host [nx][nz] m/s -> host [nxpad][nzpad] transformed."""
        v, vp = _host_f32(vel)
        nx, nz = v.shape
        out = np.zeros((nx + 2 * self.nb + 12, nz + self.nb + 12), np.float32)
        _check(lib().swfwi_damp4t10d_expand_domain(self.h, vp, nx, nz, out.ctypes.data_as(_fp)))
        return out

    def bindVelocity(self, exvel):
        self._vel = exvel   # keep it alive: the library holds the pointer
        _check(lib().swfwi_damp4t10d_bind_velocity(self.h, _ptr(exvel)))

    def stepForward(self, p0, p1):
        _check(lib().swfwi_damp4t10d_step_forward(self.h, _ptr(p0), _ptr(p1)))

    def stepBackward(self, p0, p1):
        _check(lib().swfwi_damp4t10d_step_backward(self.h, _ptr(p0), _ptr(p1)))

    def addSource(self, p, source, shot_id: int = -1):
        _check(lib().swfwi_damp4t10d_add_source(self.h, _ptr(p), _ptr(source), shot_id))

    def subSource(self, p, source, shot_id: int = -1):
        _check(lib().swfwi_damp4t10d_sub_source(self.h, _ptr(p), _ptr(source), shot_id))

    def addEncodedSource(self, p, encsrc_it):
        self.addSource(p, encsrc_it, -1)

    def subEncodedSource(self, p, encsrc_it):
        self.subSource(p, encsrc_it, -1)

    def addReceiverSource(self, p, vsrc_it):
        _check(lib().swfwi_damp4t10d_add_receiver_source(self.h, _ptr(p), _ptr(vsrc_it)))

    def recordSeis(self, seis_it, p):
        _check(lib().swfwi_damp4t10d_record_seis(self.h, _ptr(seis_it), _ptr(p)))

    def bndrySize(self) -> int:
        n = C.c_int()
        _check(lib().swfwi_damp4t10d_bndry_size(self.h, C.byref(n)))
        return n.value

    def initBndryVector(self, nt: int):
        import torch
        return torch.zeros(nt * self.bndrySize(), dtype=torch.float32, device="cuda")

    def writeBndry(self, bndr, p, it: int):
        _check(lib().swfwi_damp4t10d_write_bndry(self.h, _ptr(bndr), _ptr(p), it))

    def readBndry(self, bndr, p, it: int):
        _check(lib().swfwi_damp4t10d_read_bndry(self.h, _ptr(bndr), _ptr(p), it))

    def maskGradient(self, g):
        _check(lib().swfwi_damp4t10d_mask_gradient(self.h, _ptr(g)))

    def scaleGradient(self, g):
        _check(lib().swfwi_damp4t10d_scale_gradient(self.h, _ptr(g)))

    def refillBoundary(self, v):
        _check(lib().swfwi_damp4t10d_refill_boundary(self.h, _ptr(v)))

    def removeDirectArrival(self, data):
        _check(lib().swfwi_damp4t10d_remove_direct_arrival(self.h, _ptr(data), -1))

    def fwiRemoveDirectArrival(self, data, shot_id: int):
        _check(lib().swfwi_damp4t10d_remove_direct_arrival(self.h, _ptr(data), shot_id))

    def FwiForwardModeling(self, wlt, dcal, shot_id: int):
        _check(lib().swfwi_damp4t10d_fwi_forward_modeling(self.h, _ptr(wlt), _ptr(dcal), shot_id))

    def EssForwardModeling(self, encsrc, dcal):
        _check(lib().swfwi_damp4t10d_ess_forward_modeling(self.h, _ptr(encsrc), _ptr(dcal)))

    def ess_forward_members(self, encsrc, vels, hona):
        """EssForwardModeling with each member velocity (vels [n][nxpad][nzpad]
        CUDA) into hona [n][ng*nt] in the analysis matrix's row order."""
        _check(lib().swfwi_damp4t10d_ess_forward_members(self.h, _ptr(encsrc), _ptr(vels), vels.shape[0],
                                                         _ptr(hona)))

    # ---- batched ----
    def forward_batch(self, wlt, dcal, shot_ids):
        ids = np.ascontiguousarray(shot_ids, np.int32)
        _check(lib().swfwi_damp4t10d_forward_batch(self.h, _ptr(wlt), _ptr(dcal), ids.ctypes.data_as(_ip),
                                                   ids.size))

    def gradient_batch(self, wlt, dobs, shot_ids, grad) -> np.ndarray:
        ids = np.ascontiguousarray(shot_ids, np.int32)
        obj = np.zeros(ids.size, np.float64)
        _check(lib().swfwi_damp4t10d_gradient_batch(self.h, _ptr(wlt), _ptr(dobs), ids.ctypes.data_as(_ip),
                                                    ids.size, _ptr(grad), obj.ctypes.data_as(_dp)))
        return obj

    def gradient_host(self, exvel: np.ndarray, wlt: np.ndarray, dobs: np.ndarray, shot_ids,
                      grad_out: np.ndarray | None = None):
        """The batched gradient from host buffers (copies in and out)."""
        ids = np.ascontiguousarray(shot_ids, np.int32)
        v, vp = _host_f32(exvel)
        w, wp = _host_f32(wlt)
        d, dp = _host_f32(dobs)
        g = grad_out if grad_out is not None else np.zeros_like(v)
        obj = np.zeros(ids.size, np.float64)
        _check(lib().swfwi_gradient_host(self.h, vp, wp, dp, ids.ctypes.data_as(_ip), ids.size,
                                         g.ctypes.data_as(_fp), obj.ctypes.data_as(_dp)))
        return g, obj

    def calgradient_ess(self, encsrc, vsrc, grad):
        _check(lib().swfwi_damp4t10d_calgradient_ess(self.h, _ptr(encsrc), _ptr(vsrc), _ptr(grad)))

    def calgradient_fwi(self, wlt, vsrc, grad, shot_id: int):
        _check(lib().swfwi_damp4t10d_calgradient_fwi(self.h, _ptr(wlt), _ptr(vsrc), _ptr(grad), shot_id))

    def calgradient_fwi_f64(self, vel, wlt64, vsrc64, grad64, shot_id: int):
        _check(lib().swfwi_damp4t10d_calgradient_fwi_f64(self.h, _ptr(vel), _ptr(wlt64), _ptr(vsrc64),
                                                         _ptr(grad64), shot_id))

    def calgradient_ess_f64(self, vel, encsrc64, vsrc64, grad64):
        _check(lib().swfwi_damp4t10d_calgradient_ess_f64(self.h, _ptr(vel), _ptr(encsrc64), _ptr(vsrc64),
                                                         _ptr(grad64)))

    def FwiForwardModeling_f64(self, vel, wlt64, dcal64, shot_id: int):
        _check(lib().swfwi_damp4t10d_fwi_forward_modeling_f64(self.h, _ptr(vel), _ptr(wlt64), _ptr(dcal64),
                                                              shot_id))


class _Framework:
    encoded = 0

    def __init__(self, method: Damp4t10d, exvel: np.ndarray, vmin: float, vmax: float, nita: int,
                 maxdv: float, wlt: np.ndarray, dobs: np.ndarray):
        v, vp = _host_f32(exvel)
        w, wp = _host_f32(wlt)
        d, dp = _host_f32(dobs)
        h = C.c_void_p()
        _check(lib().swfwi_fwi_create(C.byref(h), method.h, vp, vmin, vmax, nita, maxdv, wp, dp,
                                      self.encoded))
        self.h = h
        self.method = method
        self.shape = v.shape

    def __del__(self):
        try:
            if getattr(self, "h", None):
                lib().swfwi_fwi_destroy(self.h)
                self.h = None
        except Exception:
            pass

    def epoch(self, it: int):
        _check(lib().swfwi_fwi_epoch(self.h, it))

    def getUpdateObj(self) -> float:
        o = C.c_float()
        _check(lib().swfwi_fwi_get_update_obj(self.h, C.byref(o)))
        return o.value

    def getInitObj(self) -> float:
        o = C.c_float()
        _check(lib().swfwi_fwi_get_init_obj(self.h, C.byref(o)))
        return o.value

    def velocity(self) -> np.ndarray:
        out = np.zeros(self.shape, np.float32)
        _check(lib().swfwi_fwi_get_velocity(self.h, out.ctypes.data_as(_fp)))
        return out

    def setVelocity(self, exvel: np.ndarray):
        v, vp = _host_f32(exvel)
        _check(lib().swfwi_fwi_set_velocity(self.h, vp))

    def writeVel(self) -> np.ndarray:
        nxpad, nzpad = self.shape
        nb = self.method.nb
        out = np.zeros((nxpad - 2 * nb - 12, nzpad - nb - 12), np.float32)
        _check(lib().swfwi_fwi_write_vel(self.h, out.ctypes.data_as(_fp)))
        return out

    # ---- learned preconditioner (plain FWI only) ----
    def setPreconditioner(self, net):
        """Attach a swfwi_b200.precond.Preconditioner (None detaches)."""
        _check(lib().swfwi_fwi_set_preconditioner(self.h, net.h if net is not None else None))
        self._net = net     # keep it alive while attached

    def setLearnedMinDecrease(self, frac: float):
        """Keep a learned step only if it lowers the objective by at least
        this fraction (default 0)."""
        _check(lib().swfwi_fwi_set_learned_min_decrease(self.h, frac))

    def setLearnedPatience(self, rejections: int):
        """Stop proposing learned steps after this many rejections (0: never)."""
        _check(lib().swfwi_fwi_set_learned_patience(self.h, rejections))

    def collectIllumination(self, on: bool = True):
        _check(lib().swfwi_fwi_collect_illumination(self.h, int(on)))

    def gradient(self) -> np.ndarray:
        out = np.zeros(self.shape, np.float32)
        _check(lib().swfwi_fwi_get_gradient(self.h, out.ctypes.data_as(_fp)))
        return out

    def illumination(self) -> np.ndarray:
        out = np.zeros(self.shape, np.float32)
        _check(lib().swfwi_fwi_get_illumination(self.h, out.ctypes.data_as(_fp)))
        return out

    def learnedStats(self):
        """(last epoch took the network's step, tried, accepted)."""
        a, b, c = C.c_int(), C.c_int(), C.c_int()
        _check(lib().swfwi_fwi_learned_stats(self.h, C.byref(a), C.byref(b), C.byref(c)))
        return bool(a.value), b.value, c.value

    def lastLineSearch(self):
        a = np.zeros(4, np.float32)
        o = np.zeros(4, np.float32)
        _check(lib().swfwi_fwi_last_line_search(self.h, a.ctypes.data_as(_fp), o.ctypes.data_as(_fp)))
        return a, o

    def lastTrials(self) -> int:
        """Trial objectives (forward sweeps) of the last epoch's step search."""
        n = C.c_int()
        _check(lib().swfwi_fwi_last_trials(self.h, C.byref(n)))
        return n.value


class FwiFramework(_Framework):
    """Plain per-shot FWI (src/fwi/fwiframework.h)."""
    encoded = 0


class EssFwiFramework(_Framework):
    """Encoded simultaneous-source FWI (src/essfwi/essfwiframework.h)."""
    encoded = 1

    def setRegularization(self, lambda_x: float, lambda_z: float):
        """EssFwiRegu (src/unused/essfwiregu.h): epochs with the first-difference
        regularisation lx Wx2 + lz Wz2 (0, 0: the plain encoded epoch)."""
        _check(lib().swfwi_fwi_set_regularization(self.h, lambda_x, lambda_z))
