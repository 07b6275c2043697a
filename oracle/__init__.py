"""The oracle: test infrastructure only.

CPU checkers for swfwi's acoustic FWI path, loaded with ctypes:

* ``RefLib`` wraps ``oracle/_ref/libswfwi_ref.so``: the reference's own C/C++
  sources (src/modeling, src/common, src/essfwi, src/fwi) compiled in place
  by ``oracle/Makefile`` plus the harness translation units in this folder.
* ``FdOracle`` wraps ``oracle/_ref/libfd_oracle.so``: a plain-C restatement of
  the stencil (reference arithmetic and FP64) and an FP64 restatement of the
  per-shot forward modelling and gradient (``oracle/fd_oracle.c``).
* ``PrtmRef`` wraps ``oracle/_ref/libprtm_ref.so``: the reference's LSRTM
  operator (src/unused/prtm2d.cpp) compiled in place by ``harness_prtm.cpp``.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg may import this package, and only as the checker or the timed CPU
baseline, never as the product path.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
_fp = C.POINTER(C.c_float)
_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


def reference_tree() -> str | None:
    """The reference checkout the oracle recipe compiles (``oracle/Makefile``
    decides: REF, else $SWFWI_REFERENCE, else its default); None when that
    tree is absent, as on a machine that only runs the prebuilt oracle."""
    try:
        out = subprocess.run(["make", "-s", "-C", HERE, "print-ref"], check=True, capture_output=True,
                             text=True).stdout.strip()
    except (OSError, subprocess.CalledProcessError):
        return None
    return out if out and os.path.isdir(os.path.join(out, "src")) else None


def build(reference: str | None = None) -> None:
    """Compile the oracle libraries (needs the reference tree; run where it exists)."""
    cmd = ["make", "-C", HERE, "-j8"]
    if reference:
        cmd.append(f"REF={reference}")
    subprocess.run(cmd, check=True, stdout=subprocess.DEVNULL)


def available() -> bool:
    return os.path.exists(os.path.join(REF_DIR, "libswfwi_ref.so"))


def fptr(a: np.ndarray):
    assert a.dtype == np.float32 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_fp)


def dptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_dp)


def iptr(a: np.ndarray):
    assert a.dtype == np.int32 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_ip)


class RefLib:
    """The compiled reference (``asbuilt=True``: pass 1 of the damped kernel
    serial, as the reference's SConscript builds it)."""

    def __init__(self, asbuilt: bool = False):
        name = "libswfwi_ref_asbuilt.so" if asbuilt else "libswfwi_ref.so"
        self.lib = C.CDLL(os.path.join(REF_DIR, name))
        L = self.lib
        L.ref_quiet()
        L.ref_model_create.restype = C.c_void_p
        L.ref_model_create.argtypes = [C.c_int] * 4 + [C.c_float] * 3 + [C.c_int] * 10
        for fn in ("ref_model_destroy",):
            getattr(L, fn).argtypes = [C.c_void_p]
        vp = C.c_void_p
        sig = {
            "ref_expand_domain": [vp, _fp, _fp],
            "ref_bind_velocity": [vp, _fp],
            "ref_get_velocity": [vp, _fp],
            "ref_fwi_forward": [vp, _fp, _fp, C.c_int],
            "ref_ess_forward": [vp, _fp, _fp],
            "ref_remove_direct_arrival": [vp, _fp, C.c_int],
            "ref_trans_vsrc": [_fp, C.c_int, C.c_int],
            "ref_calgradient_ess": [vp, _fp, _fp, _fp],
            "ref_calgradient_fwi": [vp, _fp, _fp, _fp, C.c_int],
            "ref_scale_gradient": [vp, _fp],
            "ref_mask_gradient": [vp, _fp],
            "ref_refill_boundary": [vp, _fp],
            "ref_write_bndry": [vp, _fp, _fp, C.c_int],
            "ref_read_bndry": [vp, _fp, _fp, C.c_int],
            "ref_bndry_size": [vp],
            "ref_add_source": [vp, _fp, _fp, C.c_int],
            "ref_sub_source": [vp, _fp, _fp, C.c_int],
            "ref_add_receiver_source": [vp, _fp, _fp],
            "ref_record_seis": [vp, _fp, _fp],
            "ref_step_forward": [vp, _fp, _fp],
            "ref_step_backward": [vp, _fp, _fp],
            "ref_update_grad": [_fp, _fp, _fp, C.c_int, C.c_int],
            "ref_cal_objective": [_fp, C.c_int],
            "ref_parabola_vertex": [C.c_float] * 7 + [_fp, _fp],
            "ref_ricker": [_fp, C.c_int, C.c_float, C.c_float, C.c_float],
            "ref_regu": [_fp, C.c_int, C.c_int, C.c_float, C.c_float, _fp, _fp],
            "ref_random_codes": [C.c_int, C.c_int, C.c_int, _ip],
            "ref_ess_fwi_run": [vp, _fp, _fp, C.c_int, C.c_int, C.c_float, C.c_float, C.c_float, _fp, _fp],
            "ref_fwi_run": [vp, _fp, _fp, C.c_int, C.c_int, C.c_float, C.c_float, C.c_float, _fp, _fp],
            "ref_fwi_gradient": [vp, _fp, _fp, _fp, _fp],
            "ref_cal_max_alpha": [vp, _fp, C.c_float, _fp, _fp],
            "ref_update_vel": [vp, _fp, _fp, _fp, C.c_float, C.c_float, C.c_float],
            "fd4t10s_damp_zjh_2d_vtrans": [_fp, _fp, _fp, _fp, C.c_int, C.c_int, C.c_int],
            "fd4t10s_zjh_2d_vtrans": [_fp, _fp, _fp, _fp, C.c_int, C.c_int],
            "ref_clip_position": [_dp, C.c_int],
            "ref_a_plus_b": [_dp, _dp, _dp, C.c_int],
        }
        for k, v in sig.items():
            getattr(L, k).argtypes = v
        L.ref_cal_objective.restype = C.c_float
        L.ref_bndry_size.restype = C.c_int

    # --- raw kernels (src/modeling/fd4t10s-*.c) ---
    def step(self, prev, curr, vel, nb: int | None):
        """One reference step in place over ``prev`` ([nx][nz] float32)."""
        nx, nz = prev.shape
        u2 = np.zeros_like(prev)
        if nb is None:
            self.lib.fd4t10s_zjh_2d_vtrans(fptr(prev), fptr(curr), fptr(vel), fptr(u2), nx, nz)
        else:
            self.lib.fd4t10s_damp_zjh_2d_vtrans(fptr(prev), fptr(curr), fptr(vel), fptr(u2), nx, nz, nb)

    def trans_vsrc(self, vsrc):
        v = np.ascontiguousarray(vsrc, dtype=np.float32).copy()
        nt, ng = v.shape
        self.lib.ref_trans_vsrc(fptr(v), nt, ng)
        return v

    def cal_objective(self, r):
        r = np.ascontiguousarray(r, dtype=np.float32).ravel()
        return float(self.lib.ref_cal_objective(fptr(r), r.size))

    def update_grad(self, pre, cur, direction, it):
        pre = pre.copy(); direction = direction.copy()
        cur = np.ascontiguousarray(cur, dtype=np.float32)
        self.lib.ref_update_grad(fptr(pre), fptr(cur), fptr(direction), cur.size, it)
        return pre, direction

    def parabola_vertex(self, x1, y1, x2, y2, x3, y3, maxa3):
        a = np.zeros(1, np.float32); b = np.zeros(1, np.float32)
        self.lib.ref_parabola_vertex(x1, y1, x2, y2, x3, y3, maxa3, fptr(a), fptr(b))
        return float(a[0]), float(b[0])

    def clip_position(self, s) -> int:
        """clipPosition (src/enfwi/Matrix.cpp:170-185), compiled."""
        s = np.ascontiguousarray(s, np.float64)
        return int(self.lib.ref_clip_position(s.ctypes.data_as(_dp), s.size))

    def a_plus_b(self, a, b):
        a = np.ascontiguousarray(a, np.float64)
        b = np.ascontiguousarray(b, np.float64)
        c = np.zeros_like(a)
        self.lib.ref_a_plus_b(a.ctypes.data_as(_dp), b.ctypes.data_as(_dp), c.ctypes.data_as(_dp), a.size)
        return c

    def ricker(self, nt, fm, dt, amp=1.0):
        w = np.zeros(nt, np.float32)
        self.lib.ref_ricker(fptr(w), nt, fm, dt, amp)
        return w

    def regu(self, vel: np.ndarray, lx: float, lz: float):
        """ReguFactor (src/unused/ReguFactor.cpp) on vel [nx][nz]: (term,
        gradient [nx][nz])."""
        v = np.ascontiguousarray(vel, np.float32)
        nx, nz = v.shape
        term = np.zeros(1, np.float32)
        g = np.zeros_like(v)
        self.lib.ref_regu(fptr(v), nx, nz, lx, lz, fptr(term), fptr(g))
        return float(term[0]), g

    def random_codes(self, seed, ns, skip=0):
        c = np.zeros(ns, np.int32)
        self.lib.ref_random_codes(seed, skip, ns, iptr(c))
        return c

    def model(self, geom) -> "RefModel":
        return RefModel(self, geom)


class RefModel:
    """A reference Damp4t10d set-up for one ``swfwi_b200.geometry.Survey``-like
    object with regular source/receiver lines (attributes nz, nx, nb, nt, dt,
    dx, fm, szbeg, sxbeg, jsz, jsx, ns, gzbeg, gxbeg, jgz, jgx, ng)."""

    def __init__(self, ref: RefLib, g):
        self.ref, self.g = ref, g
        L = ref.lib
        self.h = C.c_void_p(L.ref_model_create(g.nz, g.nx, g.nb, g.nt, g.dt, g.dx, g.fm,
                                              g.szbeg, g.sxbeg, g.jsz, g.jsx, g.ns,
                                              g.gzbeg, g.gxbeg, g.jgz, g.jgx, g.ng))
        self.nxpad = g.nx + 2 * g.nb + 12
        self.nzpad = g.nz + g.nb + 12

    def __del__(self):
        try:
            self.ref.lib.ref_model_destroy(self.h)
        except Exception:
            pass

    def expand_domain(self, vel):
        v = np.ascontiguousarray(vel, dtype=np.float32)
        out = np.zeros((self.nxpad, self.nzpad), np.float32)
        self.ref.lib.ref_expand_domain(self.h, fptr(v), fptr(out))
        return out

    def bind_velocity(self, exvel):
        self.ref.lib.ref_bind_velocity(self.h, fptr(np.ascontiguousarray(exvel, dtype=np.float32)))

    def velocity(self):
        out = np.zeros((self.nxpad, self.nzpad), np.float32)
        self.ref.lib.ref_get_velocity(self.h, fptr(out))
        return out

    def fwi_forward(self, wlt, shot):
        d = np.zeros((self.g.nt, self.g.ng), np.float32)
        self.ref.lib.ref_fwi_forward(self.h, fptr(np.ascontiguousarray(wlt, np.float32)), fptr(d), shot)
        return d

    def ess_forward(self, encsrc):
        d = np.zeros((self.g.nt, self.g.ng), np.float32)
        self.ref.lib.ref_ess_forward(self.h, fptr(np.ascontiguousarray(encsrc, np.float32)), fptr(d))
        return d

    def remove_direct_arrival(self, data, shot):
        d = np.ascontiguousarray(data, np.float32).copy()
        self.ref.lib.ref_remove_direct_arrival(self.h, fptr(d), shot)
        return d

    def calgradient_fwi(self, wlt, vsrc, shot):
        g = np.zeros((self.nxpad, self.nzpad), np.float32)
        self.ref.lib.ref_calgradient_fwi(self.h, fptr(np.ascontiguousarray(wlt, np.float32)),
                                         fptr(np.ascontiguousarray(vsrc, np.float32)), fptr(g), shot)
        return g

    def calgradient_ess(self, encsrc, vsrc):
        g = np.zeros((self.nxpad, self.nzpad), np.float32)
        self.ref.lib.ref_calgradient_ess(self.h, fptr(np.ascontiguousarray(encsrc, np.float32)),
                                         fptr(np.ascontiguousarray(vsrc, np.float32)), fptr(g))
        return g

    def scale_gradient(self, g):
        g = g.copy(); self.ref.lib.ref_scale_gradient(self.h, fptr(g)); return g

    def mask_gradient(self, g):
        g = g.copy(); self.ref.lib.ref_mask_gradient(self.h, fptr(g)); return g

    def refill_boundary(self, v):
        v = v.copy(); self.ref.lib.ref_refill_boundary(self.h, fptr(v)); return v

    def bndry_size(self):
        return self.ref.lib.ref_bndry_size(self.h)

    def write_bndry(self, p, nt_slots=1, it=0, bndr=None):
        if bndr is None:
            bndr = np.zeros(nt_slots * self.bndry_size(), np.float32)
        self.ref.lib.ref_write_bndry(self.h, fptr(bndr), fptr(p), it)
        return bndr

    def read_bndry(self, bndr, p, it=0):
        self.ref.lib.ref_read_bndry(self.h, fptr(bndr), fptr(p), it)

    def fwi_gradient(self, wlt, dobs):
        g = np.zeros((self.nxpad, self.nzpad), np.float32)
        obj = np.zeros(1, np.float32)
        self.ref.lib.ref_fwi_gradient(self.h, fptr(np.ascontiguousarray(wlt, np.float32)),
                                      fptr(np.ascontiguousarray(dobs, np.float32)), fptr(g), fptr(obj))
        return g, float(obj[0])

    def cal_max_alpha(self, grad, maxdv):
        a = np.zeros(1, np.float32); b = np.zeros(1, np.float32)
        self.ref.lib.ref_cal_max_alpha(self.h, fptr(np.ascontiguousarray(grad, np.float32)), maxdv, fptr(a), fptr(b))
        return float(a[0]), float(b[0])

    def update_vel(self, v, d, steplen, vmin, vmax):
        out = np.zeros_like(v)
        self.ref.lib.ref_update_vel(self.h, fptr(out), fptr(np.ascontiguousarray(v, np.float32)),
                                    fptr(np.ascontiguousarray(d, np.float32)), steplen, vmin, vmax)
        return out

    def fwi_run(self, wlt, dobs, niter, nita, maxdv, vmin, vmax):
        out = np.zeros((self.nxpad, self.nzpad), np.float32)
        objs = np.zeros(3 * niter, np.float32)
        self.ref.lib.ref_fwi_run(self.h, fptr(np.ascontiguousarray(wlt, np.float32)),
                                 fptr(np.ascontiguousarray(dobs, np.float32)), niter, nita, maxdv,
                                 vmin, vmax, fptr(out), fptr(objs))
        return out, objs.reshape(niter, 3)

    def ess_fwi_run(self, wlt, dobs, niter, nita, maxdv, vmin, vmax):
        out = np.zeros((self.nxpad, self.nzpad), np.float32)
        objs = np.zeros(2 * niter, np.float32)
        self.ref.lib.ref_ess_fwi_run(self.h, fptr(np.ascontiguousarray(wlt, np.float32)),
                                     fptr(np.ascontiguousarray(dobs, np.float32)), niter, nita, maxdv,
                                     vmin, vmax, fptr(out), fptr(objs))
        return out, objs.reshape(niter, 2)


class FdOracle:
    """The plain-C restatement (``oracle/fd_oracle.c``)."""

    def __init__(self):
        self.lib = C.CDLL(os.path.join(REF_DIR, "libfd_oracle.so"))
        L = self.lib
        L.fdo_step_ref.argtypes = [_fp, _fp, _fp, C.c_int, C.c_int, C.c_int, C.c_int]
        L.fdo_step_f64.argtypes = [_dp, _dp, _dp, C.c_int, C.c_int, C.c_int, C.c_int]
        L.fdo_forward_f64.argtypes = [_dp, C.c_int, C.c_int, C.c_int, C.c_int, _dp, C.c_int, _ip, C.c_int, _dp]
        L.fdo_gradient_f64.argtypes = [_dp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, _dp, C.c_int,
                                       _ip, C.c_int, _dp, _dp]
        L.fdo_strip_size.argtypes = [C.c_int] * 3
        L.fdo_strip_size.restype = C.c_int

    def step_ref(self, prev, curr, vel, nb, damped=True):
        nx, nz = prev.shape
        self.lib.fdo_step_ref(fptr(prev), fptr(curr), fptr(vel), nx, nz, nb, int(damped))

    def step_f64(self, prev, curr, vel, nb, damped=True):
        nx, nz = prev.shape
        self.lib.fdo_step_f64(dptr(prev), dptr(curr), dptr(vel), nx, nz, nb, int(damped))

    def forward_f64(self, vel, bx0, nt, wlt, src_pos, rec_pos):
        nx, nz = vel.shape
        rec = np.ascontiguousarray(rec_pos, np.int32)
        d = np.zeros((nt, rec.size), np.float64)
        self.lib.fdo_forward_f64(dptr(np.ascontiguousarray(vel, np.float64)), nx, nz, bx0, nt,
                                 dptr(np.ascontiguousarray(wlt, np.float64)), int(src_pos), iptr(rec), rec.size, dptr(d))
        return d

    def gradient_f64(self, vel, bx0, nt, dt, wlt, src_pos, rec_pos, vsrc):
        nx, nz = vel.shape
        rec = np.ascontiguousarray(rec_pos, np.int32)
        g = np.zeros((nx, nz), np.float64)
        self.lib.fdo_gradient_f64(dptr(np.ascontiguousarray(vel, np.float64)), nx, nz, bx0, nt, float(dt),
                                  dptr(np.ascontiguousarray(wlt, np.float64)), int(src_pos), iptr(rec), rec.size,
                                  dptr(np.ascontiguousarray(vsrc, np.float64)), dptr(g))
        return g


class PrtmRef:
    """The reference's LSRTM operator (src/unused/prtm2d.cpp, compiled in
    place into ``oracle/_ref/libprtm_ref.so`` by ``harness_prtm.cpp``).  The
    operator lives in file-scope variables, so one object at a time: the
    constructor is prtm2d_init (receiver-side fields cleared, which the
    reference leaves to malloc), ``close`` is prtm2d_close."""

    _open = False

    def __init__(self, vel, dz, dx, dt, amp, fm, nb, nt, ns, ng, sxbeg, szbeg, jsx, jsz, gxbeg, gzbeg, jgx, jgz,
                 csdgather=False):
        if PrtmRef._open:
            raise RuntimeError("the reference operator is a single instance: close the open one first")
        self.lib = C.CDLL(os.path.join(REF_DIR, "libprtm_ref.so"))
        L = self.lib
        L.ref_prtm_init.argtypes = [C.c_int] + [C.c_float] * 5 + [C.c_int] * 14 + [_fp]
        L.ref_prtm_lop.argtypes = [C.c_int] * 4 + [_fp, _fp]
        vel = np.ascontiguousarray(vel, np.float32)
        self.nx, self.nz = vel.shape
        self.nt, self.ns, self.ng = nt, ns, ng
        L.ref_prtm_init(int(csdgather), dz, dx, dt, amp, fm, self.nz, self.nx, nb, nt, ns, ng, sxbeg, szbeg, jsx, jsz,
                        gxbeg, gzbeg, jgx, jgz, fptr(vel))
        PrtmRef._open = True

    def lop(self, adj, add, mod, dat):
        """prtm2d_lop in place on float32 arrays mod [nx][nz], dat [ns][ng][nt]"""
        self.lib.ref_prtm_lop(int(bool(adj)), int(bool(add)), mod.size, dat.size, fptr(mod), fptr(dat))

    def clear(self):
        """zero the receiver-side fields (a per-shot operator's start)"""
        self.lib.ref_prtm_clear()

    def close(self):
        if PrtmRef._open:
            self.lib.ref_prtm_close()
            PrtmRef._open = False
