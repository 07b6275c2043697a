"""RSF (Madagascar) files through the library's C ABI: the reference tools'
file boundary (velocities n1=nz n2=nx; shots n1=nt n2=ng n3=ns)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _check, lib

_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int)


def _b(s):
    return s.encode() if isinstance(s, str) else s


def get(path: str, key: str) -> str:
    buf = C.create_string_buffer(4096)
    _check(lib().swfwi_rsf_get(_b(path), _b(key), buf, len(buf)))
    return buf.value.decode()


def dims(path: str):
    """(n, d, o) of the axes up to the last one longer than 1."""
    nd = C.c_int()
    n = np.zeros(9, np.int32)
    d = np.zeros(9, np.float32)
    o = np.zeros(9, np.float32)
    _check(lib().swfwi_rsf_dims(_b(path), C.byref(nd), n.ctypes.data_as(_ip), d.ctypes.data_as(_fp),
                                o.ctypes.data_as(_fp)))
    k = max(nd.value, 1)
    return n[:k].tolist(), d[:k].tolist(), o[:k].tolist()


def read(path: str) -> np.ndarray:
    """The whole array, shaped with axis 1 last (numpy C order)."""
    n, _, _ = dims(path)
    out = np.zeros(int(np.prod(n)), np.float32)
    _check(lib().swfwi_rsf_read(_b(path), out.ctypes.data_as(_fp), out.size, 0))
    return out.reshape(list(reversed(n)))


def write(path: str, data: np.ndarray, d=None, o=None, extra: dict | None = None, data_path: str | None = None):
    """data in numpy C order: its last axis is RSF axis 1."""
    a = np.ascontiguousarray(data, np.float32)
    n = np.array(list(reversed(a.shape)), np.int32)
    dd = None if d is None else np.ascontiguousarray(d, np.float32)
    oo = None if o is None else np.ascontiguousarray(o, np.float32)
    ex = "".join(f"\t{k}={v}\n" for k, v in (extra or {}).items())
    _check(lib().swfwi_rsf_write(_b(path), _b(data_path) if data_path else None, a.ctypes.data_as(_fp),
                                 len(n), n.ctypes.data_as(_ip),
                                 dd.ctypes.data_as(_fp) if dd is not None else None,
                                 oo.ctypes.data_as(_fp) if oo is not None else None, _b(ex)))


def read_shots(path: str, ns: int, nt: int, ng: int) -> np.ndarray:
    """[ns][nt][ng] (ShotDataReader::serialRead)."""
    out = np.zeros((ns, nt, ng), np.float32)
    _check(lib().swfwi_rsf_read_shots(_b(path), out.ctypes.data_as(_fp), ns, nt, ng))
    return out


def write_shots(path: str, dobs: np.ndarray, dt: float, dgx: float, extra: dict | None = None,
                data_path: str | None = None):
    a = np.ascontiguousarray(dobs, np.float32)
    ns, nt, ng = a.shape
    ex = "".join(f"\t{k}={v}\n" for k, v in (extra or {}).items())
    _check(lib().swfwi_rsf_write_shots(_b(path), _b(data_path) if data_path else None, a.ctypes.data_as(_fp),
                                       ns, nt, ng, dt, dgx, _b(ex)))
