"""RSF (Madagascar) file I/O through the C ABI, on the CPU: round trips,
headers written the way Madagascar writes them (history lines, repeated
keys, quoted values, embedded data), the shot layout the reference's
ShotDataReader expects, and errors."""
import os

import numpy as np
import pytest

import swfwi_b200 as S
from swfwi_b200 import rsf


def test_velocity_round_trip(tmp_path):
    v = np.random.default_rng(0).uniform(1500, 4700, (37, 23)).astype(np.float32)   # [nx][nz]
    p = str(tmp_path / "vel.rsf")
    rsf.write(p, v, d=[10.0, 10.0], o=[0.0, 0.0], extra={"label1": '"Depth"'})
    n, d, o = rsf.dims(p)
    assert n == [23, 37] and d == [10.0, 10.0] and o == [0.0, 0.0]   # n1 = nz, n2 = nx
    np.testing.assert_array_equal(rsf.read(p), v)
    assert rsf.get(p, "label1") == "Depth"
    assert rsf.get(p, "data_format") == "native_float"


def test_madagascar_style_header(tmp_path):
    data = np.arange(60, dtype=np.float32)
    (tmp_path / "x.rsf@").write_bytes(data.tobytes())
    (tmp_path / "x.rsf").write_text(
        'sfspike n1=5 n2=3 mag=1\n'
        '\tn1=4 n2=3 d1=0.004 o1=0\n'
        'sfput label1="Time (s)" n3=5\n'
        '\tin="x.rsf@"\n\tesize=4 data_format="native_float"\n'
        'sfwindow n1=4\n')
    p = str(tmp_path / "x.rsf")
    n, d, o = rsf.dims(p)
    assert n == [4, 3, 5] and abs(d[0] - 0.004) < 1e-9
    assert rsf.get(p, "label1") == "Time (s)"
    np.testing.assert_array_equal(rsf.read(p), data.reshape(5, 3, 4))


def test_embedded_binary(tmp_path):
    data = np.linspace(-1, 1, 12).astype(np.float32)
    p = tmp_path / "e.rsf"
    p.write_bytes(b'\tn1=6 n2=2\n\tin="stdin"\n\tesize=4\n\tdata_format="native_float"\n\x0c\x0c\x04'
                  + data.tobytes())
    np.testing.assert_array_equal(rsf.read(str(p)), data.reshape(2, 6))


def test_shots_layout_matches_shot_reader(tmp_path):
    rng = np.random.default_rng(1)
    dobs = rng.standard_normal((3, 11, 7)).astype(np.float32)       # [ns][nt][ng]
    p = str(tmp_path / "shots.rsf")
    rsf.write_shots(p, dobs, dt=0.001, dgx=10.0, extra={"fm": 15, "szbeg": 6, "nb": 30})
    assert rsf.dims(p)[0] == [11, 7, 3]                              # n1=nt, n2=ng, n3=ns
    disk = np.fromfile(p + "@", np.float32).reshape(3, 7, 11)        # [is][ig][it]
    np.testing.assert_array_equal(disk, dobs.transpose(0, 2, 1))
    np.testing.assert_array_equal(rsf.read_shots(p, 3, 11, 7), dobs)
    assert rsf.get(p, "label3") == "Shot" and rsf.get(p, "fm") == "15" and rsf.get(p, "nb") == "30"


def test_errors(tmp_path):
    with pytest.raises(S.SwfwiError) as e:
        rsf.read(str(tmp_path / "missing.rsf"))
    assert e.value.status == 1
    (tmp_path / "b.rsf").write_text('\tn1=4\n\tin="b.rsf@"\n\tesize=2\n\tdata_format="native_short"\n')
    (tmp_path / "b.rsf@").write_bytes(b"\0" * 8)
    with pytest.raises(S.SwfwiError):
        rsf.read(str(tmp_path / "b.rsf"))
    (tmp_path / "c.rsf").write_text('\tn1=40\n\tin="c.rsf@"\n')
    (tmp_path / "c.rsf@").write_bytes(b"\0" * 8)                      # shorter than n1 says
    with pytest.raises(S.SwfwiError):
        rsf.read(str(tmp_path / "c.rsf"))
