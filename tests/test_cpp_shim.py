"""The C++ classes in include/swfwi (the reference's ShotPosition, Velocity,
Damp4t10d, the update operators, FwiFramework, EssFwiFramework and
rickerWavelet, over the C ABI).  On CPU: a driver written in the form of the
reference's src/tool/main-fwi-damp.cpp (tests/cpp/fwi_driver.cpp) compiles
and links against them, and writeVel(sf_file) instantiates against an RSF
declaration.  On the GPU: the driver's two epochs of plain and encoded FWI
on the golden survey match the reference's own epochs (fixture), as the
Python mirror's do (tests/test_gpu_fwi.py)."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from tests.conftest import ROOT, golden, rel_l2
from tests.golden.make_golden import small_survey

CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
LIB = os.path.join(ROOT, "swfwi_b200")


def _compile(src, out, link=True):
    if not shutil.which("g++") or not os.path.exists(os.path.join(CUDA, "include", "cuda_runtime_api.h")):
        pytest.skip("no g++ or CUDA headers")
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include", "swfwi"),
           "-I", os.path.join(CUDA, "include"), src, "-o", out]
    if link:
        if not os.path.exists(os.path.join(LIB, "libswfwi_b200.so")):
            pytest.skip("library not built")
        cmd += ["-L", LIB, "-lswfwi_b200", "-L", os.path.join(CUDA, "lib64"), "-lcudart", "-Wl,-rpath," + LIB]
    else:
        cmd.insert(1, "-c")
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return out


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    d = tmp_path_factory.mktemp("cpp")
    return _compile(os.path.join(ROOT, "tests", "cpp", "fwi_driver.cpp"), str(d / "fwi_driver"))


def test_driver_compiles_and_links(driver):
    assert os.access(driver, os.X_OK)


def test_write_vel_to_an_rsf_file_compiles(tmp_path):
    src = tmp_path / "rsf_user.cpp"
    src.write_text(
        "#include <cstddef>\n"
        "struct sf_File;\n"
        "typedef sf_File *sf_file;\n"
        "void sf_floatwrite(float *, size_t, sf_file);\n"
        "#include \"fwiframework.h\"\n"
        "void write(const FwiFramework &f, sf_file file) { f.writeVel(file); }\n")
    _compile(str(src), str(tmp_path / "rsf_user.o"), link=False)


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["plain", "ess"])
def test_driver_epochs_match_reference(cuda, driver, tmp_path, kind):
    g = golden("small_survey")
    e = golden("small_epochs")
    s, _, vinit = small_survey()
    vin = tmp_path / "vinit.bin"
    dob = tmp_path / "dobs.bin"
    np.ascontiguousarray(vinit, np.float32).tofile(vin)
    np.ascontiguousarray(g["dobs"], np.float32).tofile(dob)
    out = str(tmp_path / "run")
    args = [driver, kind, str(vin), str(dob), out] + [str(x) for x in (
        s.nx, s.nz, s.nt, s.ns, s.ng, s.dx, s.dt, s.fm, s.nb, s.sxbeg, s.jsx, s.szbeg, s.gxbeg, s.jgx, s.gzbeg,
        1500.0, 4700.0, s.nita, s.maxdv, 2)]
    r = subprocess.run(args, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    exvel = np.fromfile(out + ".exvel", np.float32).reshape(e["fwi_vel"].shape)
    objs = np.fromfile(out + ".objs", np.float32)
    vel = np.fromfile(out + ".vel", np.float32).reshape(s.nx, s.nz)
    # the model is clipped to [vmin, vmax] in the transformed variable; back
    # in m/s the bounds hold to float rounding
    assert np.isfinite(vel).all() and 1500.0 * (1 - 1e-5) <= vel.min() and vel.max() <= 4700.0 * (1 + 1e-5)
    if kind == "plain":
        assert rel_l2(exvel, e["fwi_vel"]) < 1e-5
        np.testing.assert_allclose(objs[0], e["fwi_objs"][0, 0], rtol=1e-5)
        np.testing.assert_allclose(objs[1:], e["fwi_objs"][:, 2], rtol=1e-3)
    else:
        assert rel_l2(exvel, e["ess_vel"]) < 1e-5
        np.testing.assert_allclose(objs[0], e["ess_objs"][0, 0], rtol=1e-4)
        np.testing.assert_allclose(objs[1:], e["ess_objs"][:, 1], rtol=1e-4)
