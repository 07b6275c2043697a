"""Batched shot generation (fm-damp) on the GPU: the shots file against the
compiled reference's FwiForwardModeling of each shot, bit for bit."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_fm_damp_matches_reference(cuda, ref, tmp_path):
    from swfwi_b200 import fm_damp, rsf, survey as sv
    s = sv.small(nx=70, nz=40, nt=200, ns=4)
    v = sv.layered_model(s.nx, s.nz, seed=11)
    vpath, spath = str(tmp_path / "v.rsf"), str(tmp_path / "shots.rsf")
    rsf.write(vpath, v, d=[s.dx, s.dx], o=[0.0, 0.0])
    got = fm_damp.fm_damp(vpath, spath, dt=s.dt, nt=s.nt, ns=s.ns, ng=s.ng, jsx=s.jsx, sxbeg=s.sxbeg,
                          szbeg=s.szbeg, gxbeg=s.gxbeg, gzbeg=s.gzbeg, amp=1000.0, fm=s.fm, nb=s.nb,
                          jgx=s.jgx)
    M = ref.model(s)
    M.bind_velocity(M.expand_domain(v))
    wlt = ref.ricker(s.nt, s.fm, s.dt, 1000.0)
    for shot in range(s.ns):
        np.testing.assert_array_equal(got[shot], M.fwi_forward(wlt, shot))
    np.testing.assert_array_equal(rsf.read_shots(spath, s.ns, s.nt, s.ng), got)
    assert rsf.dims(spath)[0] == [s.nt, s.ng, s.ns]
    assert float(rsf.get(spath, "vmax")) == float(v.max())
