"""Trajectory and restart files (WRITETRJ.F90) written by the host library,
read back with a reader of the same layout (tests/trz.py) and with the
coordinate reader."""
import os
import shutil

import numpy as np

from ibisco_b200 import native
from oracle.oracle import Oracle

from trz import read_trz


def fake_obs(step, box):
    o = native.IbgObs()
    o.ek[0], o.ek[1] = 1234.5, 67.25
    for k, name in enumerate(("v_nb", "v_bond", "v_angle", "v_torsion", "v_oop")):
        for c in range(3):
            getattr(o, name)[c] = (k + 1) * 10.0 + c
    for k in range(6):
        o.pt[k] = 0.5 + 0.25 * k
    for k in range(3):
        o.box[k] = float(box[k])
    o.step = step
    return o


def test_trz_frames_hold_the_step_state_and_observables(sysdir, tmp_path):
    """Two frames: header (frame number, NTRJ * frame, NATOMS, time), box,
    pressure tensor times PSCALE, energies times CONV, positions and
    velocities in nm/ps (WRITETRJ.F90:28-97)."""
    d = sysdir("mix4")
    s = native.Setup(d)
    o = Oracle(d)
    f = o.finfo
    sx, vx, box = s.initial_state()
    path = str(tmp_path / "traj.trz")
    t = native.Trajectory(s, path)
    t.write(10, fake_obs(10, box), sx, vx)
    t.write(20, fake_obs(20, box * 1.01), sx + 0.5, vx * 2)
    t.close()
    title, nrec, frames = read_trz(path)
    assert nrec == 10 and len(frames) == 2 and title
    small = 1.0 / 1e12 / float(f["TIMESCALE"])
    for k, (st, x, v, b) in enumerate(((10, sx, vx, box), (20, sx + 0.5, vx * 2, box * 1.01))):
        fr = frames[k]
        assert fr["frame"] == k + 1 and fr["index"] == s.ntrj * (k + 1) and fr["natoms"] == len(sx)
        dt = float(f["DT"]) * float(f["TIMESCALE"]) * 1e12
        assert abs(fr["time_ps"] - st * dt) <= 1e-6 * st * dt
        np.testing.assert_array_equal(fr["xyz"], x.astype(np.float32))
        np.testing.assert_allclose(fr["vel"], (v.astype(np.float64) * small).astype(np.float32), rtol=0, atol=0)
        np.testing.assert_allclose(np.diag(fr["box"]), b.astype(np.float32), rtol=1e-7)
        pt = np.array([0.5 + 0.25 * q for q in range(6)], np.float32) * f["PSCALE"]
        assert abs(fr["pressure"][0] - pt[:3].sum() / 3.0) <= 1e-6 * abs(pt[:3].sum() / 3.0)
        ptot = sum((q + 1) * 30.0 + 3.0 for q in range(5))
        ek = 1234.5 + 67.25
        np.testing.assert_allclose(fr["energy"][:4], [(ptot + ek) * f["CONV"], ptot * f["CONV"], ek * f["CONV"],
                                                      ek * f["MKTEMP"]], rtol=1e-7)


def test_restart_reads_back_as_a_coordinate_file(sysdir, tmp_path):
    """WRITE_RESTART's file (WRITETRJ.F90:119-178) in the coordinate format:
    read back by the coordinate reader, positions are the same REAL*4 values
    (G21.14), velocities agree to the F16.10 rounding, and types, bonds and
    molecules are unchanged; the time becomes the next run's INITIME."""
    d = sysdir("hybrid")
    s = native.Setup(d)
    sx, vx, box = s.initial_state()
    sx = sx + np.float32(0.123456)
    vx = vx * np.float32(1.7)
    d2 = str(tmp_path / "restarted")
    shutil.copytree(d, d2)
    native.write_restart(s, os.path.join(d2, "coordinate"), 250, box * np.float32(1.002), sx, vx)
    s2 = native.Setup(d2)
    sx2, vx2, box2 = s2.initial_state()
    np.testing.assert_array_equal(sx2, sx)
    np.testing.assert_allclose(vx2, vx, rtol=1e-6, atol=1e-8)
    np.testing.assert_array_equal(box2, (box * np.float32(1.002)).astype(np.float32))
    for name in ("ITYPE", "NBONDS", "JBOND", "TYPE_LABEL", "CONNECTED_TO"):
        np.testing.assert_array_equal(s.array(name), s2.array(name), err_msg=name)
