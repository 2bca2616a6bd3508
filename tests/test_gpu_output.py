"""Trajectory output fed from the device: run_with_output steps the system in
runs of NTRJ steps (observables from the device's per-step ring, state from
ibg_get_state) and writes a TRZ frame after each, as NEW_LOOP.F90 calls
WRITETRJ every NTRJ steps; the trajectory equals an uninterrupted run."""
import numpy as np
import pytest

from ibisco_b200 import native

from trz import read_trz

pytestmark = pytest.mark.gpu


def test_run_with_output_writes_every_ntrj_steps(sysdir, tmp_path):
    d = sysdir("mix5_mts")
    s = native.Setup(d)
    g = native.System(s, native.IBG_PREC_FP32_FIXED)
    g.set_state()
    path = str(tmp_path / "traj.trz")
    obs = native.run_with_output(g, 1, 25, path, restart_path=str(tmp_path / "restart"), ntrj=10)
    assert [o["STEP"] for o in obs] == list(range(1, 26))
    _, _, frames = read_trz(path)
    assert [f["frame"] for f in frames] == [1, 2]
    ref = native.System(s, native.IBG_PREC_FP32_FIXED)
    ref.set_state()
    robs = ref.run(1, 25, observe=True)
    assert obs == robs
    x = g.state()
    assert np.array_equal(x["sxyz"], ref.state()["sxyz"])
    ref2 = native.System(s, native.IBG_PREC_FP32_FIXED)
    ref2.set_state()
    ref2.run(1, 20)
    st = ref2.state()
    np.testing.assert_array_equal(frames[1]["xyz"], st["sxyz"][: g.natoms])
    o20 = robs[19]
    conv_e = frames[1]["energy"][2]  # kinetic energy times CONV
    ek = o20["EK1"] + o20["EK2"]
    assert abs(conv_e / ek - frames[0]["energy"][2] / (robs[9]["EK1"] + robs[9]["EK2"])) < 1e-12
