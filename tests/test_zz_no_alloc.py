"""ibg_nonbonded_static: the nonbonded forces of a list for callers that
cannot allocate device memory, checked against the context path.

The caller owns every device array (here torch allocates them, standing in
for a host's own memory pool); the entry point itself allocates nothing and
keeps its scratch in a fixed __device__ array.  Two calls in a row must both
reproduce the context's force stage (ibg_forces) for a system whose only
interactions are nonbonded, within the 1e-5 tolerance of the parity tests;
the second call also shows the shared scratch is cleared between calls.
"""
import ctypes

import numpy as np
import pytest

from ibisco_b200 import native

pytestmark = pytest.mark.gpu

TOL = 1e-5


def test_static_nonbonded_matches_context_twice(sysdir):
    torch = pytest.importorskip("torch")
    assert torch.cuda.is_available()
    d = sysdir("fluid")  # LJ beads only: the force stage is the atom list's nonbonded forces
    setup = native.Setup(d)
    g = native.System(setup, native.IBG_PREC_FP32_FIXED)
    g.set_state()
    obs = g.forces(1)
    ref = g.state64()["fxyz"]
    st = g.state()
    lst, nn = g.neighbour_list(0)
    maxnab = int(nn.max()) + 1
    lst = np.ascontiguousarray(lst[:, :maxnab])
    index_list = setup.array("ATOM")
    nitems = len(setup.array("ITYPE"))
    n = len(index_list)
    nnebs = np.zeros(nitems, np.int32)
    nnebs[index_list - 1] = nn
    binnb = setup.array("BINNB")
    nnbtype = len(binnb)
    rnbond = setup.array("RNBOND")
    ld_nb = len(rnbond) // nnbtype
    ntype = int(round(len(setup.array("INBONDT")) ** 0.5))
    box = np.array([obs["BOX1"], obs["BOX2"], obs["BOX3"]], np.float32)
    rcut = float(open(d + "/control").read().split("\ncutoff")[1].split()[0])
    rcutsq = np.float32(rcut) * np.float32(rcut)

    dev = torch.device("cuda", 0)

    def up(a, dt):
        return torch.from_numpy(np.ascontiguousarray(a, dt)).to(dev)

    t = {
        "rxyz": up(st["rxyz"].ravel(), np.float32), "itype": up(setup.array("ITYPE"), np.int32),
        "label": up(setup.array("TYPE_LABEL"), np.int32), "index": up(index_list, np.int32),
        "list": up(lst.ravel(), np.int32), "nnebs": up(nnebs, np.int32), "inbondt": up(setup.array("INBONDT"), np.int32),
        "rnbond": up(rnbond, np.float32), "force": up(setup.array("NBOND_FORCE"), np.float32),
        "pot": up(setup.array("NBOND_POT"), np.float32), "binnb": up(binnb, np.float32),
        "ndatnb": up(setup.array("NDATNB"), np.int32),
    }
    f_out = torch.zeros(3 * nitems, dtype=torch.float64, device=dev)
    sums = torch.zeros(9, dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    p = lambda x: ctypes.c_void_p(x.data_ptr())
    err = ctypes.create_string_buffer(256)
    L = native.lib()
    for call in range(2):
        f_out.fill_(float("nan"))
        torch.cuda.synchronize()
        rc = L.ibg_nonbonded_static(
            nitems, n, p(t["rxyz"]), p(t["itype"]), p(t["label"]), p(t["index"]), p(t["list"]), maxnab, p(t["nnebs"]),
            ntype, p(t["inbondt"]), nnbtype, ld_nb, p(t["rnbond"]), p(t["force"]), p(t["pot"]), p(t["binnb"]),
            p(t["ndatnb"]), box.ctypes.data_as(ctypes.c_void_p), ctypes.c_float(rcutsq), p(f_out), p(sums), None, err, 256)
        assert rc == 0, err.value.decode()
        f = f_out.cpu().numpy().reshape(nitems, 3)
        assert np.abs(f - ref).max() / np.abs(ref).max() < TOL, f"call {call + 1}"
        s = sums.cpu().numpy()
        assert abs(s[0] - obs["V_NB1"]) <= TOL * abs(obs["V_NB1"])
        pt = np.array([obs[k] for k in ("PT11", "PT22", "PT33", "PT12", "PT13", "PT23")])
        assert np.abs(s[3:] - pt).max() <= TOL * np.abs(pt).max()


def test_static_rejects_oversized_input():
    err = ctypes.create_string_buffer(256)
    dummy = ctypes.c_void_p(1)
    rc = native.lib().ibg_nonbonded_static(
        300000, 10, dummy, dummy, dummy, dummy, dummy, 8, dummy, 1, dummy, 1, 8, dummy, dummy, dummy, dummy, dummy,
        np.ones(3, np.float32).ctypes.data_as(ctypes.c_void_p), ctypes.c_float(1.0), dummy, dummy, None, err, 256)
    assert rc == -11 and b"IBG_STATIC_MAX_PARTICLES" in err.value
