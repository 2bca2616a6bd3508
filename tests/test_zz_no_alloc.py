"""ibg_nonbonded_static: the nonbonded forces of a list for callers that
cannot allocate device memory (a host whose device memory all belongs to its
own pool, or a loop that must not let cudaMalloc/cudaFree synchronise the
device), checked against the context path and against the oracle.

The caller owns every device array (here torch allocates them, standing in
for a host's own memory pool); the entry point itself allocates nothing and
keeps its scratch in a fixed __device__ array.  Two calls in a row must both
reproduce the context's force stage (ibg_forces) for a system whose only
interactions are nonbonded, within the 1e-5 tolerance of the parity tests;
the second call also shows the shared scratch is cleared between calls.  On
the hybrid melt the atom list (a subset of the particles, INDEX_LIST mapping A
to i) and the bead list (explicit beads and centre-of-mass sites, so that
V_NB(2) and V_NB(3) are both filled) are checked against the oracle's
NONBONDED_FORCE on the same list, and a zeroed INBONDT entry returns
IBG_E_MISSING_TABLE.
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


def call_static(torch, n, index_list, lst, nnebs, rxyz, arrays, box, rcutsq):
    """One call on device copies of the given arrays; returns (rc, message,
    forces (NITEMS,3), sums[9])."""
    dev = torch.device("cuda", 0)

    def up(a, dt):
        return torch.from_numpy(np.ascontiguousarray(a, dt)).to(dev)

    nitems = len(arrays["ITYPE"])
    t = {"rxyz": up(rxyz.ravel(), np.float32), "itype": up(arrays["ITYPE"], np.int32),
         "label": up(arrays["TYPE_LABEL"], np.int32), "index": up(index_list, np.int32),
         "list": up(lst.ravel(), np.int32), "nnebs": up(nnebs, np.int32), "inbondt": up(arrays["INBONDT"], np.int32),
         "rnbond": up(arrays["RNBOND"], np.float32), "force": up(arrays["NBOND_FORCE"], np.float32),
         "pot": up(arrays["NBOND_POT"], np.float32), "binnb": up(arrays["BINNB"], np.float32),
         "ndatnb": up(arrays["NDATNB"], np.int32)}
    nnbtype = len(arrays["BINNB"])
    ld_nb = len(arrays["RNBOND"]) // nnbtype
    ntype = int(round(len(arrays["INBONDT"]) ** 0.5))
    f_out = torch.full((3 * nitems,), float("nan"), dtype=torch.float64, device=dev)
    sums = torch.zeros(9, dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    p = lambda x: ctypes.c_void_p(x.data_ptr())
    err = ctypes.create_string_buffer(256)
    box = np.ascontiguousarray(box, np.float32)
    rc = native.lib().ibg_nonbonded_static(
        nitems, n, p(t["rxyz"]), p(t["itype"]), p(t["label"]), p(t["index"]), p(t["list"]), lst.shape[1],
        p(t["nnebs"]), ntype, p(t["inbondt"]), nnbtype, ld_nb, p(t["rnbond"]), p(t["force"]), p(t["pot"]),
        p(t["binnb"]), p(t["ndatnb"]), box.ctypes.data_as(ctypes.c_void_p), ctypes.c_float(rcutsq), p(f_out),
        p(sums), None, err, 256)
    return rc, err.value.decode(), f_out.cpu().numpy().reshape(nitems, 3), sums.cpu().numpy()


@pytest.mark.parametrize("which", [0, 1], ids=["atom_list", "bead_list"])
def test_static_nonbonded_matches_oracle_on_hybrid_lists(sysdir, which):
    """The hybrid melt's atom list and bead list, each through the entry point
    and through the oracle's REAL*4 NONBONDED_FORCE of that list alone, on the
    oracle's positions and lists: forces and V_NB(1..3) within 1e-5 (max-norm
    relative), and the virial within 1e-5 of the FP64 restatement's.  On the bead list both V_NB(2)
    (bead-bead) and V_NB(3) (pairs with a site) are nonzero."""
    from oracle.oracle import Oracle

    torch = pytest.importorskip("torch")
    d = sysdir("hybrid")
    setup = native.Setup(d)
    o = Oracle(d)
    o.init(0)
    names = ("ITYPE", "TYPE_LABEL", "INBONDT", "RNBOND", "NBOND_FORCE", "NBOND_POT", "BINNB", "NDATNB")
    arrays = {k: setup.array(k) for k in names}
    nitems = len(arrays["ITYPE"])
    arrays["TYPE_LABEL"] = arrays["TYPE_LABEL"].copy()
    arrays["TYPE_LABEL"][o.info["NATOMS"]:] = 3  # VIRTUAL_DEF.f90:22 labels the sites
    index_list = setup.array("ATOM" if which == 0 else "BEAD")
    lst, nn = o.neighbour_list(which, 0)
    maxnab = int(nn.max()) + 1
    lst = np.ascontiguousarray(lst[:, :maxnab])
    nnebs = np.zeros(nitems, np.int32)
    nnebs[index_list - 1] = nn
    rxyz = o.state(0)["rxyz"].astype(np.float32)
    box = np.array([o.finfo["BOX1"], o.finfo["BOX2"], o.finfo["BOX3"]], np.float32)
    rc_name = "RCUTSQ_ATOM" if which == 0 else "RCUTSQ_BEAD"
    f_ref, s_ref = o.nonbonded_list(which, 0)
    # the reference sums the virial in REAL*4 (PT11... are REAL*4), which on
    # the atom list loses ~1e-3 of it to rounding; the entry point sums it in
    # double, so its virial is checked against the FP64 restatement
    o64 = Oracle(d)
    o64.init(1)
    _, s64 = o64.nonbonded_list(which, 1)
    rc, msg, f, s = call_static(torch, len(index_list), index_list, lst, nnebs, rxyz, arrays, box,
                                float(o.finfo[rc_name]))
    assert rc == 0, msg
    assert np.abs(f - f_ref).max() / np.abs(f_ref).max() < TOL
    assert np.abs(s[:3] - s_ref[:3]).max() <= TOL * np.abs(s_ref[:3]).max()
    assert np.abs(s[3:] - s64[3:]).max() <= TOL * np.abs(s64[3:]).max()
    if which == 1:
        assert abs(s_ref[1]) > 0 and abs(s_ref[2]) > 0 and s_ref[0] == 0
    # a pair type without a table: INBONDT zeroed for every pair
    arrays["INBONDT"] = np.zeros_like(arrays["INBONDT"])
    rc, msg, _, _ = call_static(torch, len(index_list), index_list, lst, nnebs, rxyz, arrays, box,
                                float(o.finfo[rc_name]))
    assert rc == native.STATUS_CODE["IBG_E_MISSING_TABLE"], msg
