"""The product's host setup (ibg_setup_read) reproduces the reference's setup
phase bit for bit: type maps, SETLIS angle/torsion/out-of-plane lists,
exclusions (BUILD_CONNECTIVITY + RDVIRTBONDS), virtual-site maps (RDVIRTUAL)
and the FTABLE force tables, checked against the oracle's restatement."""
import os

import numpy as np
import pytest

from ibisco_b200 import native
from oracle.oracle import Oracle

ONE_BASED = {"ITYPE", "NBONDS", "NIJK", "NOANGLEIJK", "NIJKL", "FNIJKL", "NOOPIJKL", "CONNECTIONS", "ATOM", "BEAD",
             "VITYPE", "VIRT_CENTER", "VIRT_NUMATOMS", "NDATB", "NDATAN", "NDATT", "NDATNB", "NDATO", "MASS",
             "INVMASS", "VIRT_INVMASS", "VIRT_MASS", "BINB", "BINA", "BINNB", "BINO", "BINT", "BOND_TYPE_LABEL",
             "ANGLE_TYPE_LABEL", "TORSION_TYPE_LABEL", "OOP_TYPE_LABEL"}
INT_ARRAYS = ["ITYPE", "NBONDS", "JBOND", "NIJK", "JANGLEIJK", "KANGLEIJK", "NOANGLEIJK", "NOJANGLEIJK",
              "NOKANGLEIJK", "NIJKL", "JTORIJKL", "KTORIJKL", "LTORIJKL", "FNIJKL", "FJTORIJKL", "FKTORIJKL",
              "FLTORIJKL", "NOOPIJKL", "JOOPIJKL", "KOOPIJKL", "LOOPIJKL", "CONNECTIONS", "CONNECTED_TO", "IBONDT",
              "INBONDT", "IANGT", "ITORT", "IOOPT", "VITYPE", "VIRT_CENTER", "VIRT_NUMATOMS", "VIRT_ATM_IND",
              "NDATB", "NDATAN", "NDATT", "NDATNB", "NDATO", "ATOM", "BEAD", "BOND_TYPE_LABEL",
              "ANGLE_TYPE_LABEL", "TORSION_TYPE_LABEL", "OOP_TYPE_LABEL"]
FLOAT_ARRAYS = ["MASS", "INVMASS", "VXYZ", "VIRT_INVMASS", "VIRT_MASSCOEFF", "BINB", "BINA", "BINNB", "BINO",
                "BINT"]
TABLES = [("NBTYPE", "NDATB", ["RBOND", "BOND_POT", "BOND_FORCE"], False),
          ("NATYPE", "NDATAN", ["ANGLE", "BEND_POT", "BEND_FORCE"], False),
          ("NTTYPE", "NDATT", ["ANGLE_TOR", "TOR_POT", "TOR_FORCE"], False),
          ("NNBTYPE", "NDATNB", ["RNBOND", "NBOND_POT", "NBOND_FORCE"], False),
          ("NOTYPE", "NDATO", ["ANGLE_OOP", "OOP_POT", "OOP_FORCE"], False)]


def compare_setup(d):
    o = Oracle(d)
    s = native.Setup(d)
    for name in INT_ARRAYS + FLOAT_ARRAYS:
        a = o.array(name)
        b = s.array(name)
        if name in ONE_BASED:
            a = a[1:]
        n = min(len(a), len(b)) if name in ("VIRT_ATM_IND",) else None
        if len(a) == 0 and len(b) <= 1:
            continue
        np.testing.assert_array_equal(a if n is None else a[:n], b if n is None else b[:n], err_msg=name)
    sx = o.array("SXYZ")[: 3 * o.info["NATOMS"]]
    np.testing.assert_array_equal(sx, s.array("SXYZ"))
    # tables: the oracle keeps X(NT, 0:W-1), the product X(NT, 0:ld-1); rows
    # 0..NDAT+1 (everything the step can read) must agree bit for bit
    for count, ndat_name, names, _ in TABLES:
        nt = o.info[count]
        if nt == 0:
            continue
        nd = o.array(ndat_name)[1:]
        for name in names:
            a = o.array(name)
            b = s.array(name)
            wa = len(a) // nt
            wb = len(b) // nt
            for t in range(nt):
                rows = nd[t] + 2
                if name.startswith(("RNBOND", "NBOND")):
                    # product keeps the reference's index-fastest nonbonded layout
                    ra = a[t + nt * np.arange(rows)]
                    rb = b[wb * t + np.arange(rows)]
                else:
                    ra = a[t + nt * np.arange(rows)]
                    rb = b[t + nt * np.arange(rows)]
                np.testing.assert_array_equal(ra, rb, err_msg=f"{name} table {t + 1}")


@pytest.mark.parametrize("name", ["fluid", "melt", "mix4", "mix5_mts", "mix_npt", "mix_y"])
def test_host_setup_matches_oracle(sysdir, name):
    compare_setup(sysdir(name))


def test_scalev_rescales_to_the_control_temperature(sysdir):
    """initialize_velocities Y runs SCALEV (SCALEV.f90:13-26, main.F90:168-171):
    the velocities (bit for bit the oracle's, above) now carry the control
    file's temperature, TEMP = EK * MKTEMP = TEMP_IN, to REAL*4 rounding; with
    N they are the coordinate file's, unscaled."""
    s = native.Setup(sysdir("mix_y"))
    assert s.restart == 1
    o = Oracle(sysdir("mix_y"))
    v = s.array("VXYZ").reshape(-1, 3).astype(np.float64)
    m = s.array("MASS").astype(np.float64)[s.array("ITYPE")[: v.shape[0]] - 1]
    t = 0.5 * float((m[:, None] * v * v).sum()) * float(o.finfo["MKTEMP"])
    assert abs(t / float(o.finfo["TEMP_IN"]) - 1.0) < 1e-6
    n = native.Setup(sysdir("mix4"))
    assert n.restart == 0
    _, v0, _ = n.initial_state()
    np.testing.assert_array_equal(v0.ravel()[: len(n.array("VXYZ"))], n.array("VXYZ"))


@pytest.mark.parametrize("fixture", ["atomisticPA", "hybridPA"])
def test_host_setup_matches_oracle_on_reference_fixtures(reftree, fixture):
    compare_setup(reftree(fixture))


def test_setup_reports_missing_keyword(tmp_path, sysdir):
    import shutil
    d = str(tmp_path / "bad")
    shutil.copytree(sysdir("fluid"), d)
    lines = [l for l in open(d + "/control").read().splitlines() if not l.startswith("mts")]
    open(d + "/control", "w").write("\n".join(lines) + "\n")
    with pytest.raises(native.IbiscoError) as e:
        native.Setup(d)
    assert e.value.code == -12 and "mts" in str(e.value)


def test_setup_reports_missing_file(tmp_path):
    with pytest.raises(native.IbiscoError) as e:
        native.Setup(str(tmp_path / "nothing"))
    assert e.value.code == -12


def test_exclusions_rows_are_sorted_and_bounded(sysdir):
    s = native.Setup(sysdir("mix5_mts"))
    n = len(s.array("ITYPE"))
    conn = s.array("CONNECTIONS")
    to = s.array("CONNECTED_TO").reshape(20, n)
    natoms = len(s.array("SXYZ")) // 3
    for i in range(natoms):
        row = to[: conn[i], i]
        assert (conn[i] <= 20) and np.all(row[:-1] < row[1:]) if len(row) > 1 else True


def read_files(d):
    return {f: open(os.path.join(d, f), "rb").read() for f in os.listdir(d)}


def same_setup(a, b):
    """Every array of two setups bit for bit; tables over the rows a step can
    read (0..NDAT+1), whatever their leading dimension."""
    for name in INT_ARRAYS + FLOAT_ARRAYS + ["SXYZ", "NDATNB", "BINNB"]:
        np.testing.assert_array_equal(a.array(name), b.array(name), err_msg=name)
    nd = a.array("NDATNB")
    for name in ("RNBOND", "NBOND_POT", "NBOND_FORCE"):
        xa, xb = a.array(name), b.array(name)
        wa, wb = len(xa) // len(nd), len(xb) // len(nd)
        for t in range(len(nd)):
            rows = nd[t] + 2
            np.testing.assert_array_equal(xa[wa * t + np.arange(rows)], xb[wb * t + np.arange(rows)],
                                          err_msg=f"{name} table {t + 1}")


@pytest.mark.parametrize("name", ["mix4", "hybrid", "mix5_mts"])
def test_setup_from_files_in_memory_equals_directory(sysdir, name):
    """ibg_setup_read_mem runs the same readers on buffers as ibg_setup_read
    on the directory's files."""
    d = sysdir(name)
    same_setup(native.Setup(d), native.Setup(files=read_files(d)))


def test_setup_from_memory_reports_a_missing_file(sysdir):
    files = read_files(sysdir("mix4"))
    del files["coordinate"]
    with pytest.raises(native.IbiscoError, match="coordinate"):
        native.Setup(files=files)


@pytest.mark.parametrize("case", ["same_length", "longer", "offset_start"])
def test_nonbonded_table_replacement_equals_reading_that_table(sysdir, tmp_path, case):
    """ibg_setup_set_nb_table gives the arrays of a setup read from files whose
    table holds the same rows (RDINTERACT.f90:504-533 and FTABLE.f90:59-75):
    a perturbed table of the same length, a longer one (the table columns
    widen), and one that does not start at r = 0 (a row 0 is inserted)."""
    import shutil

    from ibisco_b200 import synth

    src = sysdir("fluid")
    rmax, dr = {"same_length": (1.2, 0.002), "longer": (1.6, 0.002), "offset_start": (1.2, 0.002)}[case]
    t = synth.perturbed_lj_table("nb11", 0.47, 3.5, rmax, dr, [0.3, -0.2, 0.1, 0.05, -0.05])
    r, v = np.asarray(t.x, np.float32), np.asarray(t.v, np.float32)
    if case == "offset_start":
        r, v = r[5:], v[5:]
    d2 = str(tmp_path / "replaced")
    shutil.copytree(src, d2)
    with open(os.path.join(d2, "nb11"), "w") as f:
        for a, b in zip(r.astype(np.float64), v.astype(np.float64)):
            f.write("%.9g  %.9g\n" % (a, b))
    s = native.Setup(src)
    s.set_nb_table(1, r, v)
    same_setup(native.Setup(d2), s)
    with pytest.raises(native.IbiscoError):
        s.set_nb_table(2, r, v)
