"""The reference's own regression fixtures through the CUDA path.

testsuite/atomisticPA (NVT, 18,360 atoms: bonds, angles, torsions, 21
nonbonded tables, exclusions with non_bonded 4, halt_drift 10) and
testsuite/hybridPA (NPT: 6,744 atoms, 1,440 beads and 960 centre virtual
sites, 36 tables, SCALEBP) are read with the `mts 0` key added, as the oracle's
golden test reads them.  Through the C ABI:

* the atom and bead Verlet lists equal the REAL*4 restatement's, order
  included;
* the FP32/fixed-point forces lie within 1e-5 (max-norm relative) of the FP64
  restatement's, and the FP64 path's within 1e-9;
* the first three atoms' coordinates, velocities and the box after 10 and 40
  steps lie within the golden tolerances of testsuite/tests.py:10-68 that the
  oracle meets (tests/test_oracle_golden.py), on both GPU paths.
"""
import numpy as np
import pytest

from ibisco_b200 import native
from oracle.oracle import Oracle

from conftest import rel_maxnorm
from test_oracle_golden import GOLD, TOL

pytestmark = pytest.mark.gpu

FIXTURES = ["atomisticPA", "hybridPA"]


def make(d, prec):
    g = native.System(native.Setup(d), prec)
    g.set_state()
    return g


@pytest.mark.parametrize("fixture", FIXTURES)
def test_lists_match_reference_order(reftree, fixture):
    d = reftree(fixture)
    g = make(d, native.IBG_PREC_FP32_FIXED)
    o = Oracle(d, threads=8)
    o.init(0)
    for which in (0, 1):
        if which == 1 and o.info["NCOARSE"] == 0:
            continue
        _, no = o.neighbour_list(which, 0, maxnab=1000)
        m = int(no.max()) + 1
        lg, ng = g.neighbour_list(which, maxnab=m)
        lo, no = o.neighbour_list(which, 0, maxnab=m)
        np.testing.assert_array_equal(ng, no)
        np.testing.assert_array_equal(lg, lo)


@pytest.mark.parametrize("fixture", FIXTURES)
def test_forces_against_fp64_oracle(reftree, fixture):
    d = reftree(fixture)
    o = Oracle(d, threads=8)
    o.init(1)
    o.forces(1, 1)
    eo = o.obs(1)
    fo = o.state(1)["fxyz"]
    g = make(d, native.IBG_PREC_FP32_FIXED)
    og = g.forces(1)
    err = rel_maxnorm(g.state64()["fxyz"], fo)
    print(f"{fixture}: FP32/fixed force max-norm relative error against the FP64 oracle {err:.3g}")
    assert err < 1e-5
    for k in ("V_NB1", "V_NB2", "V_BOND1", "V_ANGLE1", "V_TORSION1", "PT11", "PT22", "PT33"):
        assert abs(og[k] - eo[k]) <= 1e-5 * max(abs(eo[k]), 1.0), k
    g64 = make(d, native.IBG_PREC_FP64_PLAIN)
    g64.forces(1)
    assert rel_maxnorm(g64.state64()["fxyz"], fo) < 1e-9


def frames(g, timescale):
    """Coordinates (Angstrom) and velocities (Angstrom/ps) of atoms 1-3 and the
    box (Angstrom) after steps 10 and 40, as WRITETRJ.F90 writes them."""
    small = 1.0 / 1e12 / float(timescale)
    out = {}
    first = 1
    for st in (10, 40):
        obs = g.run(first, st - first + 1, observe=True)
        first = st + 1
        s = g.state()
        x = s["sxyz"][:3].astype(np.float32) * np.float32(10)
        v = (s["vxyz"][:3].astype(np.float64) * small).astype(np.float32) * np.float32(10)
        b = np.float32(obs[-1]["BOX1"]) * np.float32(10)
        out[st] = (x, v, b)
    return out


@pytest.mark.parametrize("prec", [native.IBG_PREC_FP32_FIXED, native.IBG_PREC_FP64_PLAIN], ids=["fp32", "fp64"])
@pytest.mark.parametrize("fixture", FIXTURES)
def test_trajectory_against_reference_goldens(reftree, fixture, prec):
    d = reftree(fixture)
    o = Oracle(d)
    g = make(d, prec)
    fr = frames(g, o.finfo["TIMESCALE"])
    gold = GOLD[fixture]
    for key, st in (("short", 10), ("long", 40)):
        x, v, b = fr[st]
        tx, tv, tb = TOL[fixture][key]
        dx = np.abs(x - np.array(gold[f"ref_coords_{key}"])).max()
        dv = np.abs(v - np.array(gold[f"ref_velos_{key}"])).max()
        db = abs(b - gold[f"ref_box_{key}"][0])
        print(f"{fixture} step {st}: |dx| {dx:.2e} A, |dv| {dv:.2e} A/ps, |dbox| {db:.2e} A")
        assert dx < tx and dv < tv and db < tb
