"""The benchmark configurations themselves through the CUDA path, against the
oracle, at their full sizes.

* the small plain case as written: 4,000 beads of one LJ type at 8 nm^-3,
  positions rejected below 0.3 nm (the bench's fluid4k rejects below 0.42 nm,
  because at 0.3 nm and dt 10 fs the REAL*4 restatement of the reference itself
  diverges within ten steps); checked at step 1;
* the hybrid case as specified (hybrid3a: 48,000 atoms, 4,000 centre-of-mass
  sites, MTS 9);
* the 2,000,000-bead CG melt of the roofline study (melt2m).

For each: the Verlet lists equal the REAL*4 restatement's (order included),
the FP32/fixed-point forces of the first force stage lie within 1e-5
(max-norm relative over particles) of the FP64 restatement's, with energies
and virial within 1e-5, and the FP64 path's forces within 1e-9.
"""
import os

import numpy as np
import pytest

from ibisco_b200 import native, synth
from oracle.oracle import Oracle

from conftest import rel_maxnorm

pytestmark = pytest.mark.gpu

CONFIGS = {
    "fluid4k_dmin03": lambda: synth.lj_fluid(n=4000, seed=1, dmin=0.3),
    "hybrid3a": lambda: synth.hybrid_melt(n_atomistic=200, n_cg=0),
    "melt2m": lambda: synth.cg_melt(),
}


@pytest.fixture(scope="module")
def cfgdir(tmp_path_factory):
    base = tmp_path_factory.mktemp("configs")
    made = {}

    def get(name):
        if name not in made:
            d = str(base / name)
            synth.write_system(CONFIGS[name](), d)
            made[name] = d
        return made[name]

    return get


def compare_lists(g, o, which):
    _, no = o.neighbour_list(which, 0, maxnab=1000)
    m = int(no.max()) + 1
    lg, ng = g.neighbour_list(which, maxnab=m)
    np.testing.assert_array_equal(ng, no)
    lo, _ = o.neighbour_list(which, 0, maxnab=m)
    np.testing.assert_array_equal(lg, lo)


@pytest.mark.parametrize("name", list(CONFIGS))
def test_config_lists_and_forces_against_oracle(cfgdir, name):
    d = cfgdir(name)
    threads = os.cpu_count() or 1
    s = native.Setup(d)
    g = native.System(s, native.IBG_PREC_FP32_FIXED)
    g.set_state()
    o32 = Oracle(d, threads=threads)
    o32.init(0)
    for which in (0, 1):
        if which == 1 and o32.info["NCOARSE"] == 0:
            continue
        compare_lists(g, o32, which)
    o32.close()
    o = Oracle(d, threads=threads)
    o.init(1)
    o.forces(1, 1)
    eo = o.obs(1)
    fo = o.state(1)["fxyz"]
    og = g.forces(1)
    err = rel_maxnorm(g.state64()["fxyz"], fo)
    print(f"{name}: FP32/fixed force max-norm relative error against the FP64 oracle {err:.3g}")
    assert err < 1e-5
    for k in ("V_NB1", "V_NB2", "V_NB3", "V_BOND1", "V_ANGLE1", "V_TORSION1"):
        assert abs(og[k] - eo[k]) <= 1e-5 * max(abs(eo[k]), 1.0), k
    pt_g = np.array([og[k] for k in ("PT11", "PT22", "PT33", "PT12", "PT13", "PT23")])
    pt_o = np.array([eo[k] for k in ("PT11", "PT22", "PT33", "PT12", "PT13", "PT23")])
    assert np.abs(pt_g - pt_o).max() / max(np.abs(pt_o).max(), 1.0) < 1e-5
    g.close()
    g64 = native.System(s, native.IBG_PREC_FP64_PLAIN)
    g64.set_state()
    g64.forces(1)
    assert rel_maxnorm(g64.state64()["fxyz"], fo) < 1e-9
