"""Centre-of-mass virtual sites in the reference's own form, on the GPU.

VIRTUAL_DEF.f90:31 resets only SUMTOTXYZ(1) before each centre-of-mass site,
so the y and z sums run on from one such site to the next.  The default
device path resets all three (each site at its centre of mass);
ibg_set_vsite_com(ctx, IBG_VS_COM_REFERENCE) reproduces the reference.  Here
that form is checked against the oracle run with its COM fix off:

* the virtual sites' positions and the bead list (which holds the sites) are
  identical to the REAL*4 restatement's;
* the FP64 path's forces and trajectory match the FP64 restatement's to 1e-9.

The FP32 path is not held to the FP64 restatement here: the running sums
reach thousands of nm*mass, where REAL*4 and FP64 positions of the sites
differ by far more than the force tolerance measures.
"""
import numpy as np
import pytest

from ibisco_b200 import native
from oracle.oracle import Oracle

from conftest import rel_maxnorm

pytestmark = pytest.mark.gpu


def make(d, prec, form):
    g = native.System(native.Setup(d), prec)
    g.set_vsite_com(form)
    g.set_state()
    return g


@pytest.mark.parametrize("name", ["mix4", "hybrid"])
def test_reference_com_form_sites_and_lists_match_oracle(sysdir, name):
    d = sysdir(name)
    g = make(d, native.IBG_PREC_FP32_FIXED, native.IBG_VS_COM_REFERENCE)
    o = Oracle(d, com_fix=False)
    o.init(0)
    na, ni = g.natoms, g.nitems
    rg = g.state()["rxyz"][na:ni]
    ro = o.state(0)["rxyz"][na:ni].astype(np.float32)
    np.testing.assert_array_equal(rg, ro)
    lg, ng = g.neighbour_list(1)
    lo, no = o.neighbour_list(1, 0)
    np.testing.assert_array_equal(ng, no)
    np.testing.assert_array_equal(lg, lo)
    # the fixed form puts the sites elsewhere
    f = make(d, native.IBG_PREC_FP32_FIXED, native.IBG_VS_COM_FIXED)
    assert not np.array_equal(f.state()["rxyz"][na:ni], rg)


@pytest.mark.parametrize("name", ["mix4", "hybrid"])
def test_reference_com_form_fp64_path_matches_oracle(sysdir, name):
    """Forces of the first step within 1e-9 of the FP64 restatement's, then up
    to 12 steps.  The running y and z sums throw the sites far from their
    members, so the forces through a site grow without bound and angles and
    torsions through one can leave their tables: the reference then stops
    (TORSIONS.inc:105-109), and the device must report IBG_E_TORSION_TABLE at
    that same step.  States are compared (1e-9) up to the last step the
    restatement completes with finite values."""
    from oracle.oracle import OracleError

    d = sysdir(name)
    g = make(d, native.IBG_PREC_FP64_PLAIN, native.IBG_VS_COM_REFERENCE)
    o = Oracle(d, com_fix=False)
    o.init(1)
    g.forces(1)
    o.forces(1, 1)
    assert rel_maxnorm(g.state64()["fxyz"], o.state(1)["fxyz"]) < 1e-9
    # how far the restatement gets: a torsion off its table stops it, and the
    # far-flung sites can also blow the state up to non-finite values, after
    # which there is nothing left to compare
    o = Oracle(d, com_fix=False)
    o.init(1)
    stop, done = None, 0
    for st in range(1, 13):
        try:
            o.step(st, 1)
        except OracleError as e:
            assert "torsion" in str(e).lower()
            stop = st
            break
        x = o.state(1)
        if not (np.isfinite(x["sxyz"]).all() and np.isfinite(x["vxyz"]).all()):
            break
        done = st
    assert done >= 1
    g = make(d, native.IBG_PREC_FP64_PLAIN, native.IBG_VS_COM_REFERENCE)
    o = Oracle(d, com_fix=False)
    o.init(1)
    for st in range(1, done + 1):
        o.step(st, 1)
    g.run(1, done)
    na = g.natoms
    so, sg = o.state(1), g.state64()
    span = np.abs(so["sxyz"][:na]).max()
    assert np.abs(sg["sxyz"][:na] - so["sxyz"][:na]).max() / span < 1e-9
    assert rel_maxnorm(sg["vxyz"], so["vxyz"]) < 1e-8
    if stop == done + 1:
        with pytest.raises(native.IbiscoError) as e:
            g.step(stop)
        assert e.value.code == native.STATUS_CODE["IBG_E_TORSION_TABLE"]


def test_reference_com_form_is_refused_in_a_batch_and_for_bad_values(sysdir):
    g = native.System(native.Setup(sysdir("mix4")), native.IBG_PREC_FP32_FIXED)
    with pytest.raises(native.IbiscoError):
        g.set_vsite_com(7)
