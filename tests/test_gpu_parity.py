"""CUDA path against the oracle, through the C ABI.

* neighbour lists: identical to the reference's, including order, for the
  same REAL*4 state (NEW_NEIGHBOUR_WITHLIST.f90); exclusions identical;
* forces and energies of the FP32/fixed-point path within 1e-5 relative
  (max-norm over particles) of the oracle's FP64 engine on the same positions;
* the FP64 path agrees with the oracle's FP64 engine to 1e-9;
* short trajectories (NVT, NVE, NPT, MTS, and from velocities rescaled by
  SCALEV when initialize_velocities is Y) track the FP64 oracle;
* FP32/fixed-point results are bitwise reproducible run to run.
"""
import numpy as np
import pytest

from ibisco_b200 import native
from oracle.oracle import Oracle

from conftest import rel_maxnorm

pytestmark = pytest.mark.gpu

FORCE_TOL = 1e-5     # FP32/fixed vs FP64, max-norm relative
ENERGY_TOL = 1e-5
FP64_TOL = 1e-9      # FP64 path vs FP64 oracle

SYSTEMS = ["fluid", "melt", "mix4", "mix5_mts", "mix_npt", "mix_nve", "hybrid", "mix_y"]


def make(d, prec):
    s = native.Setup(d)
    g = native.System(s, prec)
    g.set_state()
    return s, g


def oracle_init(d, prec):
    o = Oracle(d)
    o.init(prec)
    return o


@pytest.mark.parametrize("name", SYSTEMS)
def test_neighbour_lists_match_reference_order(sysdir, name):
    d = sysdir(name)
    _, g = make(d, native.IBG_PREC_FP32_FIXED)
    o = oracle_init(d, 0)
    for which in (0, 1):
        if which == 1 and o.info["NCOARSE"] == 0:
            continue
        lg, ng = g.neighbour_list(which)
        lo, no = o.neighbour_list(which, 0)
        np.testing.assert_array_equal(ng, no)
        np.testing.assert_array_equal(lg, lo)


@pytest.mark.parametrize("prec", [0, 1], ids=["fp32", "fp64"])
@pytest.mark.parametrize("name", ["melt", "dense"])
def test_neighbour_lists_staged_and_unstaged_cells(sysdir, name, prec):
    """The list build stages a cell's candidates in shared memory when they
    fit (2,304 in FP32, 1,152 in FP64) and reads them from global memory
    otherwise; the dense fluid takes the second way on both paths.  Each
    path's lists equal the oracle's at its own precision."""
    d = sysdir(name)
    _, g = make(d, native.IBG_PREC_FP32_FIXED if prec == 0 else native.IBG_PREC_FP64_PLAIN)
    o = oracle_init(d, prec)
    lg, ng = g.neighbour_list(0)
    lo, no = o.neighbour_list(0, prec)
    np.testing.assert_array_equal(ng, no)
    np.testing.assert_array_equal(lg, lo)


@pytest.mark.parametrize("name", ["mix4", "mix5_mts"])
def test_exclusions_on_device(sysdir, name):
    d = sysdir(name)
    s, g = make(d, native.IBG_PREC_FP32_FIXED)
    c, t = g.exclusions()
    np.testing.assert_array_equal(c, s.array("CONNECTIONS"))
    np.testing.assert_array_equal(t, s.array("CONNECTED_TO"))


def energies(obs):
    keys = [k for k in obs if k.startswith(("V_NB", "V_BOND", "V_ANGLE", "V_TORSION", "V_OOP"))]
    return np.array([obs[k] for k in sorted(keys)])


@pytest.mark.parametrize("smem", [0, 1], ids=["tables_l1", "tables_smem"])
@pytest.mark.parametrize("name", SYSTEMS)
def test_forces_fp32_fixed_against_fp64_oracle(sysdir, name, smem):
    d = sysdir(name)
    _, g = make(d, native.IBG_PREC_FP32_FIXED)
    g.set_tuning(nb_tables_smem=smem)
    o = oracle_init(d, 1)
    og = g.forces(1)
    o.forces(1, 1)
    fo = o.state(1)["fxyz"]
    fg = g.state64()["fxyz"]
    assert rel_maxnorm(fg, fo) < FORCE_TOL
    eo = o.obs(1)
    e_gpu, e_orc = energies(og), energies(eo)
    scale = max(np.abs(e_orc).max(), 1.0)
    assert np.abs(e_gpu - e_orc).max() / scale < ENERGY_TOL
    pt_g = np.array([og[k] for k in ("PT11", "PT22", "PT33", "PT12", "PT13", "PT23")])
    pt_o = np.array([eo[k] for k in ("PT11", "PT22", "PT33", "PT12", "PT13", "PT23")])
    assert np.abs(pt_g - pt_o).max() / max(np.abs(pt_o).max(), 1.0) < ENERGY_TOL


def test_forces_fp32_fixed_against_fp64_path_in_a_large_box(tmp_path):
    """The 1e-5 bar (max-norm relative over particles) against the plain FP64
    GPU path, on the 40,000-bead melt (12.6 nm box).  Far from the box centre
    a REAL*4 coordinate resolves only ~5e-7 nm, which the steep LJ wall turns
    into ~2e-5 force errors, so the nonbonded kernel takes its displacements
    from 32-bit box fractions; and a pair that sits at the cutoff within FP32
    rounding is decided as the FP64 path decides it."""
    from ibisco_b200 import synth

    d = str(tmp_path / "melt40k")
    synth.write_system(synth.polymer_melt(nchains=400, nper=100, seed=2, nsteps=20), d)
    s = native.Setup(d)
    out = {}
    for prec in (native.IBG_PREC_FP32_FIXED, native.IBG_PREC_FP64_PLAIN):
        g = native.System(s, prec)
        g.set_state()
        out[prec] = (g.forces(1), g.state64()["fxyz"])
    (o32, f32), (o64, f64) = out[native.IBG_PREC_FP32_FIXED], out[native.IBG_PREC_FP64_PLAIN]
    err = rel_maxnorm(f32, f64)
    print(f"FP32/fixed vs FP64 path, 40,000 beads: force max-norm relative error {err:.3g}")
    assert err < FORCE_TOL
    for k in ("V_NB1", "PT11", "PT22", "PT33"):
        assert abs(o32[k] - o64[k]) <= ENERGY_TOL * abs(o64[k]), k


def test_cutoff_pairs_beyond_their_buffer_repeat_the_step(tmp_path):
    """A simple cubic lattice (20^3 beads, spacing 0.5 nm, cutoff 1.0 nm) puts
    24,000 pairs exactly at the cutoff, far more than the FP32 kernel's first
    buffer for them holds (4,096).  The step is aborted, the buffer grows and
    the step is repeated: the run completes and its energies match the FP64
    path's, which decides those pairs the same way (outside)."""
    from ibisco_b200 import synth

    spec = synth.lj_fluid(n=8000, rho=8.0, seed=21, nsteps=10, dmin=0.42)
    L = spec.box[0]
    k = np.arange(20)
    spec.pos = np.stack(np.meshgrid(k, k, k, indexing="ij"), -1).reshape(-1, 3) * (L / 20) - L / 2
    spec.control = dict(spec.control, cutoff=1.0, bead_cutoff=1.0)
    d = str(tmp_path / "lattice")
    synth.write_system(spec, d)
    s = native.Setup(d)
    out = {}
    for prec in (native.IBG_PREC_FP32_FIXED, native.IBG_PREC_FP64_PLAIN):
        g = native.System(s, prec)
        g.set_state()
        out[prec] = g.run(1, 3, observe=True)
    for o32, o64 in zip(out[native.IBG_PREC_FP32_FIXED], out[native.IBG_PREC_FP64_PLAIN]):
        assert abs(o32["V_NB1"] - o64["V_NB1"]) <= ENERGY_TOL * abs(o64["V_NB1"])


@pytest.mark.parametrize("name", SYSTEMS)
def test_forces_fp64_path_against_fp64_oracle(sysdir, name):
    d = sysdir(name)
    _, g = make(d, native.IBG_PREC_FP64_PLAIN)
    o = oracle_init(d, 1)
    og = g.forces(1)
    o.forces(1, 1)
    assert rel_maxnorm(g.state64()["fxyz"], o.state(1)["fxyz"]) < FP64_TOL
    e_gpu, e_orc = energies(og), energies(o.obs(1))
    assert np.abs(e_gpu - e_orc).max() / max(np.abs(e_orc).max(), 1.0) < FP64_TOL


@pytest.mark.parametrize("name", SYSTEMS)
def test_trajectory_against_fp64_oracle(sysdir, name):
    """12 steps (two list rebuilds, MTS explicit and extrapolated steps, a
    momentum removal and a barostat update where the system has them)."""
    d = sysdir(name)
    _, g = make(d, native.IBG_PREC_FP32_FIXED)
    _, g64 = make(d, native.IBG_PREC_FP64_PLAIN)
    o = oracle_init(d, 1)
    nsteps = 12
    obs = g.run(1, nsteps, observe=True)
    obs64 = g64.run(1, nsteps, observe=True)
    for st in range(1, nsteps + 1):
        o.step(st, 1)
    so = o.state(1)
    s32, s64 = g.state64(), g64.state64()
    na = so["vxyz"].shape[0]
    span = np.abs(so["sxyz"][:na]).max()
    assert np.abs(s64["sxyz"][:na] - so["sxyz"][:na]).max() / span < 1e-9
    assert rel_maxnorm(s64["vxyz"], so["vxyz"]) < 1e-8
    assert np.abs(s32["sxyz"][:na] - so["sxyz"][:na]).max() / span < 1e-6
    assert rel_maxnorm(s32["vxyz"], so["vxyz"]) < 1e-4
    eo = o.obs(1)
    for k in ("TEMP", "BOX1"):
        assert abs(obs64[-1][k] - eo[k]) <= 1e-9 * max(abs(eo[k]), 1.0)
        assert abs(obs[-1][k] - eo[k]) <= 1e-5 * max(abs(eo[k]), 1.0)
    assert [o_["STEP"] for o_ in obs] == list(range(1, nsteps + 1))


def test_run_is_bitwise_reproducible(sysdir):
    d = sysdir("melt")
    _, a = make(d, native.IBG_PREC_FP32_FIXED)
    _, b = make(d, native.IBG_PREC_FP32_FIXED)
    a.run(1, 25)
    b.run(1, 25)
    sa, sb = a.state64(), b.state64()
    assert np.array_equal(sa["sxyz"], sb["sxyz"])
    assert np.array_equal(sa["vxyz"], sb["vxyz"])
    assert np.array_equal(sa["fxyz"], sb["fxyz"])


def test_step_and_run_agree(sysdir):
    """Direct kernel launches (timing mode) and CUDA-graph replay give the same state."""
    d = sysdir("mix5_mts")
    _, a = make(d, native.IBG_PREC_FP32_FIXED)
    _, b = make(d, native.IBG_PREC_FP32_FIXED)
    native.lib().ibg_set_timing(a._h, 1)
    for st in range(1, 11):
        a.step(st)
    b.run(1, 10)
    assert np.array_equal(a.state64()["sxyz"], b.state64()["sxyz"])


def test_list_storage_growth_mid_run_is_exact(sysdir):
    """A rebuild that outgrows the list storage stops the run at that step; the
    storage grows and the step is repeated.  The result is bitwise the run that
    never ran out of storage."""
    d = sysdir("melt")
    _, a = make(d, native.IBG_PREC_FP32_FIXED)
    _, b = make(d, native.IBG_PREC_FP32_FIXED)
    a.run(1, 29)
    b.run(1, 9)
    g0 = b.timing()["list_growths"]
    native.lib().ibg_set_list_rows(b._h, 1)  # step 10 rebuilds the lists
    obs = b.run(10, 20, observe=True)
    assert b.timing()["list_growths"] > g0
    assert [o["STEP"] for o in obs] == list(range(10, 30))
    sa, sb = a.state64(), b.state64()
    assert np.array_equal(sa["sxyz"], sb["sxyz"])
    assert np.array_equal(sa["vxyz"], sb["vxyz"])


def test_lists_after_steps_match_reference(sysdir):
    """After the system has moved, the lists built from the current REAL*4
    state are again identical to the reference's."""
    d = sysdir("fluid")
    _, g = make(d, native.IBG_PREC_FP32_FIXED)
    g.run(1, 15)
    st = g.state()
    _, v, b = native.Setup(d).initial_state()
    box = np.array([g.step(16)["BOX1"]] * 3, np.float32)
    st = g.state()
    g.set_state(st["sxyz"][: g.natoms], st["vxyz"], box)
    o = Oracle(d)
    o.set_state(st["sxyz"][: g.natoms], st["vxyz"], box, 0)
    lg, ng = g.neighbour_list(0)
    lo, no = o.neighbour_list(0, 0)
    np.testing.assert_array_equal(ng, no)
    np.testing.assert_array_equal(lg, lo)


def test_list_overflow_is_reported(sysdir):
    """A neighbour count reaching MAXNAB is the reference's 'LIST TOO SMALL'
    STOP (NEW_NEIGHBOUR_WITHLIST.f90:72); here it is a status code."""
    s = native.Setup(sysdir("fluid"))
    g = native.System(s, native.IBG_PREC_FP32_FIXED, maxnab=20)
    with pytest.raises(native.IbiscoError) as e:
        g.set_state()
    assert e.value.code == -2


def test_too_few_cells_is_reported(sysdir, tmp_path):
    """MAPS.f90's 13-cell stencil needs 3 cells per dimension."""
    import shutil
    d = str(tmp_path / "coarse")
    shutil.copytree(sysdir("fluid"), d)
    ctl = open(d + "/control").read().replace("neighbour_list_cutoff      1.4", "neighbour_list_cutoff      2.9")
    open(d + "/control", "w").write(ctl)
    g = native.System(native.Setup(d), native.IBG_PREC_FP32_FIXED)
    with pytest.raises(native.IbiscoError) as e:
        g.set_state()
    assert e.value.code == -6


@pytest.mark.parametrize("name", ["melt", "mix5_mts", "mix_npt"])
def test_programmatic_launches_change_no_trajectory(sysdir, name):
    """A graph-replayed step starts each kernel of a stream by programmatic
    dependent launch and runs the bonded branch on a second stream; timing
    mode launches the same kernels in the ordinary way on one stream.  The
    fixed-point sums make the two trajectories identical bit for bit, list
    rebuilds included."""
    d = sysdir(name)
    _, a = make(d, native.IBG_PREC_FP32_FIXED)
    _, b = make(d, native.IBG_PREC_FP32_FIXED)
    b.set_timing(True)
    oa, ob = a.run(1, 30, observe=True), b.run(1, 30, observe=True)
    sa, sb = a.state64(), b.state64()
    for k in ("sxyz", "vxyz", "fxyz"):
        assert np.array_equal(sa[k], sb[k]), k
    assert oa == ob


def test_tuning_changes_no_trajectory(sysdir):
    """Forces are exact integer sums and FP32 energies are summed per work unit,
    so every launch tuning gives the same trajectory and observables;
    autotuning times candidates without touching the state."""
    d = sysdir("mix5_mts")
    _, a = make(d, native.IBG_PREC_FP32_FIXED)
    _, b = make(d, native.IBG_PREC_FP32_FIXED)
    _, c = make(d, native.IBG_PREC_FP32_FIXED)
    _, w = make(d, native.IBG_PREC_FP32_FIXED)
    best, cands = a.autotune(reps=3)
    assert len(cands) >= 2 and all(us > 0 for _, us in cands)
    assert a.tuning() == best
    c.set_tuning(nb_tables_smem=1 - best["nb_tables_smem"], nb_blocks_per_sm=2,
                 nb_chunk=16 if best["nb_chunk"] == 0 else 0, nb_rows=8 if best["nb_rows"] == 16 else 16)
    # runs of two units dealt to the blocks in turn
    w.set_tuning(nb_tables_smem=0, nb_blocks_per_sm=0, nb_chunk=24, nb_rows=8, nb_window=2)
    oa, ob, oc = a.run(1, 20, observe=True), b.run(1, 20, observe=True), c.run(1, 20, observe=True)
    ow = w.run(1, 20, observe=True)
    sa, sb, sc, sw = a.state64(), b.state64(), c.state64(), w.state64()
    for k in ("sxyz", "vxyz", "fxyz"):
        assert np.array_equal(sa[k], sb[k]) and np.array_equal(sb[k], sc[k]) and np.array_equal(sa[k], sw[k])
    assert oa == ob == oc == ow


def make_form(d, form):
    s = native.Setup(d)
    g = native.System(s, native.IBG_PREC_FP32_FIXED)
    g.set_list_form(form)
    g.set_state()
    assert g.list_form() == form
    return s, g


@pytest.mark.parametrize("name", ["melt", "mix4", "mix5_mts", "mix_nve", "hybrid"])
def test_list_forms_agree(sysdir, name):
    """The slice lists (each neighbour once per slice of four slots, with a mask
    of its pairs) hold exactly the per-particle lists' pairs: the exported
    LIST and NNEBS are identical, every force sum is the same integer, so the
    trajectory is the same bit for bit; only the order of the FP32 energy and
    virial partial sums differs."""
    d = sysdir(name)
    _, a = make_form(d, native.LIST_PER_PARTICLE)
    _, b = make_form(d, native.LIST_PER_SLICE)
    for which in (0, 1):
        la, na = a.neighbour_list(which)
        lb, nb = b.neighbour_list(which)
        np.testing.assert_array_equal(na, nb)
        np.testing.assert_array_equal(la, lb)
    fa, fb = a.forces(1), b.forces(1)
    assert np.array_equal(a.state64()["fxyz"], b.state64()["fxyz"])
    # FP32 partial sums in another order: within the energy tolerance
    for k in ("V_NB1", "V_NB2", "V_NB3"):
        assert fa[k] == pytest.approx(fb[k], rel=ENERGY_TOL, abs=1e-9), k
    a.set_state()
    b.set_state()
    oa, ob = a.run(1, 25, observe=True), b.run(1, 25, observe=True)
    sa, sb = a.state64(), b.state64()
    for k in ("sxyz", "vxyz", "fxyz"):
        assert np.array_equal(sa[k], sb[k]), k
    for x, y in zip(oa, ob):
        for k in ("V_NB1", "V_NB2", "V_NB3"):
            assert x[k] == pytest.approx(y[k], rel=ENERGY_TOL, abs=1e-9), k


def test_list_form_switch_needs_a_new_state(sysdir):
    d = sysdir("melt")
    # the automatic form takes slice lists only from 2*64*32 particles per SM
    _, auto = make(d, native.IBG_PREC_FP32_FIXED)
    assert auto.list_form() == native.LIST_PER_PARTICLE
    _, g = make_form(d, native.LIST_PER_SLICE)
    g.set_list_form(native.LIST_PER_PARTICLE)
    with pytest.raises(native.IbiscoError):
        g.run(1, 2)
    g.set_state()
    g.run(1, 2)
    s64 = native.System(native.Setup(d), native.IBG_PREC_FP64_PLAIN)
    assert s64.list_form() == native.LIST_PER_PARTICLE
    with pytest.raises(native.IbiscoError):
        s64.set_list_form(native.LIST_PER_SLICE)
