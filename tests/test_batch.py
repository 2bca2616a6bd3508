"""Batched systems (ibg_batch): one launch per stage over many systems.

Each system in a batch keeps its own step counter, list schedule, MTS phase,
thermostat and barostat.  Force and nonbonded energy sums are integers and the
statically scheduled kernels keep per-system launch shapes, so a system's
trajectory, forces and observables are bitwise the same alone and in any mix.
"""
import numpy as np
import pytest

from ibisco_b200 import native

pytestmark = pytest.mark.gpu

MIX = ["melt", "mix5_mts", "fluid", "mix_npt", "mix4"]
OBS_KEYS = ("EK1", "EK2", "TEMP", "V_NB1", "V_NB2", "V_NB3", "V_BOND1", "V_ANGLE1", "V_TORSION1", "V_OOP1",
            "PT11", "PT22", "PT33", "PT12", "PT13", "PT23", "BOX1", "STEP")


def system(d):
    g = native.System(native.Setup(d), native.IBG_PREC_FP32_FIXED)
    g.set_state()
    return g


def same_state(a, b):
    sa, sb = a.state64(), b.state64()
    for k in ("sxyz", "vxyz", "fxyz"):
        assert np.array_equal(sa[k], sb[k]), k


def test_batch_equals_alone(sysdir):
    dirs = [sysdir(n) for n in MIX]
    alone = [system(d) for d in dirs]
    ref_obs = [g.run(1, 23, observe=True)[-1] for g in alone]
    mixed = [system(d) for d in dirs]
    b = native.Batch(mixed)
    obs = b.run(23, observe=True)
    for k, (g0, g1) in enumerate(zip(alone, mixed)):
        same_state(g0, g1)
        for key in OBS_KEYS:
            assert obs[k][key] == ref_obs[k][key], (MIX[k], key)


def test_batch_systems_at_different_steps_and_limits(sysdir):
    """Systems enter the batch at different steps and stop at their own last
    step; the batch continues the others."""
    dirs = [sysdir(n) for n in ("melt", "mix5_mts", "fluid")]
    alone = [system(d) for d in dirs]
    for g, last in zip(alone, (17, 30, 26)):
        g.run(1, last)
    mixed = [system(d) for d in dirs]
    mixed[1].run(1, 7)  # starts 7 steps ahead
    b = native.Batch(mixed)
    obs = b.run(12, last_step=[17, 30, 26], observe=True)
    assert [o["STEP"] for o in obs] == [12, 19, 12]
    obs = b.run(100, last_step=[17, 30, 26], observe=True)
    assert [o["STEP"] for o in obs] == [17, 30, 26]
    for g0, g1 in zip(alone, mixed):
        same_state(g0, g1)
    b.close()
    mixed[0].run(18, 3)  # usable on its own after the batch
    alone[0].run(18, 3)
    same_state(alone[0], mixed[0])


def test_batch_list_growth_of_one_system_is_exact(sysdir):
    dirs = [sysdir(n) for n in ("melt", "fluid")]
    alone = [system(d) for d in dirs]
    for g in alone:
        g.run(1, 25)
    mixed = [system(d) for d in dirs]
    b = native.Batch(mixed)
    b.run(9)
    native.lib().ibg_set_list_rows(mixed[0]._h, 1)  # step 10 rebuilds and outgrows it
    b.run(16)
    assert mixed[0].timing()["list_growths"] > 0
    for g0, g1 in zip(alone, mixed):
        same_state(g0, g1)


def test_energies_are_bitwise_reproducible(sysdir):
    d = sysdir("mix_npt")  # the barostat feeds the virial back into the positions
    a, b = system(d), system(d)
    oa = a.run(1, 30, observe=True)
    ob = b.run(1, 30, observe=True)
    assert oa == ob
    same_state(a, b)


def test_batch_mixes_list_forms(sysdir):
    """Systems with slice lists and systems with per-particle lists share a
    batch (one launch per list form and stage); each system's trajectory is
    bitwise the one it has alone in either form."""
    names = ["melt", "mix5_mts", "fluid"]
    dirs = [sysdir(n) for n in names]
    alone = [system(d) for d in dirs]
    for g in alone:
        g.run(1, 23)
    mixed = []
    for k, d in enumerate(dirs):
        g = native.System(native.Setup(d), native.IBG_PREC_FP32_FIXED)
        g.set_list_form(native.LIST_PER_SLICE if k != 1 else native.LIST_PER_PARTICLE)
        g.set_state()
        mixed.append(g)
    b = native.Batch(mixed)
    b.run(23)
    for g0, g1 in zip(alone, mixed):
        same_state(g0, g1)
