"""Serving loop (ibg_server): continuous batching of jobs on one GPU.

Jobs are submitted while others run, are admitted by device-memory footprint,
and each result is bitwise the result of the same system run alone."""
import os
import time

import numpy as np
import pytest

from ibisco_b200 import native, synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def jobdirs(tmp_path_factory):
    base = tmp_path_factory.mktemp("jobs")
    out = []
    for k, n in enumerate((600, 2500, 900, 4000, 1500, 700)):
        d = str(base / f"job{k}")
        synth.write_system(synth.serving_job(1000 + k, n, nsteps=60), d)
        out.append(d)
    return out


def alone(d, nsteps):
    g = native.System(native.Setup(d), native.IBG_PREC_FP32_FIXED)
    g.set_state()
    obs = g.run(1, nsteps, observe=True)[-1]
    st = g.state()
    g.close()
    return st, obs


def test_served_results_equal_alone(jobdirs):
    nsteps = [60, 45, 60, 30, 60, 50]
    srv = native.Server(tick_steps=20, max_jobs=8)
    ids = [srv.submit(d, n) for d, n in zip(jobdirs[:3], nsteps[:3])]
    time.sleep(0.05)  # the first jobs are running when the rest arrive
    ids += [srv.submit(d, n) for d, n in zip(jobdirs[3:], nsteps[3:])]
    assert srv.drain(120.0)
    st = srv.stats()
    assert st["done"] == len(jobdirs) and st["failed"] == 0
    for jid, d, n in zip(ids, jobdirs, nsteps):
        r = srv.result(jid)
        ref, robs = alone(d, n)
        assert r["obs"]["STEP"] == n
        assert np.array_equal(r["sxyz"], ref["sxyz"])
        assert np.array_equal(r["vxyz"], ref["vxyz"])
        for key in ("EK1", "V_NB1", "V_BOND1", "PT11", "TEMP"):
            assert r["obs"][key] == robs[key]
        assert r["latency_s"] >= r["run_s"] > 0
    assert st["p99_s"] >= st["p50_s"] > 0 and st["jobs_per_s"] > 0
    srv.close()


def test_admission_by_memory_budget(jobdirs):
    """A budget that holds two or three of the jobs keeps the others queued
    until memory frees up; every job still completes.  Admission adds the
    next job's estimate (generous: about three times what a small job takes)
    to the memory the running jobs really hold, so the budget is set from the
    largest job's estimate."""
    s = native.Setup(jobdirs[3])
    _, _, box = s.initial_state()
    est = native.lib().ibg_estimate_bytes(s.desc(), native.IBG_PREC_FP32_FIXED, native._fp(box))
    assert est > 0
    srv = native.Server(tick_steps=10, max_jobs=8, hbm_budget=int(1.2 * est))
    ids = [srv.submit(d, 30) for d in jobdirs]
    assert srv.drain(120.0)
    st = srv.stats()
    assert st["done"] == len(jobdirs)
    assert st["peak_jobs"] < len(jobdirs)
    assert st["peak_bytes"] <= st["budget_bytes"]
    assert st["batch_builds"] > 1
    waited = [srv.result(j)["queued_s"] for j in ids]
    assert max(waited) > 0
    srv.close()


def test_failed_job_does_not_stop_the_others(jobdirs, tmp_path):
    import shutil
    bad = str(tmp_path / "bad")
    shutil.copytree(jobdirs[0], bad)
    ctl = open(bad + "/control").read().replace("neighbour_list_cutoff      1.2", "neighbour_list_cutoff      2.9")
    open(bad + "/control", "w").write(ctl)
    srv = native.Server(tick_steps=10)
    good = srv.submit(jobdirs[1], 20)
    badj = srv.submit(bad, 20)
    assert srv.drain(60.0)
    assert srv.wait(good, 1.0) == native.IBG_JOB_DONE
    assert srv.wait(badj, 1.0) == native.IBG_JOB_FAILED
    with pytest.raises(native.IbiscoError) as e:
        srv.result(badj)
    assert e.value.code == -6
    srv.close()


def test_served_job_from_memory_with_a_replaced_table(jobdirs, tmp_path):
    """An iterative Boltzmann inversion trial without files: the job's inputs
    are read from memory (ibg_setup_read_mem), its nonbonded table is replaced
    (ibg_setup_set_nb_table) and the setup is submitted.  Its result is bitwise
    that of the same system read from a directory whose table file holds the
    new rows, run alone."""
    import shutil

    src = jobdirs[1]
    files = {f: open(os.path.join(src, f), "rb").read() for f in os.listdir(src)}
    s = native.Setup(files=files)
    name = "nb11"  # table 1: the (1, 1) type pair of synth.serving_job
    t = synth.perturbed_lj_table(name, 0.47, 3.5, 1.2, 0.002, [0.2, 0.1, -0.1, 0.05, 0.02])
    r, v = np.asarray(t.x, np.float32), np.asarray(t.v, np.float32)
    s.set_nb_table(1, r, v)
    d2 = str(tmp_path / "trial")
    shutil.copytree(src, d2)
    with open(os.path.join(d2, name), "w") as f:
        for a, b in zip(r.astype(np.float64), v.astype(np.float64)):
            f.write("%.9g  %.9g\n" % (a, b))
    srv = native.Server(tick_steps=20, max_jobs=4)
    jid = srv.submit(s, 40)
    assert srv.drain(120.0)
    res = srv.result(jid)
    srv.close()
    ref, robs = alone(d2, 40)
    assert np.array_equal(res["sxyz"], ref["sxyz"]) and np.array_equal(res["vxyz"], ref["vxyz"])
    assert res["obs"]["V_NB1"] == robs["V_NB1"]
