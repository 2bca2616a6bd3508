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
