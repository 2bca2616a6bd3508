"""Driving a served job stream: arrivals, partitioning over GPUs, statistics.

The serving loop itself is native (``ibg_server_*`` in the library): it
admits jobs by device-memory footprint, keeps them resident and steps them as
one batch with continuous admission.  This module replays a stream of
arrivals against it in wall-clock time, splits a stream over ranks (one GPU
per rank, jobs are independent, so there is no collective on the data path)
and computes the latency percentiles and throughput of a stream, for the
served form and for the same jobs run one after another on the plain path.
"""
from __future__ import annotations

import os
import time
from dataclasses import dataclass

import numpy as np


@dataclass
class JobSpec:
    index: int         # position in the stream
    arrival_s: float   # seconds after the stream starts
    directory: str     # system input files
    nsteps: int
    particles: int


def partition(jobs, rank: int, world: int):
    """Jobs of one rank: a greedy split in arrival order that gives each job to
    the rank with the least particle-steps so far.  Every rank computes the
    same split."""
    load = [0.0] * world
    mine = []
    for j in sorted(jobs, key=lambda j: j.index):
        r = int(np.argmin(load))
        load[r] += j.particles * j.nsteps
        if r == rank:
            mine.append(j)
    return mine


def percentiles(latencies):
    lat = np.asarray(latencies, float)
    if lat.size == 0:
        return {"p50_s": None, "p99_s": None, "mean_s": None}
    return {"p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "mean_s": float(lat.mean())}


def summarize(records, atom_steps: float):
    """records: [(arrival_s, done_s)] of completed jobs on one clock."""
    if not records:
        return {"jobs": 0}
    arr = np.array([r[0] for r in records])
    done = np.array([r[1] for r in records])
    span = float(done.max() - arr.min())
    out = {"jobs": len(records), "span_s": span, "jobs_per_s": len(records) / span if span > 0 else None,
           "atom_steps_per_s": atom_steps / span if span > 0 else None}
    out.update(percentiles(done - arr))
    return out


def serial_schedule(arrivals, service_s):
    """Completion times of jobs served one at a time in arrival order, given
    each job's service time: done_k = max(arrival_k, done_{k-1}) + service_k."""
    done, t = [], 0.0
    for a, s in zip(arrivals, service_s):
        t = max(t, a) + s
        done.append(t)
    return done


def replay(server, jobs, time_scale: float = 1.0):
    """Submit each job at its arrival time (scaled), wait for all; returns
    [(arrival_s, done_s)] in stream-clock seconds and the job ids.  A job's
    latency runs from its scheduled arrival to its completion, so it includes
    reading its input files (ibg_setup_read, on this thread before the
    submission) and any lag of the submission behind the schedule, as the
    serial baseline's service time includes its setup."""
    t0 = time.perf_counter()
    ids = []
    for j in sorted(jobs, key=lambda j: j.arrival_s):
        wait = j.arrival_s * time_scale - (time.perf_counter() - t0)
        if wait > 0:
            time.sleep(wait)
        ids.append((j, server.submit(j.directory, j.nsteps)))
    server.drain()
    records = []
    for j, jid in ids:
        r = server.result(jid)
        records.append((j.arrival_s * time_scale, r["submitted_at"] - t0 + r["latency_s"]))
    return records, ids


def merge(pg, records):
    """All ranks' completion records (one clock per rank, each starting at its
    stream's start) gathered on every rank."""
    if pg is None:
        return list(records)
    out = [None] * pg.get_world_size()
    pg.all_gather_object(out, list(records))
    return [r for part in out for r in part]


def stream_dirs(base: str, stream, nsteps: int):
    """Write the systems of a stream [(arrival_s, n_target, seed)] under base."""
    from . import synth

    jobs = []
    for k, (t, n, seed) in enumerate(stream):
        d = os.path.join(base, f"job{k:04d}")
        spec = synth.serving_job(seed, n, nsteps=nsteps)
        synth.write_system(spec, d)
        jobs.append(JobSpec(k, t, d, nsteps, spec.pos.shape[0]))
    return jobs
