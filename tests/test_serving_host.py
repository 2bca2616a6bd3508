"""Host logic of the served stream (no GPU): splitting a stream over ranks,
the serial schedule of the comparison path, latency statistics, and the
gathering of per-rank records over a 2-rank gloo process group."""
import os
import socket

import numpy as np
import pytest

from ibisco_b200 import serving, synth


def jobs_of(n=40, seed=3):
    st = synth.job_stream(n, seed=seed)
    return [serving.JobSpec(k, t, f"/nonexistent/{k}", 2000, size) for k, (t, size, _) in enumerate(st)]


@pytest.mark.parametrize("world", [1, 2, 3, 4])
def test_partition_covers_each_job_once_and_balances(world):
    jobs = jobs_of()
    parts = [serving.partition(jobs, r, world) for r in range(world)]
    got = sorted(j.index for p in parts for j in p)
    assert got == list(range(len(jobs)))
    loads = [sum(j.particles * j.nsteps for j in p) for p in parts]
    biggest = max(j.particles * j.nsteps for j in jobs)
    assert max(loads) - min(loads) <= biggest


def test_job_stream_sizes_and_arrivals():
    st = synth.job_stream(512, seed=5)
    sizes = np.array([s for _, s, _ in st])
    t = np.array([a for a, _, _ in st])
    assert sizes.min() >= 500 and sizes.max() <= 50000
    assert np.all(np.diff(t) >= 0) and t[0] == 0.0
    rate = (len(t) - 1) / t[-1]
    assert 15.0 < rate < 25.0  # Poisson at 20 jobs/s
    # log-uniform: the median is near the geometric mean of the bounds
    assert 3000 < np.median(sizes) < 8000


def test_serial_schedule_queues_in_arrival_order():
    done = serving.serial_schedule([0.0, 0.1, 5.0], [1.0, 1.0, 0.5])
    assert done == [1.0, 2.0, 5.5]


def test_summarize_latency_and_throughput():
    rec = [(0.0, 1.0), (0.5, 2.5), (1.0, 4.0)]
    s = serving.summarize(rec, atom_steps=4000.0)
    assert s["jobs"] == 3
    assert s["span_s"] == 4.0 and s["jobs_per_s"] == 0.75 and s["atom_steps_per_s"] == 1000.0
    assert s["p50_s"] == 2.0 and abs(s["p99_s"] - 2.98) < 1e-9


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        jobs = serving.partition(jobs_of(12), rank, world)
        records = [(j.arrival_s, j.arrival_s + 1.0 + rank) for j in jobs]
        merged = serving.merge(dist, records)
        q.put((rank, sorted(merged), len(jobs)))
    finally:
        dist.destroy_process_group()


def test_merge_over_two_gloo_ranks():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    assert out[0][1] == out[1][1]            # every rank sees all records
    assert len(out[0][1]) == 12              # each job exactly once
    assert out[0][2] + out[1][2] == 12
