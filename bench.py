#!/usr/bin/env python
"""Benchmark of the B200 force-and-integrate step (one JSON line on rank 0).

Workload (default): the CG melt of the roofline study (melt2m) -- 10,000
chains x 200 beads (2,000,000 beads, 4 types), tabulated bond and angle
terms, ten LJ tables to 1.4 nm (list 1.6 nm, rebuilt every 10 steps), NVT at
300 K, dt 10 fs; seeded synthetic input written in the reference's file
formats.  A step is one loop body of NEW_LOOP.F90 (SHIFT, list rebuild when
due, nonbonded + bonded forces, MOVE, Berendsen scaling).  --workload picks
the other configurations (melt40k, fluid4k, hybrid3a, hybrid3b).

Legs:
  value      device time (CUDA events on the library's stream) of K steps
             replayed as CUDA graphs, state resident in HBM, L2 flushed
             before each step (a 256 MiB write, outside the timed interval);
  e2e        wall time through the C ABI with host buffers: ibg_set_state
             from page-locked host arrays, K x ibg_step with its observables
             read back each step, ibg_get_state into page-locked arrays at
             the end (the L2 flush before each step stays outside the timed
             intervals);
  fp64_plain the same K steps on the plain FP64 path (comparison path);
  batched    the first B jobs of the served stream (mixed sizes) stepped as
             one batch (ibg_batch: one launch per stage over all systems, one
             CUDA graph per batch step), against the same systems run one
             after another on the plain FP64 and FP32 single-system paths;
  serving    the seeded stream of 512 jobs of mixed sizes with Poisson
             arrivals, replayed against the continuous-batching server
             (ibg_server), p50/p99 latency and jobs/s, against the same jobs
             run one after another on the plain FP64 path; latencies run
             from the scheduled arrival and include reading the job's files;
  roofline   nonbonded kernel, the dominant launch: algorithmic bytes per
             launch (16 B position + 4 B per listed pair, per particle) over its
             event-timed average duration, against the measured HBM copy peak;
  cpu_baseline  the oracle (C++ restatement of the reference, OpenMP) on this
             host's cores over a bounded sample of the same workload;
  clocks     SM clock and clock-event reasons polled through NVML over the
             warm-up and the timed region.

--impl reference times that CPU restatement alone (the reference itself is
Fortran and no Fortran compiler is available here or on the GPU host).
Multi-GPU (torchrun): one independent replica per GPU, weak scaling, timing =
max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    "melt40k": "bead-spring melt: 400 chains x 100 beads (40,000), 3 types, bond/angle/torsion tables, "
               "6 LJ tables rc 1.0 nm, list 1.2 nm every 10 steps, NVT 500 K, dt 1 fs",
    "fluid4k": "single-type LJ fluid: 4,000 beads, rho 8/nm^3, overlaps rejected below 0.42 nm, rc 1.2 nm, "
               "list 1.4 nm every 10 steps, NVE, dt 10 fs",
    "melt2m": "CG melt: 10,000 chains x 200 beads (2,000,000), 4 types, bond/angle tables, 10 LJ tables "
              "rc 1.4 nm, list 1.6 nm every 10 steps, NVT 300 K, dt 10 fs",
    "hybrid3a": "hybrid melt as specified: 200 atomistic chains x 20 monomers x 12 atoms (48,000) with a "
                "centre-of-mass virtual site per monomer (4,000); atom tables rc 1.0 nm, site tables rc 1.4 nm "
                "(no pair reaches them: sites pair with neither atoms nor sites), MTS 9, NVT 300 K, dt 1 fs",
    "hybrid3b": "hybrid melt with a CG half: 100 atomistic chains x 20 monomers x 12 atoms (24,000) with a "
                "centre-of-mass virtual site per monomer (2,000) and 100 CG chains x 20 beads (2,000); atom tables "
                "rc 1.0 nm, bead/site tables rc 1.4 nm, MTS 9 (CG nonbonded on 3 of 12 steps), NVT 300 K, dt 1 fs",
}


def make_workload(name: str, directory: str):
    from ibisco_b200 import synth

    if name == "melt40k":
        spec = synth.polymer_melt(nchains=400, nper=100, seed=2)
    elif name == "fluid4k":
        # overlap rejection below 0.42 nm: at 0.3 nm (sigma 0.47 nm, dt 10 fs) the
        # REAL*4 restatement of the reference itself diverges within 10 steps
        spec = synth.lj_fluid(n=4000, seed=1, dmin=0.42)
    elif name == "melt2m":
        spec = synth.cg_melt()
    elif name == "hybrid3a":
        spec = synth.hybrid_melt(n_atomistic=200, n_cg=0)
    elif name == "hybrid3b":
        spec = synth.hybrid_melt(n_atomistic=100, n_cg=100)
    else:
        raise SystemExit(f"unknown workload {name}")
    synth.write_system(spec, directory)
    return spec


class Clocks:
    """SM clock and clock-event reasons of this rank's GPU, polled through
    NVML every 5 ms from a thread (read-only queries), or with nvidia-smi at
    200 ms where NVML cannot be loaded.  mark(True)/mark(False) bracket the
    timed region; summary() reports the samples inside it and, beside them,
    those of the whole window the sampler ran (warm-up and timed region),
    which a short timed region needs for a median under load."""

    FIELDS = "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active," \
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown," \
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"
    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.samples = []      # (t, sm_mhz, reasons)
        self.max_mhz = None
        self.marks = [None, None]
        self._stop = threading.Event()
        self.t = None
        self.proc = None
        self.source = None

    def _nvml_handle(self):
        import pynvml
        import torch

        pynvml.nvmlInit()
        try:
            p = torch.cuda.get_device_properties(self.gpu)
            return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(
                f"{p.pci_domain_id:08x}:{p.pci_bus_id:02x}:{p.pci_device_id:02x}.0")
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.gpu)

    def _poll_nvml(self, nv, h):
        bits = {"hw_slowdown": nv.nvmlClocksEventReasonHwSlowdown,
                "hw_thermal_slowdown": nv.nvmlClocksEventReasonHwThermalSlowdown,
                "sw_thermal_slowdown": nv.nvmlClocksEventReasonSwThermalSlowdown,
                "sw_power_cap": nv.nvmlClocksEventReasonSwPowerCap}
        while not self._stop.is_set():
            try:
                mhz = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                self.samples.append((time.perf_counter(), float(mhz), {k for k, b in bits.items() if r & b}))
            except Exception:
                pass
            self._stop.wait(0.005)

    def _read_smi(self):
        for line in self.proc.stdout:
            p = [x.strip() for x in line.split(",")]
            if len(p) < 9:
                continue
            try:
                mhz, self.max_mhz = float(p[1]), float(p[2])
            except ValueError:
                continue
            self.samples.append((time.perf_counter(), mhz,
                                 {n for k, n in enumerate(self.NAMES) if p[5 + k].lower() == "active"}))

    def __enter__(self):
        try:
            nv, h = self._nvml_handle()
            self.max_mhz = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            self.source = "nvml, 5 ms"
            self.t = threading.Thread(target=self._poll_nvml, args=(nv, h), daemon=True)
            self.t.start()
            return self
        except Exception:
            pass
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.gpu)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.source = "nvidia-smi, 200 ms"
            self.t = threading.Thread(target=self._read_smi, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def mark(self, begin: bool):
        self.marks[0 if begin else 1] = time.perf_counter()

    def __exit__(self, *a):
        self._stop.set()
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if self.t:
            self.t.join(timeout=2)

    def summary(self):
        def stats(rows):
            sm = [r[1] for r in rows]
            return (float(np.median(sm)) if sm else None), sorted(set().union(*[r[2] for r in rows])), len(rows)

        b, e = self.marks
        timed = [r for r in self.samples if b is not None and e is not None and b <= r[0] <= e]
        sm_t, rs_t, n_t = stats(timed)
        sm_w, rs_w, n_w = stats(self.samples)
        out = {"sm_mhz": sm_t if n_t else sm_w, "sm_max_mhz": self.max_mhz, "reasons": sorted(set(rs_t) | set(rs_w)),
               "samples": n_t, "window_samples": n_w, "window_sm_mhz": sm_w, "source": self.source}
        if self.samples:
            out["window_s"] = self.samples[-1][0] - self.samples[0][0]
        return out


def workload_config(args, n: int) -> dict:
    """The workload as both arms name it (the same dict on the reference arm)."""
    cfg = {"workload": args.workload, "description": WORKLOADS[args.workload], "particles": n}
    if args.vs_com == "reference":
        cfg["virtual_sites"] = "reference centre-of-mass form (VIRTUAL_DEF.f90:31 resets only the x sum)"
    if args.list_form == "slice":
        cfg["verlet_lists"] = "FP32 path: one list per slice of four slots, a pair mask per neighbour"
    elif args.list_form == "per-particle":
        cfg["verlet_lists"] = "FP32 path: one list per particle"
    return cfg


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ncu_traffic(workload: str, slice_lists: bool):
    """DRAM bytes (read + write) per nonbonded launch of this workload and
    list form, from its committed ncu summary (a 'dram_bytes_per_launch: <n>'
    line), or None where no capture of this workload exists."""
    kernel = "nonbonded_slices" if slice_lists else "nonbonded"
    p = os.path.join(ROOT, "profiles", f"{kernel}_{workload}.md")
    if not os.path.exists(p):
        return None
    m = re.search(r"dram_bytes_per_launch:\s*([0-9.eE+]+)", open(p).read())
    return float(m.group(1)) if m else None


def cpu_baseline(directory: str, n_particles: int, budget_s: float = 20.0, max_steps: int = 100000):
    """Oracle (OpenMP) on this host's cores: init, one warm-up step, then steps
    until the time budget is used."""
    from oracle import oracle as orc

    threads = os.cpu_count() or 1
    o = orc.Oracle(directory, threads=threads, com_fix=VS_COM["form"] != "reference")
    o.init(0)
    o.step(1, 0)
    t0 = time.perf_counter()
    k = 0
    while k < max_steps:
        o.step(2 + k, 0)
        k += 1
        if time.perf_counter() - t0 > budget_s:
            break
    dt = time.perf_counter() - t0
    return {"value": n_particles * k / dt, "unit": "atom-steps/s", "cores": threads, "kind": "port",
            "sample": f"{k} steps of the full {n_particles}-particle workload after 1 warm-up step "
                      f"({dt:.1f} s, REAL*4 restatement of the reference, OpenMP {threads} threads)"}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        pg = dist
    return world, rank, local, pg


def reduce_max(pg, x: float) -> float:
    if pg is None:
        return x
    import torch

    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def barrier(pg):
    if pg is not None:
        pg.barrier()


def run_reference(args, world, rank, pg):
    if rank != 0:
        return
    with tempfile.TemporaryDirectory() as d:
        make_workload(args.workload, d)
        from oracle import oracle as orc

        threads = os.cpu_count() or 1
        o = orc.Oracle(d, threads=threads, com_fix=VS_COM["form"] != "reference")
        n = o.info["NATOMS"]
        o.init(0)
        for k in range(min(args.warmup, 5)):
            o.step(1 + k, 0)
        # bounded sample: the requested steps, or as many as fit in 240 s
        # (melt2m takes about 2 s a step on 16 cores)
        t0 = time.perf_counter()
        done = 0
        for k in range(args.steps):
            o.step(1 + min(args.warmup, 5) + k, 0)
            done += 1
            if time.perf_counter() - t0 > 240.0:
                break
        el = time.perf_counter() - t0
        value = n * done / el
        line = {"impl": "reference", "metric": "atom-steps/s", "value": value, "unit": "atom-steps/s",
                "n_gpus": world, "steps": done, "warmup": args.warmup, "ms_per_step": 1000 * el / done,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic", "config": workload_config(args, n),
                "cpu_baseline": {"value": value, "unit": "atom-steps/s", "cores": threads, "kind": "port",
                                 "sample": f"{done} of {args.steps} requested steps in {el:.1f} s after {min(args.warmup, 5)} "
                                           f"warm-up steps (C++ REAL*4 restatement of the reference, OpenMP "
                                           f"{threads} threads; no Fortran compiler here)"},
                "e2e": {"value": value, "unit": "atom-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)


def stream_jobs(args, workdir):
    """The seeded served job stream (sizes log-uniform in 500..50,000 beads,
    1-3 types, chains of 10-100, per-job perturbed LJ tables, Poisson arrivals
    at 20 jobs/s), written once in the reference's input format; the batched
    leg takes its first jobs, the serving leg all of them."""
    from ibisco_b200 import serving, synth

    njobs = max(args.serve_jobs, args.batch_jobs)
    stream = synth.job_stream(njobs, seed=5)
    return serving.stream_dirs(os.path.join(workdir, "stream"), stream, args.serve_steps)


def run_serving(args, world, rank, local, pg, jobs):
    """Served job stream: the first J jobs of the seeded stream, replayed in
    wall-clock time against the continuous-batching server; then the same jobs
    one after another on the plain FP64 path, served in arrival order (computed
    from the measured per-job times).  Both latencies run from a job's
    scheduled arrival and include reading its input files.  Jobs are split over
    ranks (no collective on the data path); latencies and throughput are over
    all ranks."""
    from ibisco_b200 import native, serving

    jobs = jobs[: args.serve_jobs]
    mine = serving.partition(jobs, rank, world)
    barrier(pg)
    srv = native.Server(device=local, tick_steps=args.serve_tick, max_jobs=256)
    records, ids = serving.replay(srv, mine)
    st = srv.stats()
    srv.close()
    atom_steps = float(sum(j.particles * j.nsteps for j in mine))
    # plain FP64 path, one job at a time
    service = []
    for j in sorted(mine, key=lambda j: j.arrival_s):
        t0 = time.perf_counter()
        g = native.System(native.Setup(j.directory), native.IBG_PREC_FP64_PLAIN)
        g.set_state()
        g.run(1, j.nsteps)
        g.state()
        g.close()
        service.append(time.perf_counter() - t0)
    arr = [j.arrival_s for j in sorted(mine, key=lambda j: j.arrival_s)]
    serial = list(zip(arr, serving.serial_schedule(arr, service)))
    all_served = serving.merge(pg, records)
    all_serial = serving.merge(pg, serial)
    total_as = reduce_sum(pg, atom_steps)
    out = {"jobs": len(all_served),
           "stream": f"{'all' if args.serve_jobs >= 512 else 'first ' + str(args.serve_jobs) + ' of the'} "
                     f"{len(jobs) if args.serve_jobs >= 512 else 512} jobs of the seeded 20 jobs/s stream",
           "steps_per_job": args.serve_steps, "tick_steps": args.serve_tick,
           "latency": "from the scheduled arrival to completion, including ibg_setup_read of the job's files",
           "served": serving.summarize(all_served, total_as),
           "serial_fp64_plain": serving.summarize(all_serial, total_as),
           "server": {k: st[k] for k in ("peak_jobs", "peak_bytes", "budget_bytes", "ticks", "batch_builds", "gpu_s")}}
    s_, p_ = out["served"], out["serial_fp64_plain"]
    if s_.get("jobs_per_s") and p_.get("jobs_per_s"):
        out["jobs_per_s_ratio"] = s_["jobs_per_s"] / p_["jobs_per_s"]
        out["p99_ratio"] = p_["p99_s"] / s_["p99_s"]
    return out


BATCH_CANDIDATES = [dict(nb_tables_smem=0, nb_blocks_per_sm=0, nb_chunk=ch, nb_rows=rows)
                    for rows in (8, 16) for ch in (0, 24, 48)]


def run_batched_mixed(args, world, local, pg, jobs):
    """The batched form on systems of mixed size: the first B jobs of the
    served stream stepped together (FP32/fixed point, one launch per stage over
    all systems, one CUDA graph per batch step, tuned by timing short batch
    runs), against the same systems run one after another on the plain FP64
    single-system path and on the FP32/fixed-point single-system path.  Device
    time (CUDA events on each path's stream), state resident, K steps after W
    warm-up steps on every path; the L2 is not flushed (the batch's working set
    exceeds it; a small system alone fits in it, which favours the
    single-system paths)."""
    from ibisco_b200 import native

    sel = jobs[: args.batch_jobs]
    setups = [native.Setup(j.directory) for j in sel]
    n_tot = sum(j.particles for j in sel)
    K, W = args.batch_steps, args.warmup

    def make_systems():
        out = []
        for st in setups:
            g = native.System(st, native.IBG_PREC_FP32_FIXED)
            g.set_state()
            out.append(g)
        return out

    btuned, btimes = native.tune_batch(make_systems, BATCH_CANDIDATES, steps=50)
    systems = make_systems()
    for g in systems:
        g.set_tuning(**btuned)
    bat = native.Batch(systems)
    with Clocks(local) as clk:
        bat.run(W)
        barrier(pg)
        clk.mark(True)
        bat.run(K)
        clk.mark(False)
    bms = reduce_max(pg, bat.timing()["run_ms"])
    launches = bat.timing()["launches"]
    bat.close()
    for g in systems:
        g.close()
    bval = world * n_tot * K / (bms / 1000.0)

    def single(prec):
        total = 0.0
        for st in setups:
            g = native.System(st, prec)
            g.set_state()
            g.run(1, W)
            g.run(1 + W, K)
            total += g.timing()["run_ms"]
            g.close()
        total = reduce_max(pg, total)
        return world * n_tot * K / (total / 1000.0), total / K

    v64, ms64 = single(native.IBG_PREC_FP64_PLAIN)
    v32, ms32 = single(native.IBG_PREC_FP32_FIXED)
    sizes = [j.particles for j in sel]
    return {"systems": len(sel), "particles": n_tot, "sizes": {"min": min(sizes), "max": max(sizes),
                                                               "median": float(np.median(sizes))},
            "workload": "first jobs of the seeded served stream (sizes log-uniform in 500..50,000 beads, 1-3 types, "
                        "chains of 10-100, per-job perturbed LJ tables, dt 10 fs)",
            "steps": K, "warmup": W, "value": bval, "unit": "atom-steps/s", "ms_per_batch_step": bms / K,
            "tuning": btuned, "candidates_us_per_batch_step": [[t, u] for t, u in btimes],
            "fp64_plain_single": {"value": v64, "ms_per_step_all_systems": ms64},
            "fp32_fixed_single": {"value": v32, "ms_per_step_all_systems": ms32},
            "ratio_over_fp64_plain_single": bval / v64, "ratio_over_fp32_fixed_single": bval / v32,
            "gpu_launches": launches, "clocks": clk.summary(),
            "l2": "not flushed (the batch's working set exceeds the 126 MB L2; single small systems fit in it)"}


def reduce_sum(pg, x: float) -> float:
    if pg is None:
        return x
    import torch

    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    pg.all_reduce(t)
    return float(t.item())


TUNING_KEYS = ("nb_tables_smem", "nb_blocks_per_sm", "nb_chunk", "nb_rows", "nb_window")
VS_COM = {"form": "fixed"}  # --vs-com
LIST_FORM = {"form": "auto"}  # --list-form


def new_system(native, setup, prec):
    """A system of the benchmark workload, with the centre-of-mass form of its
    virtual sites as --vs-com selects."""
    g = native.System(setup, prec)
    if VS_COM["form"] == "reference":
        g.set_vsite_com(native.IBG_VS_COM_REFERENCE)
    if LIST_FORM["form"] != "auto" and prec == native.IBG_PREC_FP32_FIXED:
        g.set_list_form(native.LIST_PER_SLICE if LIST_FORM["form"] == "slice" else native.LIST_PER_PARTICLE)
    return g


def precision_report(native, setup, state):
    """Error of the FP32/fixed-point path against the plain FP64 GPU path on
    the same state: the force stage of step 1 on both paths (ibg_forces),
    max-norm relative error of the total force over particles, and the
    relative error of each nonzero energy and virial term."""
    out = {}
    for name, prec in (("fp32", native.IBG_PREC_FP32_FIXED), ("fp64", native.IBG_PREC_FP64_PLAIN)):
        g = new_system(native, setup, prec)
        g.set_state(*state)
        obs = g.forces(1)
        out[name] = (obs, g.state64()["fxyz"])
        g.close()
    (o32, f32), (o64, f64) = out["fp32"], out["fp64"]
    ferr = float(np.abs(f32 - f64).max() / np.abs(f64).max())
    energies = {k: abs(o32[k] - v) / abs(v) for k, v in o64.items() if k.startswith("V_") and abs(v) > 0}
    # the virial tensor as a whole, max-norm like the forces: an off-diagonal
    # term that vanishes by symmetry has no meaningful error of its own
    pt = [k for k in ("PT11", "PT22", "PT33", "PT12", "PT13", "PT23") if k in o64]
    w64 = np.array([o64[k] for k in pt])
    w32 = np.array([o32[k] for k in pt])
    verr = float(np.abs(w32 - w64).max() / np.abs(w64).max()) if len(pt) and np.abs(w64).max() > 0 else 0.0
    return {"reference": "plain FP64 GPU path, same state, force stage of step 1",
            "force_max_rel_err": ferr, "force_tolerance": 1e-5,
            "energy_rel_err_max": max(energies.values()) if energies else 0.0,
            "energy_rel_err": energies,
            "virial_max_norm_rel_err": verr,
            "choices": {"displacements": "32-bit box fractions from the FP64 state, wrapped integer difference",
                        "pair_math": "FP32 table interpolation and rsqrt",
                        "cutoff": "FP32 r^2; pairs within 1e-6 of rc^2 decided from the FP64 state",
                        "force_sums": "int64 fixed point, 2^-32 per pair contribution (exact, order-independent sums)",
                        "energy_virial_sums": "FP32 over 8 list rows, then int64 fixed point at 2^-24",
                        "integration": "FP64 (positions, velocities, momentum removal, thermostat, barostat)"}}


def pick_tuning(native, g, setup, prec, state, flush, reps=20, top=6):
    """Launch tuning of the nonbonded kernel: rank the candidates by their
    launches alone (ibg_autotune, L2 flushed before each), then time whole
    steps of the `top` fastest on fresh systems and apply the fastest to g.
    Returns (tuning, [(candidate, us per launch)], [(candidate, us per step)])."""
    _, cands = g.autotune(reps=reps)
    best = [dict(zip(TUNING_KEYS, c)) for c, _ in sorted(cands, key=lambda t: t[1])[:top]]

    def make_one():
        x = new_system(native, setup, prec)
        x.set_state(*state)
        return x

    n = state[0].shape[0]
    tuned, steps = native.tune_steps(make_one, best, steps=100 if n < 500000 else 20, l2_flush=flush)
    g.set_tuning(**tuned)
    return tuned, cands, steps


def run_b200(args, world, rank, local, pg):
    import ctypes

    from ibisco_b200 import native

    native.lib()
    native.lib().ibg_set_device(local)
    with tempfile.TemporaryDirectory() as d:
        make_workload(args.workload, d)
        setup = native.Setup(d)
        s0, v0, b0 = setup.initial_state()
        n = s0.shape[0]
        nitems = len(setup.array("ITYPE"))
        dt_ps = next(float(l.split()[1]) for l in open(os.path.join(d, "control")) if l.split()[0] == "time_step")
        prec = native.IBG_PREC_FP64_PLAIN if args.precision == "fp64" else native.IBG_PREC_FP32_FIXED
        g = new_system(native, setup, prec)
        g.set_state(s0, v0, b0)
        # launch tuning of the nonbonded kernel, picked by timing (state
        # unchanged), or fixed by --tuning (profiling runs)
        flush = 256 << 20
        g.set_l2_flush(flush)
        if args.tuning:
            vals = [int(x) for x in args.tuning.split(",")]
            g.set_tuning(**dict(zip(TUNING_KEYS, vals)))
            tuned, tune_cands, tune_steps = g.tuning(), [], []
        else:
            tuned, tune_cands, tune_steps = pick_tuning(native, g, setup, prec, (s0, v0, b0), flush)
        # ---- warm-up (captures the CUDA graphs) and device-timed region, with
        # the clock sampler running over both
        with Clocks(local) as clk:
            g.run(1, args.warmup)
            barrier(pg)
            l0 = g.timing()["launches"]
            clk.mark(True)
            g.run(1 + args.warmup, args.steps)
            clk.mark(False)
        tm = g.timing()
        launches = tm["launches"] - l0
        ms = reduce_max(pg, tm["run_ms"])
        barrier(pg)
        value = world * n * args.steps / (ms / 1000.0)
        # ---- roofline of the nonbonded kernel (event-timed stage pass)
        g.set_l2_flush(flush)
        g.set_timing(True)
        k_roof = min(args.steps, 200)
        g.run(1 + args.warmup + args.steps, k_roof)
        t2 = g.timing()
        g.set_timing(False)
        # algorithmic bytes of every nonbonded launch of the pass: 16 B of own
        # position per particle of the list plus 4 B per listed pair
        lists = {}
        for w in (0, 1):
            nn = g.neighbour_counts(w)
            if len(nn):
                lists[w] = (len(nn), float(nn.sum()))
        nlaunch = {1: t2["nonbonded_bead_launches"]}
        nlaunch[0] = t2["nonbonded_launches"] - nlaunch[1]
        nb_bytes = sum(nlaunch[w] * (16.0 * nw + 4.0 * pw) for w, (nw, pw) in lists.items())
        nb_count = max(1, t2["nonbonded_launches"])
        nb_launch_s = t2["nonbonded_ms"] / nb_count / 1000.0
        bytes_launch = nb_bytes / nb_count
        peak, peak_kind = measured_peak()
        achieved = bytes_launch / nb_launch_s / 1e9
        slice_lists = prec == native.IBG_PREC_FP32_FIXED and g.list_form() == native.LIST_PER_SLICE
        roof = {"bound": "hbm", "kernel": "k_nonbonded_slices" if slice_lists else "k_nonbonded",
                "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": ncu_traffic(args.workload, slice_lists),
                "peak_kind": peak_kind, "launch_us": nb_launch_s * 1e6,
                "algorithmic_bytes_per_launch": bytes_launch,
                "mean_half_list": {("atom", "bead")[w]: pw / nw for w, (nw, pw) in lists.items()}}
        stage = {k: t2[k] / k_roof for k in ("list_ms", "nonbonded_ms", "bonded_ms", "integrate_ms", "other_ms")}
        # ---- end to end through the C ABI with host buffers.  The L2 is
        # flushed before every step, as in the device-timed leg, and outside
        # the wall-clock intervals: flush, synchronise the device, then time
        # the call (each ibg_step returns with its observables on the host).
        # The host arrays are page-locked (the user's buffers, filled before
        # the timed interval), so the copies run at DMA speed.
        import torch

        def pinned(shape, src=None):
            a = torch.empty(shape, dtype=torch.float32, pin_memory=True).numpy()
            a[...] = 0 if src is None else src
            return a

        sp = pinned(np.shape(s0), s0)
        vp = pinned(np.shape(v0), v0)
        bp = pinned(np.shape(b0), b0)
        out = {k: pinned((nitems, 3)) for k in ("s", "r", "f")}
        vo = pinned((n, 3))
        obs = native.IbgObs()
        L = native.lib()
        k_e2e = args.steps
        g.set_l2_flush(0)
        flush_buf = torch.empty(flush, dtype=torch.uint8, device=f"cuda:{local}")
        barrier(pg)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        g.set_state(sp, vp, bp)
        set_s = time.perf_counter() - t0
        e2e_s = set_s
        for k in range(k_e2e):
            flush_buf.fill_(k & 0xff)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            rc = L.ibg_step(g._h, 1 + k, ctypes.byref(obs))
            e2e_s += time.perf_counter() - t0
            if rc:
                raise native.IbiscoError(rc, L.ibg_last_error(g._h).decode())
        steps_s = e2e_s - set_s
        t0 = time.perf_counter()
        g._check(L.ibg_get_state(g._h, native._fp(out["s"]), native._fp(out["r"]), native._fp(vo),
                                 native._fp(out["f"])))
        get_s = time.perf_counter() - t0
        e2e_s = reduce_max(pg, e2e_s + get_s)
        del flush_buf
        h2d = (sp.nbytes + vp.nbytes + bp.nbytes) / k_e2e
        d2h = ctypes.sizeof(native.IbgObs) + (3 * out["s"].nbytes + vo.nbytes) / k_e2e
        e2e = {"value": world * n * k_e2e / e2e_s, "unit": "atom-steps/s", "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": d2h,
               "seconds": {"ibg_set_state": set_s, "ibg_step_total": steps_s, "ibg_get_state": get_s}}
        # ---- error of the FP32/fixed-point path against the plain FP64 path
        precision = None
        if prec == native.IBG_PREC_FP32_FIXED and not args.no_fp64:
            precision = precision_report(native, setup, (s0, v0, b0))
        # ---- plain FP64 path, same workload and timing
        fp64 = None
        if prec == native.IBG_PREC_FP32_FIXED and not args.no_fp64:
            g64 = new_system(native, setup, native.IBG_PREC_FP64_PLAIN)
            g64.set_state(s0, v0, b0)
            g64.set_l2_flush(flush)
            if not args.tuning:  # the comparison path gets its own best launch tuning
                pick_tuning(native, g64, setup, native.IBG_PREC_FP64_PLAIN, (s0, v0, b0), flush, reps=10)
            g64.run(1, args.warmup)
            g64.run(1 + args.warmup, args.steps)
            ms64 = reduce_max(pg, g64.timing()["run_ms"])
            fp64 = {"value": world * n * args.steps / (ms64 / 1000.0), "ms_per_step": ms64 / args.steps,
                    "ratio_fp32_fixed_over_fp64": ms64 / ms}
            g64.close()
        # ---- batched form on a mix of system sizes, and the served job stream
        jobs = None
        if prec == native.IBG_PREC_FP32_FIXED and (args.batch_jobs > 1 or args.serve_jobs > 0):
            jobs = stream_jobs(args, d)
        batched = None
        if jobs is not None and args.batch_jobs > 1:
            batched = run_batched_mixed(args, world, local, pg, jobs)
        serving = None
        if jobs is not None and args.serve_jobs > 0:
            serving = run_serving(args, world, rank, local, pg, jobs)
        cpu = None
        if rank == 0 and world == 1 and not args.no_cpu:
            cpu = cpu_baseline(d, n)
        if rank == 0:
            steps_per_s = args.steps / (ms / 1000.0)
            line = {
                "metric": "atom-steps/s", "value": value, "unit": "atom-steps/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32" if prec == native.IBG_PREC_FP32_FIXED else "f64",
                "data": "synthetic",
                "config": workload_config(args, n),
                "precision": "FP32 pair math, int64 fixed-point force sums, FP64 integration"
                if prec == native.IBG_PREC_FP32_FIXED else "FP64 throughout",
                "parallelism": f"{world} independent replica(s), one per GPU",
                "l2": "flushed before every step (256 MiB write, outside the timed interval)",
                "ns_per_day": steps_per_s * dt_ps * 1e-3 * 86400.0,
                "roofline": roof, "stage_ms_per_step": stage,
                "tuning": {"nonbonded": tuned, "candidates_us": [[list(c), u] for c, u in tune_cands],
                           "steps_us": [[t, u] for t, u in tune_steps]},
                "cpu_baseline": cpu, "e2e": e2e, "fp64_plain": fp64, "precision_vs_fp64": precision,
                "batched": batched, "serving": serving,
                "gpu_launches": launches,
                "clocks": clk.summary(),
            }
            print(json.dumps(line), flush=True)
        g.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="melt2m")
    ap.add_argument("--vs-com", choices=["fixed", "reference"], default="fixed",
                    help="centre-of-mass virtual sites: each at its centre of mass, or the reference's form "
                         "(VIRTUAL_DEF.f90:31 resets only the x sum)")
    ap.add_argument("--list-form", choices=["auto", "per-particle", "slice"], default="auto",
                    help="Verlet lists of the FP32 single-system legs: the library's choice by list size, a list "
                         "per particle, or one per slice of four slots with a pair mask per neighbour "
                         "(ibg_set_list_form)")
    ap.add_argument("--precision", choices=["fp32", "fp64"], default="fp32")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--batch-jobs", type=int, default=64,
                    help="systems of mixed size in the batched leg (0 or 1: no batched leg)")
    ap.add_argument("--batch", dest="batch_jobs", type=int, help="same as --batch-jobs")
    ap.add_argument("--batch-steps", type=int, default=200, help="steps of the batched leg and its comparisons")
    ap.add_argument("--serve-jobs", type=int, default=512, help="jobs of the served stream (0: no serving leg)")
    ap.add_argument("--tuning", default="", help="fixed nonbonded tuning 'tables_smem,blocks_per_sm,chunk[,rows[,window]]' "
                                                  "instead of the autotuner (for profiling)")
    ap.add_argument("--serve-steps", type=int, default=2000)
    ap.add_argument("--serve-tick", type=int, default=100)
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    VS_COM["form"] = args.vs_com
    LIST_FORM["form"] = args.list_form
    world, rank, local, pg = dist_setup()
    try:
        if args.impl == "reference":
            run_reference(args, world, rank, pg)
        else:
            run_b200(args, world, rank, local, pg)
    finally:
        if pg is not None:
            pg.destroy_process_group()


if __name__ == "__main__":
    main()
