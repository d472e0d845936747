#!/usr/bin/env python
"""Benchmark of the gromos-rs nonbonded hot path on B200.

Workload (one "step" = one Forcefield::apply nonbonded evaluation): 30,000
SPC waters (90,000 atoms) in a 9.65 nm cubic box, twin-range cutoffs
0.8/1.4 nm, reaction field EPSRF 61, pairlist rebuilt every NSNB = 5 steps;
short-range pairs every step, long-range pairs (twin-range cache) at every
rebuild.  Synthetic seeded coordinates (no external data).

Metric: atom-pair interactions per second (pair-int/s) = atom pairs of the
listed charge-group pairs evaluated per step (short every step, long on
rebuild steps) / device time; ns/day follows for dt = 2 fs.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--kernel fixed|plain]
  python bench.py --impl reference ...   # CPU reference arm (FP64, all host threads)

Under torchrun each rank evaluates its own replica of the workload (the
path has no exchange step: replicas only); time = max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
for _p in (os.path.join(ROOT, "gromos-rs_b200"), os.path.join(ROOT, "tests")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

DT_PS = 0.002
OPS_PER_PAIR = 37          # FP32 pipe ops per atom pair, energies + virial step
METRIC = "pair-int/s"
WORKLOAD = "spc30000_twinrange_0.8_1.4_nsnb5"
# DRAM bytes (read + write) of one short-range water-kernel launch on this
# workload, dram__bytes_read.sum + dram__bytes_write.sum from an ncu capture of
# the first short-range launch of this script's small run (--steps 3 --warmup 3):
# 6,675,712 B read, 0 written.  A recorded constant: this run does not measure it.
SHORT_KERNEL_DRAM_BYTES = 6.675712e6


def ns_per_day(ms_per_step: float) -> float:
    return 86400.0 / (ms_per_step * 1e-3) * DT_PS * 1e-3


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = float(p[2])
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if p[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_baseline_sample(seconds_budget: float = 20.0):
    """FP64 oracle on the host's cores, bounded samples of the same workload:
    threaded (fold/reduce over all cores; the reported value) and serial (one
    core, one pairlist period; reported beside it)."""
    import oracle_binding as ob
    from gromos_nb import generators

    s = generators.config2_spc30000()
    nth = os.cpu_count() or 1
    t0 = time.perf_counter()
    orc = ob.OracleForcefield(s, nthreads=nth)
    t_build = time.perf_counter() - t0
    lists = ob.pairlist(s, algorithm=2, nthreads=nth)
    n_short = len(lists[0]) + 9 * len(lists[2])
    n_long = len(lists[1]) + len(lists[3])
    steps = 0
    pairs = 0
    t0 = time.perf_counter()
    while True:
        orc.apply(s.pos)
        pairs += n_short + (n_long if steps % s.params.nsnb == 0 else 0)
        steps += 1
        el = time.perf_counter() - t0
        if steps >= s.params.nsnb and (el > seconds_budget / 2 or steps >= 10):
            break
    el = time.perf_counter() - t0 + t_build  # the first pairlist build is part of the work
    orc.close()
    # the serial mode of the same restatement (one core): one pairlist period
    t0 = time.perf_counter()
    orc1 = ob.OracleForcefield(s, nthreads=1)
    pairs1 = 0
    for k in range(s.params.nsnb):
        orc1.apply(s.pos)
        pairs1 += n_short + (n_long if k == 0 else 0)
    el1 = time.perf_counter() - t0
    orc1.close()
    return {"value": pairs / el, "unit": METRIC, "cores": nth, "kind": "port",
            "sample": f"{steps} Forcefield::apply steps of {WORKLOAD} incl. {-(-steps // s.params.nsnb)} cell-list "
                      f"pairlist builds and long-range refreshes, FP64 C++ restatement, {nth} threads",
            "ms_per_step": 1e3 * el / steps,
            "serial": {"value": pairs1 / el1, "unit": METRIC, "cores": 1, "ms_per_step": 1e3 * el1 / s.params.nsnb,
                       "sample": f"{s.params.nsnb} Forcefield::apply steps (one pairlist period incl. its build "
                                 f"and long-range refresh), one thread"}}


def run_reference(args, rank, world):
    if rank != 0:
        return 0
    import oracle_binding as ob
    from gromos_nb import generators

    s = generators.config2_spc30000()
    nth = os.cpu_count() or 1
    lists = ob.pairlist(s, algorithm=2, nthreads=nth)
    n_short = len(lists[0]) + 9 * len(lists[2])
    n_long = len(lists[1]) + len(lists[3])
    orc = ob.OracleForcefield(s, nthreads=nth)
    for _ in range(args.warmup):
        orc.apply(s.pos)
    # continue the NSNB cadence from where warm-up left it
    pairs = 0
    t0 = time.perf_counter()
    for k in range(args.steps):
        orc.apply(s.pos)
        pairs += n_short + (n_long if (args.warmup + k) % s.params.nsnb == 0 else 0)
    el = time.perf_counter() - t0
    orc.close()
    v = pairs / el
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": METRIC, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps,
            "ns_per_day": ns_per_day(1e3 * el / args.steps),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded SPC water box)",
            "config": {"workload": WORKLOAD, "n_atoms": s.topo.n_atoms, "rcutp": 0.8, "rcutl": 1.4, "nsnb": 5,
                       "pairlist": "cell list", "parallelism": f"host threads x{nth}"},
            "cpu_baseline": {"value": v, "unit": METRIC, "cores": nth, "kind": "port",
                             "sample": f"{args.steps} steps of {WORKLOAD}, FP64 C++ restatement of the gromos-rs "
                                       f"nonbonded path (the Rust reference cannot be built here), {nth} threads"},
            "e2e": {"value": v, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def hbm_peak_gbs():
    """Measured copy bandwidth of this pool's B200s (MEASURED_PEAKS.json), else the fallback figure."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def pairlist_summary(s, n_short, n_long, build_ms, ms_per_step):
    """The pairlist build on the rebuild steps of the timed region: device time per rebuild
    (CUDA events around the build, inside the step graph) and its algorithmic bytes per
    rebuild: the FP64 reference position of every CG read (24 B), cell key and permutation
    written and read (16 B), CSR offsets (8 B), and one 4-byte j entry per listed CG pair."""
    ncg = s.topo.n_cg
    cg_pairs = (n_short + n_long) / 9.0    # water-water CG pairs: 9 atom pairs each
    nbytes = 48.0 * ncg + 4.0 * cg_pairs
    peak, src = hbm_peak_gbs()
    if not build_ms:
        return None
    t = statistics.median(build_ms)
    gbs = nbytes / (t * 1e-3) / 1e9
    return {"build_us_per_rebuild": 1e3 * t, "rebuilds_timed": len(build_ms),
            "algorithmic_bytes_per_rebuild": nbytes, "achieved_gbs": gbs, "hbm_peak_gbs": peak,
            "peak_source": src, "frac_of_hbm": gbs / peak, "traffic": None,
            "share_of_step_time": t / (s.params.nsnb * ms_per_step) if ms_per_step > 0 else None}


def run_md(ff, s, args, generators):
    """MD steps (force evaluation + leap-frog + SETTLE, device resident) for ns/day.

    Timed with CUDA events on the library's stream around gr_md_run; the
    runner synchronises once per pairlist period (overflow check), which is
    inside the timed region.
    """
    import torch

    mass = generators.masses(s)
    vel = generators.maxwell_velocities(mass, 300.0, seed=2002)
    ff.upload_positions(s.pos)
    # Berendsen bath at 300 K (tau 0.1 ps): the synthetic start releases potential
    # energy and would heat an NVE run far above 300 K
    ff.md_init(mass, vel, dt=DT_PS, settle=True, dist_oh=0.1, dist_hh=generators.SPC_DHH, temperature=300.0,
               tau=0.1)
    ff.md_run(max(args.warmup, 3) * 5)
    n = max(args.md_steps, 1)
    stream = torch.cuda.ExternalStream(ff.stream())
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    st = ff.md_run(n)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    return {"steps": n, "dt_ps": DT_PS, "ms_per_step": ms / n, "ns_per_day": ns_per_day(ms / n),
            "settle": True, "settle_failures": st["settle_failures"], "rollbacks": st["rollbacks"],
            "e_kin_final": st["e_kin"],
            # degrees of freedom as the bath counts them: 3N minus 3 SETTLE constraints per water
            "t_final_k": 2.0 * st["e_kin"] / ((3 * s.topo.n_atoms - (s.topo.n_atoms - s.topo.n_solute_atoms))
                                              * generators.BOLTZ),
            "thermostat": "Berendsen 300 K, tau 0.1 ps",
            "start": "seeded Maxwell-Boltzmann velocities at 300 K"}


def run_gpu(args, rank, world, local_rank):
    import torch

    from gromos_nb import generators
    from gromos_nb.nonbonded import Forcefield, ffma_peak
    from gromos_nb.replicas import aggregate

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
    s = generators.config2_spc30000(seed=1002 + rank)
    ff = Forcefield(s, kernel=args.kernel, device=local_rank, cluster_size=args.cluster_size,
                    water_layout=args.layout)
    # pair counts of this configuration (short per step, long per rebuild)
    r0 = ff.apply(s.pos, count_pairs=True)
    n_short, n_long = int(r0["n_pairs_short"]), int(r0["n_pairs_long"])
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")
    graph = not args.no_graph
    for _ in range(args.warmup):
        ff.eval_async(graph=graph)
    torch.cuda.synchronize()
    # continue the cadence: the next eval after (1 + warmup) evals
    evals_done = 1 + args.warmup
    clocks = ClockSampler(local_rank)
    clocks.start()
    launches0 = ff.launches()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    step_ms, short_ms, long_ms, build_ms = [], [], [], []
    kshort_ms, klong_ms, prep_ms = [], [], []
    pairs = 0
    rebuilds = 0
    for k in range(args.steps):
        flush.zero_()                      # L2 flush between steps (not in the step's events)
        torch.cuda.synchronize()
        rebuild = (evals_done % s.params.nsnb) == 0
        ff.eval_async(graph=graph)
        evals_done += 1
        t = ff.timings()                   # CUDA events on the library's stream (first and last graph node)
        step_ms.append(t[4])
        if rebuild:
            rebuilds += 1
        pairs += n_short + (n_long if rebuild else 0)
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    launches = ff.launches() - launches0
    clk = clocks.stop()
    # stage windows (pairlist build, short-range, long-range kernels) from a kernel-by-kernel
    # pass with the same L2 flush: a recorded graph carries no events inside it
    stage_steps = max(4 * s.params.nsnb, min(args.steps, 100))
    for k in range(stage_steps):
        flush.zero_()
        torch.cuda.synchronize()
        rebuild = (evals_done % s.params.nsnb) == 0
        ff.eval_async(graph=False)
        evals_done += 1
        t = ff.timings()
        kt = ff.kernel_timings()
        if rebuild:
            long_ms.append(t[2])
            build_ms.append(t[0])
            if kt[2] >= 0:
                klong_ms.append(kt[2])
        else:
            short_ms.append(t[1])
            if kt[1] >= 0:
                kshort_ms.append(kt[1])
                prep_ms.append(kt[0])
    torch.cuda.synchronize()
    total_ms, pairs_all = aggregate(float(sum(step_ms)), float(pairs), device="cuda")
    value = pairs_all / (total_ms * 1e-3)
    ms_per_step = total_ms / args.steps
    # end to end through the public API: host positions in, host forces out
    pinned = torch.from_numpy(np.ascontiguousarray(s.pos)).pin_memory().numpy()
    fout = torch.empty((s.topo.n_atoms, 3), dtype=torch.float64).pin_memory().numpy()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e2e_pairs = 0
    for k in range(args.steps):
        rebuild = (evals_done % s.params.nsnb) == 0
        ff.apply(pinned, count_pairs=False, out=fout, graph=graph)
        evals_done += 1
        e2e_pairs += n_short + (n_long if rebuild else 0)
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    e2e_value = e2e_pairs * world / e2e_s
    h2d = s.topo.n_atoms * 3 * 8
    d2h = s.topo.n_atoms * 3 * 8 + 8 * (2 * ff.G * ff.G + 10)
    md = run_md(ff, s, args, generators)
    if args.kernel == "fixed" and not args.no_plain_md:
        # the same MD on the plain FP32 kernel (the baseline the fixed-point path is compared to)
        ff_plain = Forcefield(s, kernel="plain", device=local_rank)
        md_plain = run_md(ff_plain, s, argparse.Namespace(warmup=args.warmup, md_steps=max(50, args.md_steps // 10)),
                          generators)
        ff_plain.close()
        md["plain_kernel"] = {"ms_per_step": md_plain["ms_per_step"], "ns_per_day": md_plain["ns_per_day"],
                              "steps": md_plain["steps"]}
    out = None
    if rank == 0:
        peak = ffma_peak(local_rank)
        t_short = statistics.median(short_ms) if short_ms else float("nan")
        t_kshort = statistics.median(kshort_ms) if kshort_ms else float("nan")
        t_klong = statistics.median(klong_ms) if klong_ms else float("nan")
        achieved = OPS_PER_PAIR * n_short / (t_kshort * 1e-3)
        achieved_window = OPS_PER_PAIR * n_short / (t_short * 1e-3)
        cpu = None
        if not args.no_cpu_baseline:
            cpu = cpu_baseline_sample()
        out = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": ms_per_step, "ns_per_day": md["ns_per_day"],
               "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32+i64",
               "data": "synthetic (seeded SPC water box)",
               "config": {"workload": WORKLOAD, "n_atoms": s.topo.n_atoms, "box_nm": 9.65, "rcutp": 0.8,
                          "rcutl": 1.4, "nsnb": 5, "kernel": args.kernel, "cluster_size": args.cluster_size,
                          "water_layout": args.layout, "pairs_short_per_step": n_short,
                          "launch": "kernel by kernel" if args.no_graph else "recorded CUDA graph per step",
                          "pairs_long_per_rebuild": n_long, "rebuild_steps_timed": rebuilds,
                          "l2": "flushed (256 MiB write) between steps, outside the step events",
                          "stage_windows": f"{stage_steps} kernel-by-kernel steps after the timed region "
                                           "(short-range, long-range and build windows; CUDA events per stage)",
                          "step": "value: force evaluation (positions static); md: force evaluation + leap-frog + SETTLE",
                          "parallelism": "replicas" if world > 1 else "single system"},
               "e2e": {"value": e2e_value, "unit": METRIC, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
               "roofline": {"bound": "fp32",
                            "kernel": "short-range water force kernel (k_water_force_it, deferred pairs in its "
                                      "last block), CUDA events around its launch on the library's stream",
                            "achieved": achieved / 1e12, "peak": peak / 1e12, "unit": "Tops/s (FP32 pipe)",
                            "frac": achieved / peak, "traffic": SHORT_KERNEL_DRAM_BYTES,
                            "traffic_source": "ncu dram bytes of one short-range launch, recorded from a "
                                              "capture of this build's kernel (not measured by this run)",
                            "peak_source": "measured FFMA-chain kernel (gr_ffma_peak), one FFMA = one op",
                            "ops_per_pair": OPS_PER_PAIR, "short_kernel_ms": t_kshort,
                            "prep_kernel_ms": statistics.median(prep_ms) if prep_ms else None,
                            "short_window_ms": t_short, "frac_short_window": achieved_window / peak,
                            "long_kernel_ms": t_klong,
                            "frac_long_kernel": OPS_PER_PAIR * n_long / (t_klong * 1e-3) / peak,
                            "long_window_ms": statistics.median(long_ms) if long_ms else None},
               "pairlist": pairlist_summary(s, n_short, n_long, build_ms, ms_per_step),
               "md": md, "cpu_baseline": cpu, "clocks": clk, "gpu_launches": launches}
    ff.close()
    return out


# ---------------------------------------------------------------------------
# Batched workloads: REMD replicas, FEP lambda windows, serving.  Each prints
# its own JSON line; the default workload above is the single large system.

def _make_system(spec):
    from gromos_nb import generators

    nw, ns, seed, perturbed, lam = spec
    s = generators.solvated_solute_system(nw, ns, seed=seed, perturbed=perturbed, lam=lam, rc=1.4, nsnb=5)
    s.params.lam = lam
    return s


def _generate(specs):
    """Seeded systems, generated on the host's cores by a spawn pool (no GPU
    work has started in this process yet)."""
    import concurrent.futures as cf
    import multiprocessing as mp

    with cf.ProcessPoolExecutor(max_workers=min(len(specs), os.cpu_count() or 1),
                                mp_context=mp.get_context("spawn")) as ex:
        return list(ex.map(_make_system, specs))


def _member(s, seed, T, kernel="fixed", tau=0.1):
    """A replica: seeded Maxwell-Boltzmann start at T, Berendsen bath at T (tau in ps)."""
    from gromos_nb import generators
    from gromos_nb.nonbonded import Forcefield

    ff = Forcefield(s, kernel=kernel)
    ff.upload_positions(s.pos)
    m = generators.masses(s)
    ff.md_init(m, generators.maxwell_velocities(m, T, seed), dt=DT_PS, settle=True, dist_oh=0.1,
               dist_hh=generators.SPC_DHH, temperature=T, tau=tau)
    return ff


def _pairs_per_step(ff, s):
    r = ff.apply(s.pos, count_pairs=True, download_forces=False)
    ff.upload_positions(s.pos)
    return r["n_pairs_short"] + r["n_pairs_long"] / max(1, s.params.nsnb)


def _one_by_one(systems, seeds, temps, steps, kernel):
    """Members run alone, one after the other (device time per member summed)."""
    import torch

    total_ms = 0.0
    for s, seed, T in zip(systems, seeds, temps):
        ff = _member(s, seed, T, kernel)
        ff.md_run(max(1, s.params.nsnb))          # warm-up period
        stream = torch.cuda.ExternalStream(ff.stream())
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ff.md_run(steps)
        e1.record(stream)
        e1.synchronize()
        total_ms += e0.elapsed_time(e1)
        ff.close()
    return total_ms


def _jobs_one_by_one(jobs, kernel):
    """Each serving job alone, from its own start to its last step (device time summed, and wall)."""
    import torch

    from gromos_nb import generators
    from gromos_nb.nonbonded import Forcefield

    total_ms = 0.0
    t0 = time.perf_counter()
    for job in jobs:
        ff = Forcefield(job.system, kernel=kernel)
        ff.upload_positions(job.system.pos)
        ff.md_init(job.mass, job.vel, dt=job.dt, settle=True, dist_oh=0.1, dist_hh=generators.SPC_DHH,
                   temperature=job.temperature, tau=job.tau)
        stream = torch.cuda.ExternalStream(ff.stream())
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ff.md_run(job.n_steps)
        e1.record(stream)
        e1.synchronize()
        total_ms += e0.elapsed_time(e1)
        ff.close()
    return total_ms, time.perf_counter() - t0


def run_batched(args, kind, rank=0, world=1, local_rank=0):
    """REMD replicas (uneven sizes) or FEP lambda windows in one batch.  Under
    torchrun the members are spread over the ranks by size (whole systems, no
    collective on the force path); rank 0 prints the aggregate."""
    import torch

    from gromos_nb import generators
    from gromos_nb.nonbonded import Batch
    from gromos_nb.replicas import aggregate, shard_by_work

    torch.cuda.set_device(local_rank)

    rng = np.random.default_rng(1003 if kind == "remd" else 1004)
    systems, seeds, temps, lams = [], [], [], []
    if kind == "remd":
        n = args.replicas
        temps = list(300.0 * (450.0 / 300.0) ** (np.arange(n) / max(1, n - 1)))
        specs = [(int(rng.integers(500, 8001)), 200, 1003 + r, False, 0.0) for r in range(n)]
        seeds = [5000 + r for r in range(n)]
        workload = f"remd_{n}_replicas_spc500-8000_solute200_rc1.4"
    else:
        lams = [round(0.05 * k, 2) for k in range(21)]
        specs = [(5000, 30, 1004, True, lam) for lam in lams]
        seeds = [6000] * len(lams)                  # same start in every window
        temps = [300.0] * len(lams)
        workload = "fep_21_windows_spc5000_solute30_rc1.4"
    n_members = len(specs)
    if world > 1:
        mine = shard_by_work([sp[0] + sp[1] for sp in specs], world)[rank]
        specs = [specs[i] for i in mine]
        seeds = [seeds[i] for i in mine]
        temps = [temps[i] for i in mine]
        lams = [lams[i] for i in mine] if lams else lams
    systems = _generate(specs)
    ffs = [_member(s, seed, T) for s, seed, T in zip(systems, seeds, temps)]
    pairs = [_pairs_per_step(ff, s) for ff, s in zip(ffs, systems)]
    b = Batch()
    for ff in ffs:
        b.add(ff)
    tune = b.autotune(periods=1)
    b.md_run(5)                                     # warm-up period (graph capture)
    launches0 = b.launches()
    ms = b.md_run(args.batch_steps)
    launches = b.launches() - launches0
    per_step, pairs_all = aggregate(ms / args.batch_steps, sum(pairs), device="cuda")
    value = pairs_all / (per_step * 1e-3)
    stats = [ff.md_stats() for ff in ffs]
    out_fep = None
    if kind == "fep":
        b.eval()
        res = [ff.result() for ff in ffs]
        out_fep = {"lambda": lams, "dhdl": [r["dhdl"] for r in res], "e_lj": [r["e_lj"] for r in res],
                   "e_crf": [r["e_crf"] for r in res]}
    b.close()
    for ff in ffs:
        ff.close()
    # the same members one by one: fixed-point kernel, and the plain FP32 kernel
    sample = min(len(systems), args.sample_members)
    idx = list(range(0, len(systems), max(1, len(systems) // sample)))[:sample]
    sub = [systems[i] for i in idx]
    sub_pairs = sum(pairs[i] for i in idx)
    steps_alone = min(args.batch_steps, 20)
    ms_fixed = _one_by_one(sub, [seeds[i] for i in idx], [temps[i] for i in idx], steps_alone, "fixed")
    ms_plain = _one_by_one(sub, [seeds[i] for i in idx], [temps[i] for i in idx], steps_alone, "plain")
    if rank != 0:
        return None
    line = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.batch_steps,
            "warmup": 5, "ms_per_step": per_step,
            "ns_per_day": ns_per_day(per_step), "ns_per_day_aggregate": ns_per_day(per_step) * n_members,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32+i64",
            "data": "synthetic (seeded water boxes + seeded solutes)",
            "config": {"workload": workload, "members": n_members, "members_rank0": len(systems),
                       "atoms_rank0": int(sum(s.topo.n_atoms for s in systems)),
                       "pairs_per_batch_step": pairs_all,
                       "parallelism": f"members sharded over {world} GPUs" if world > 1 else "one GPU",
                       "step": "MD step (forces + leap-frog + Berendsen bath at the replica temperature + SETTLE)",
                       "launch": "one CUDA graph launch per batch step", "autotune": tune},
            "gpu_launches": launches,
            "one_by_one": {"sample_members": len(idx), "steps": steps_alone,
                           "fixed_pair_int_per_s": sub_pairs * steps_alone / (ms_fixed * 1e-3),
                           "plain_pair_int_per_s": sub_pairs * steps_alone / (ms_plain * 1e-3)},
            "md": {"settle_failures": int(sum(s["settle_failures"] for s in stats)),
                   "rollbacks": int(sum(s["rollbacks"] for s in stats))}}
    if out_fep:
        line["fep"] = out_fep
    return line


def run_serving(args):
    from gromos_nb.serving import Server, poisson_jobs

    jobs = poisson_jobs(args.jobs, rate=20.0, seed=1005, waters=(300, 20000), steps=(100, 2000), solute_prob=0.5,
                        solute_atoms=(50, 500), rc=1.4, nsnb=5)
    srv = Server(hbm_budget=int(args.hbm_budget_gb * 2 ** 30), chunk_steps=5, count_pairs=True)
    srv.run(jobs, timeout=1800)
    rep = srv.report()
    srv.close()
    # the same jobs one by one on the plain FP32 kernel, every job in full (measured, not extrapolated)
    ms_plain, wall_plain = _jobs_one_by_one(jobs, "plain")
    total_pairs = sum(j.pairs_per_step * j.n_steps for j in jobs)
    line = {"metric": METRIC, "value": rep["pair_int_per_s"], "unit": METRIC, "n_gpus": 1,
            "steps": rep["batch_steps"], "warmup": 0, "ms_per_step": rep["gpu_ms"] / max(1, rep["batch_steps"]),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32+i64",
            "data": "synthetic (seeded Poisson job stream, seeded systems)",
            "config": {"workload": f"serving_{len(jobs)}_jobs_poisson20_spc300-20000_steps100-2000",
                       "hbm_budget_gb": args.hbm_budget_gb, "chunk_steps": 5},
            "serving": rep,
            "one_by_one_plain": {"jobs": len(jobs), "device_s": ms_plain * 1e-3, "wall_s": wall_plain,
                                 "pair_int_per_s": total_pairs / (ms_plain * 1e-3)}}
    return line


_LINE_KEYS = ("metric", "unit", "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "n_gpus", "warmup")


def batched_summary(args):
    """The batched workloads at bounded size for the default line (one GPU): the 21 FEP
    lambda windows, 32 of the 256 REMD replicas (same generator and size range), and the
    serving stream with its one-by-one plain-kernel baseline measured in full."""
    out = {}
    t0 = time.perf_counter()
    a = argparse.Namespace(**vars(args))
    a.batch_steps, a.sample_members = 100, 4
    fep = run_batched(a, "fep")
    a.replicas = 32
    remd = run_batched(a, "remd")
    srv = run_serving(args)
    for name, line in (("fep_21_windows", fep), ("remd_32_replicas", remd), ("serving", srv)):
        out[name] = {k: v for k, v in line.items() if k not in _LINE_KEYS}
    for name in ("fep_21_windows", "remd_32_replicas"):
        o = out[name]
        o["speedup_vs_plain_one_by_one"] = o["value"] / o["one_by_one"]["plain_pair_int_per_s"]
        o["speedup_vs_fixed_one_by_one"] = o["value"] / o["one_by_one"]["fixed_pair_int_per_s"]
    sv = out["serving"]
    sv["makespan_speedup_vs_plain_one_by_one"] = sv["one_by_one_plain"]["wall_s"] / sv["serving"]["wall_s"]
    out["seconds"] = time.perf_counter() - t0
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--kernel", default="fixed", choices=["fixed", "plain"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cluster-size", type=int, default=0, help="water i-cluster width 4 or 8 (0 = default)")
    ap.add_argument("--md-steps", type=int, default=1000, help="MD steps timed for ns/day")
    ap.add_argument("--layout", type=int, default=0, help="water kernel layout: 1 shared bits, 2 per-lane bits")
    ap.add_argument("--no-graph", action="store_true", help="launch kernel by kernel instead of replaying graphs")
    ap.add_argument("--no-plain-md", action="store_true", help="skip the plain-kernel MD comparison")
    ap.add_argument("--workload", default="spc30000", choices=["spc30000", "remd", "fep", "serving"])
    ap.add_argument("--replicas", type=int, default=256)
    ap.add_argument("--batch-steps", type=int, default=None,
                    help="MD steps per batched run (default: 500 for fep, the FEP windows' length; 100 for remd)")
    ap.add_argument("--sample-members", type=int, default=8, help="members timed one by one for comparison")
    ap.add_argument("--jobs", type=int, default=40)
    ap.add_argument("--hbm-budget-gb", type=float, default=150.0)
    ap.add_argument("--no-batched", action="store_true",
                    help="default workload: leave out the batched FEP / REMD / serving sub-object")
    args = ap.parse_args()
    if args.batch_steps is None:
        args.batch_steps = 500 if args.workload == "fep" else 100
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if args.workload in ("remd", "fep"):
        if world > 1:
            import datetime

            import torch
            import torch.distributed as dist
            torch.cuda.set_device(local_rank)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
            try:
                line = run_batched(args, args.workload, rank, world, local_rank)
            finally:
                dist.destroy_process_group()
        else:
            line = run_batched(args, args.workload)
        if line is not None:
            print(json.dumps(line), flush=True)
        return 0
    if args.workload == "serving":
        if rank == 0:
            print(json.dumps(run_serving(args)), flush=True)
        return 0
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        out = run_gpu(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
    if out is not None:
        if world == 1 and not args.no_batched:
            out["batched"] = batched_summary(args)
        print(json.dumps(out), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
