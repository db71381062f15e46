"""Throughput of the particle-move hot path on B200 (particle-steps/s).

Workload (the precision-form configuration, plain FP32 forcing): the analytic 128x128 grid with
10 sigma levels over lon 14.00-14.20 E, lat 40.70-40.90 N, uniform current u=0.2, v=0.1 m/s,
25 hourly FP32 records; 16,777,216 particles per GPU placed uniformly at 0-5 m depth;
deterministic, explicit midpoint, dt=30 s (120 substeps per interval). One step = one forcing
interval of every particle. Synthetic, seeded inputs stand in for the unavailable benchmark data.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line (rank 0). `value` is device-timed with the particles resident in HBM;
`e2e` moves the same particles through the public host-buffer entry point with the copies in the
timed region; `cpu_baseline` times the reference's own CPU path (move and concentration) on a
bounded sample. `surrogate` is the second arm of the metric, the learned form: the same workload
with FP16 forcing storage, the tcgen05 MLP's one-interval displacement and the plain stochastic
operator every substep (Philox streams), device-timed the same way, beside the plain FP32 step with
the same random walk and the deterministic surrogate; with the tensor-core roofline of its step
kernel and its position error after 24 hours against the FP64 reference-arithmetic kernel, on the
analytic grid (1,048,576-particle subset) and on a non-uniform streamfunction flow. `precision`
gives the plain step with FP32, FP16 and BF16 forcing storage (throughput and 24-hour error) and
the FP64 reference-arithmetic kernel's throughput. `realistic` runs the realistic grid
(1024x1024x30, ~20 % land, records generated on the device, 4,194,304 particles from the device
emitter, Philox random walk, dt = 15 s) for 5 intervals after 3 warm-up ones, with its own
roofline and CPU baseline (`--workload realistic` runs it alone, longer). Kernel times come from
per-interval events recorded inside the timed loops.
"""
import argparse
import json
import os

# The reference's CPU path is timed as its solver runs it: OpenMP threads bound one per physical
# core, packed (set before any OpenMP runtime is loaded).
os.environ.setdefault("OMP_PLACES", "cores")
os.environ.setdefault("OMP_PROC_BIND", "close")
# The CPUs this process may run on, read before the first OpenMP region: with OMP_PROC_BIND set,
# that region binds the calling thread to its own place, after which the thread's affinity mask
# names one core only.
CPU_SET = sorted(os.sched_getaffinity(0))
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

B_ALG = 118.0  # algorithmic bytes per particle-step: one read + one write of the 59-byte state


SURROGATE_FLOP = 2 * 2 * 256 * 256  # tensor-core FLOPs per particle-interval: layers 2 and 3


def measured_peaks(key="hbm_gbs", fallback=6650.0):
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as fh:
            data = json.load(fh)
        if key in data:
            return float(data[key]), "measured"
    return fallback, "fallback"


def profile_traffic(summary="move_kernel_config3.md", key="traffic_bytes_per_particle_step"):
    """DRAM bytes per unit of work of a kernel from its committed ncu summary."""
    path = os.path.join(ROOT, "profiles", summary)
    if not os.path.exists(path):
        return None
    for line in open(path):
        if line.startswith(key + ":"):
            return float(line.split(":", 1)[1].strip().split()[0])
    return None


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", str(self.gpu)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, ValueError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def physical_cores():
    """(count, how) of the physical cores among the CPUs this process could run on at start: one per
    (package, core) pair of the CPU topology. Where the topology is not exposed (a virtual machine
    may report every CPU as core 0, or more than two CPUs per core), the logical CPUs are counted
    and `how` says so."""
    cpus = CPU_SET
    seen = set()
    for cpu in cpus:
        base = f"/sys/devices/system/cpu/cpu{cpu}/topology/"
        try:
            with open(base + "core_id") as a, open(base + "physical_package_id") as b:
                seen.add((b.read().strip(), a.read().strip()))
        except OSError:
            return len(cpus), "logical CPUs (no CPU topology exposed)"
    if not seen or len(cpus) > 2 * len(seen):
        return len(cpus), "logical CPUs (the CPU topology reports fewer cores than plausible)"
    return len(seen), "physical cores (CPU topology)"


def physical_gpu(local_rank):
    visible = os.environ.get("CUDA_VISIBLE_DEVICES")
    if visible:
        ids = [x for x in visible.split(",") if x.strip()]
        if local_rank < len(ids) and ids[local_rank].strip().isdigit():
            return int(ids[local_rank])
    return local_rank


def workload(n_particles, rank, frames=25):
    from wacommplusplus_b200 import synthetic as syn
    from wacommplusplus_b200.types import default_config
    win = syn.config1_window(n_frames=frames)
    particles = syn.uniform_particles(n_particles, win.eta, win.xi, seed=1 + rank,
                                      first_id=rank * n_particles)
    cfg = default_config(random=False)
    return win, particles, cfg


def cpu_interval(kind, cfg, recs, win, t, threads):
    """One interval of the reference CPU path on `recs`: Particle::move under OpenMP dynamic,64
    (Wacomm.cpp:501-525), then Concentration::evaluate (Wacomm.cpp:722) into the float grid (the
    oracle port of both where the reference build is absent). Returns seconds."""
    from oracle import bindings as ob
    t0 = time.perf_counter()
    if kind == "reference":
        ob.ref_move(cfg, recs, win, t, threads=threads)
        ob.ref_concentration(recs, t + 1, win.T, win, threads=threads)
    else:
        ob.oracle_move(cfg, recs, win, t, threads=threads)
        ob.oracle_concentration(recs, t + 1, win.T, win)
    return time.perf_counter() - t0


def cpu_reference_rate(win, particles, cfg, threads, repeats=3, sample=262144):
    """Particle-steps/s of the reference CPU path (move + concentration of one interval) on
    `sample` particles; median of `repeats` after a warm-up."""
    from oracle import bindings as ob
    kind = "reference" if ob.ref_available() else "port"
    sample = min(sample, len(particles))
    rates = []
    for r in range(repeats + 1):
        recs = particles[:sample].copy()
        dt = cpu_interval(kind, cfg, recs, win, r % (win.T - 1), threads)
        steps = sample * int(round(3600.0 / cfg.dti))
        if r > 0:  # first run warms caches and the thread pool
            rates.append(steps / dt)
    return statistics.median(rates), kind, sample


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    threads, how = physical_cores()
    win, particles, cfg = workload(1 << 18, 0)
    from oracle import bindings as ob
    kind = "reference" if ob.ref_available() else "port"
    sample = len(particles)
    steps_per = sample * 120
    for _ in range(args.warmup):
        cpu_interval(kind, cfg, particles.copy(), win, 0, threads)
    dt = 0.0
    for s in range(args.steps):
        dt += cpu_interval(kind, cfg, particles.copy(), win, s % (win.T - 1), threads)
    value = steps_per * args.steps / dt
    line = {
        "impl": "reference", "metric": "particle-steps/s", "value": value,
        "unit": "particle-steps/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1000 * dt / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "precision-form analytic grid 128x128x10, plain FP32 forcing, "
                               f"{sample} particles per step (bounded CPU sample), midpoint, dt=30 s",
                   "l2": "inputs larger than L2"},
        "cpu_baseline": {"value": value, "unit": "particle-steps/s", "cores": threads,
                         "cores_counted_as": how, "kind": kind,
                         "sample": f"{sample} particles x 120 substeps per step (Particle::move, "
                                   "OpenMP dynamic,64) + Concentration::evaluate, one thread per "
                                   "physical core (OMP_PLACES=cores, OMP_PROC_BIND=close)"},
        "e2e": {"value": value, "unit": "particle-steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_realistic(args):
    n_total = args.particles if args.particles != 1 << 24 else 1 << 22
    line = realistic_leg(n_total, max(args.warmup, 3), args.steps, not args.no_cpu)
    print(json.dumps(line), flush=True)


def realistic_leg(n_total, warm, steps, with_cpu):
    """The realistic configuration on one GPU: 1024x1024 rho nodes, 30 Vtransform-2 levels, ~20 %
    land, hourly FP32 records of a 64-mode streamfunction flow (generated on the device, as many
    as the run needs, at most 24); n_total particles released by the device emitter from 64
    uniform-rate sources during the first hour; dt = 15 s, random walk with Philox streams,
    fused uint32 concentration, dead-record compaction each interval. One step = emission + cell
    sort + move + concentration + compaction of one interval, device-timed."""
    import torch
    from wacommplusplus_b200 import synthetic as syn
    from wacommplusplus_b200.engine import Engine
    from wacommplusplus_b200.types import PARTICLE_DTYPE, default_config, make_sources

    n_sources = 64
    n_steps = min(steps, 24 - 1 - warm)
    frames = warm + n_steps + 1
    forcing = syn.RealisticForcing(eta=1024, xi=1024, s_rho=30, n_frames=frames, seed=2)
    cfg = default_config(random=True, dti=15.0, randomSeed=11)
    engine = Engine(0, arithmetic="fp32", storage="fp32", rng="philox")
    engine.set_config(cfg)
    t_build = time.perf_counter()
    engine.set_grid(forcing.eta, forcing.xi, forcing.s_rho, forcing.s_w, forcing.lonRad,
                    forcing.latRad, forcing.h, forcing.depthIntervals, forcing.mask)
    engine.set_times(forcing.times)
    frame_bytes = 0
    kept = {}
    for t in range(frames):
        f = forcing.frame_device(t)
        engine.upload_frame(t, f["zeta"], f["u"], f["v"], f["w"], f["akt"])
        frame_bytes = sum(a.nbytes for a in f.values())
        if t in (warm, warm + 1):
            kept[t] = f  # the records of the CPU baseline's interval
    t_build = time.perf_counter() - t_build
    engine.concentration_reset(frames)
    pos = forcing.sources(n_sources, seed=3)
    t0 = forcing.times[0]
    day = 86400.0
    sources = make_sources([(k, j, i, t0 / day, (t0 + 3600.0) / day, n_total / n_sources,
                             "uniform_rate") for k, j, i in pos])
    engine.set_particles(np.zeros(0, dtype=PARTICLE_DTYPE))

    def step(t):
        engine.emit(sources, forcing.times[t], forcing.times[t + 1])
        engine.move_interval(t)
        st = engine.stats()
        engine.remove_dead()
        return st

    for t in range(warm):
        step(t)
    ext = torch.cuda.ExternalStream(engine.stream)
    sampler = ClockSampler(physical_gpu(0))
    sampler.start()
    torch.cuda.synchronize()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    steps_total, launches, move_ms = 0.0, 0, []
    count = engine.count()
    start.record(ext)
    for s in range(n_steps):
        st = step(warm + s)
        steps_total += st["particle_steps"]
        launches += st["launches"] + 2
        move_ms.append(st["move_ms"])
    end.record(ext)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    elapsed_ms = start.elapsed_time(end)
    cpu = None
    if with_cpu:
        # the reference CPU step on a sample of the live particles over one interval
        win2 = forcing.window_of([warm, warm + 1], [kept[warm], kept[warm + 1]])
        live = engine.get_particles()
        sample = live[np.random.default_rng(0).permutation(len(live))[:65536]]
        sample = np.ascontiguousarray(np.sort(sample, order="id"))
        threads, how = physical_cores()
        rate, kind, n = cpu_reference_rate(win2, sample, cfg, threads, repeats=2, sample=65536)
        cpu = {"value": rate, "unit": "particle-steps/s", "cores": threads,
               "cores_counted_as": how, "kind": kind,
               "sample": f"{n} live particles x 240 substeps, one interval, Particle::move "
                         "(OpenMP dynamic,64) + Concentration::evaluate, one thread per physical "
                         "core, median of 2 after a warm-up"}
    peak, peak_src = measured_peaks()
    achieved = steps_total / n_steps * B_ALG / (statistics.mean(move_ms) * 1e-3) / 1e9
    line = {
        "metric": "particle-steps/s", "value": steps_total / (elapsed_ms / 1000.0),
        "unit": "particle-steps/s", "n_gpus": 1, "steps": n_steps, "warmup": warm,
        "ms_per_step": elapsed_ms / n_steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "realistic: 1024x1024x30 ROMS-shaped grid (Vtransform 2, ~20 % land), "
                               f"{frames} hourly FP32 records (generated on the device), "
                               f"{n_total} particles from {n_sources} "
                               "uniform-rate sources (device emission, first hour), dt=15 s, "
                               "Philox random walk, fused concentration, compaction each interval",
                   "particles_alive_at_timing": count,
                   "forcing_build_s": t_build, "record_bytes": frame_bytes},
        "move_kernel_ms": statistics.mean(move_ms),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_source": peak_src, "traffic": None,
                     "kernel": "move_fast_kernel (FP32 step, random-walk form)",
                     "kernel_ms": statistics.mean(move_ms),
                     "algorithmic_bytes_per_particle_step": B_ALG},
        "cpu_baseline": cpu, "e2e": None, "gpu_launches": launches, "clocks": clocks,
    }
    engine.close()
    return line


def run_batched(args):
    """The batched configuration on one GPU: 256 independent drift scenarios (sizes log-uniform
    1 k-256 k, 11,443,932 particles in all, each with its own point source, release window in the
    first 24 h and leeway-catalogue object) on the analytic 128x128x10 ocean over 48 h (49 hourly
    records); wind on a curvilinear 340x340 3-km grid (hourly, rms 8 m/s) and Stokes drift on a
    0.05-degree grid (3-hourly, rms 0.1 m/s) regridded on the device to the ocean nodes and the
    hourly times; leeway drift, Philox random walk, dt = 30 s, fused concentration. The move
    kernel's launch shape is autotuned and the 48 intervals are captured as one CUDA graph. One
    step = the whole 48-hour run of the batch (one graph launch), device-timed."""
    import torch
    from wacommplusplus_b200 import synthetic as syn
    from wacommplusplus_b200.engine import Engine
    from wacommplusplus_b200.types import PARTICLE_DTYPE, default_config

    hours = 48
    win = syn.config1_window(n_frames=hours + 1)
    records, table = syn.batched_scenarios(win, n_scenarios=args.scenarios)
    n = len(records)
    env = syn.environment(win.times[0], hours)
    cfg = default_config(random=True, randomSeed=23, driftModel=1)
    engine = Engine(0, arithmetic="fp32", storage="fp32", rng="philox")
    engine.set_config(cfg)
    engine.load_window(win)
    engine.set_geo_grid(win.lon, win.lat, win.sWValues)
    t_regrid = time.perf_counter()
    engine.regrid_environment("wind", "curvilinear", *env["wind"])
    engine.regrid_environment("stokes", "geographic", *env["stokes"])
    t_regrid = time.perf_counter() - t_regrid
    engine.concentration_reset(win.T)
    # pinned host copy of the batch: the e2e leg uploads it and reads the result back each step
    host_in = torch.empty(n * PARTICLE_DTYPE.itemsize, dtype=torch.uint8, pin_memory=True)
    host_out = torch.empty_like(host_in, pin_memory=True)
    batch_in = host_in.numpy().view(PARTICLE_DTYPE)
    batch_out = host_out.numpy().view(PARTICLE_DTYPE)
    batch_in[:] = records
    engine.set_particles(batch_in)
    shape, tune_ms = engine.autotune(hours // 2)
    engine.graph_capture(0, hours)

    def run():
        engine.set_particles(batch_in)
        engine.concentration_reset(win.T)
        engine.graph_launch()
        st = engine.stats()  # waits for the run
        return st

    for _ in range(max(args.warmup, 3)):
        run()
    sampler = ClockSampler(physical_gpu(0))
    sampler.start()
    device_ms, steps_total = [], 0.0
    for _ in range(args.steps):
        st = run()
        device_ms.append(st["device_ms"])
        steps_total += st["particle_steps"]
    clocks = sampler.stop()
    launches = engine.stats()["launches"]
    # e2e: batch from pinned host memory, the graph, the records back to pinned host memory
    t0 = time.perf_counter()
    for _ in range(args.steps):
        engine.set_particles(batch_in)
        engine.concentration_reset(win.T)
        engine.graph_launch()
        engine._check(engine._lib.wacomm_b200_get_particles(engine._ctx, batch_out.ctypes.data, n))
    e2e_s = time.perf_counter() - t0
    per_step = steps_total / args.steps
    peak, peak_kind = measured_peaks("hbm_gbs", 6650.0)
    mean_ms = statistics.mean(device_ms)
    achieved = per_step * B_ALG / (mean_ms / 1000.0) / 1e9
    traffic = profile_traffic("move_kernel_batched.md")
    cpu = None
    if not args.no_cpu:
        # the reference CPU step (leeway objects, wind and Stokes on the ocean grid) on a sample
        # of the batch over one interval in which every sampled record is released
        t = hours // 2
        wind = [engine.environment("wind", x) for x in (t, t + 1)]
        stokes = [engine.environment("stokes", x) for x in (t, t + 1)]
        win2 = syn.config1_window(n_frames=2, t0=win.times[t])
        win2.windU10 = np.ascontiguousarray([w[0] for w in wind])
        win2.windV10 = np.ascontiguousarray([w[1] for w in wind])
        win2.stokesU = np.ascontiguousarray([w[0] for w in stokes])
        win2.stokesV = np.ascontiguousarray([w[1] for w in stokes])
        sample = records[np.random.default_rng(0).permutation(n)[:65536]]
        sample = np.ascontiguousarray(np.sort(sample, order="id"))
        threads, how = physical_cores()
        rate, kind, m = cpu_reference_rate(win2, sample, cfg, threads, repeats=2, sample=65536)
        cpu = {"value": rate, "unit": "particle-steps/s", "cores": threads,
               "cores_counted_as": how, "kind": kind,
               "sample": f"{m} records of the batch x 120 substeps, one interval with leeway "
                         "drift, wind and Stokes, Particle::move (OpenMP dynamic,64) + "
                         "Concentration::evaluate, one thread per physical core, median of 2 "
                         "after a warm-up"}
    line = {
        "metric": "particle-steps/s", "value": per_step / (mean_ms / 1000.0),
        "unit": "particle-steps/s", "n_gpus": 1, "steps": args.steps,
        "warmup": max(args.warmup, 3), "ms_per_step": mean_ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"batched: {args.scenarios} drift scenarios (log-uniform 1k-256k, "
                               f"{n} particles, own source, release window and leeway object), "
                               "analytic 128x128x10 ocean, 48 h at dt=30 s, wind 340x340 3-km "
                               "curvilinear hourly and Stokes 0.05-degree 3-hourly regridded on "
                               "the device, Philox random walk, fused concentration, one CUDA "
                               "graph per 48-hour run",
                   "launch_shape": shape, "sort_cadence": engine.options().sort_by_cell,
                   "particles_per_thread": engine.options().particles_per_thread,
                   "autotune_ms": tune_ms, "regrid_s": t_regrid,
                   "l2": "inputs larger than L2"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak,
                     "traffic": None if traffic is None else traffic * per_step,
                     "note": f"B_alg 118 B per particle-step over the whole graph (sorts and "
                             f"packing included), {peak_kind} peak; traffic per run from the "
                             f"ncu summary's bytes per particle-step"},
        "cpu_baseline": cpu,
        "e2e": {"value": steps_total / e2e_s, "unit": "particle-steps/s",
                "h2d_bytes_per_step": n * PARTICLE_DTYPE.itemsize,
                "d2h_bytes_per_step": n * PARTICLE_DTYPE.itemsize},
        "gpu_launches": launches * args.steps, "clocks": clocks,
    }
    print(json.dumps(line), flush=True)
    engine.graph_release()
    engine.close()


def timed_run(engine, args, n_intervals, exchange, barrier, steps=None, warmup=None):
    """W untimed intervals, then K intervals enqueued back to back and device-timed with CUDA
    events on the engine's stream (a barrier and a synchronize on both sides). The engine records
    its dominant kernels' times per interval inside the same loop. Returns (elapsed ms,
    particle-steps counted by the kernels, per-interval kernel times [K][3], kernel launches of
    one interval)."""
    import torch
    steps = args.steps if steps is None else steps
    warmup = args.warmup if warmup is None else warmup
    for s in range(warmup):
        engine.move_interval(s % n_intervals)
        exchange(engine, s % n_intervals)
    ext = torch.cuda.ExternalStream(engine.stream)
    barrier()
    torch.cuda.synchronize()
    engine.kernel_times()  # drop the warm-up records
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    engine.steps_total(reset=True)
    start.record(ext)
    for s in range(steps):
        t = (warmup + s) % n_intervals
        engine.move_interval(t)
        exchange(engine, t)
    end.record(ext)
    torch.cuda.synchronize()
    barrier()
    launches = engine.stats()["launches"] + 1  # + the device-side step accumulation
    return start.elapsed_time(end), engine.steps_total(), engine.kernel_times(), launches


def over_ranks(dist, world, elapsed_ms, count):
    """Max of the elapsed time and sum of the work over the ranks."""
    if world <= 1:
        return elapsed_ms, count
    import torch
    t = torch.tensor([elapsed_ms, count], dtype=torch.float64, device="cuda")
    mx = t.clone()
    dist.all_reduce(mx, op=dist.ReduceOp.MAX)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(mx[0]), float(t[1])


def error_stats(win, got, want, hours, against):
    from wacommplusplus_b200 import surrogate as sg
    err = sg.geo_error_m(win, got, want)
    err = err[np.isfinite(err)]
    return {"mean": float(err.mean()), "p99": float(np.quantile(err, 0.99)),
            "max": float(err.max()), "hours": hours, "particles": int(len(got)),
            "against": against}


def run_hours(win, cfg, records, hours, local_rank, surrogate=False, **options):
    """Records after `hours` intervals of one engine configuration."""
    from wacommplusplus_b200.engine import Engine
    e = Engine(local_rank, surrogate=int(surrogate), **options)
    e.set_config(cfg)
    e.load_window(win)
    if surrogate:
        e.set_surrogate()
    e.set_particles(records)
    for t in range(hours):
        e.move_interval(t)
    out = e.get_particles()
    e.close()
    return out


FP64 = "FP64 reference-arithmetic kernel (parity-pinned to the oracle)"


def nonuniform_error(local_rank, hours=24, n=65536):
    """The surrogate's 24-hour error where its network acts: a streamfunction flow (64 Fourier
    modes, rms 0.3 m/s, 256x256x12 Vtransform-2 grid at 0.0015 degrees, no land, seed held out
    of training), deterministic, against the FP64 kernel; the plain FP32 step beside it."""
    from wacommplusplus_b200 import synthetic as syn
    from wacommplusplus_b200.surrogate_train import segment_particles, training_config
    win = syn.RealisticForcing(eta=256, xi=256, s_rho=12, n_frames=hours + 1, seed=4242,
                               dlon=0.0015, dlat=0.0015, land_fraction=0.0,
                               water_border=0).window()
    start = segment_particles(np.random.default_rng(1), win, 0, n)
    start["time"] = win.times[0]
    cfg = training_config()
    truth = run_hours(win, cfg, start, hours, local_rank, arithmetic="reference")
    surr = run_hours(win, cfg, start, hours, local_rank, surrogate=True, arithmetic="fp32",
                     storage="fp16")
    plain = run_hours(win, cfg, start, hours, local_rank, arithmetic="fp32", storage="fp16")
    out = error_stats(win, surr, truth, hours, FP64)
    out["flow"] = ("streamfunction of 64 Fourier modes, rms 0.3 m/s, wavelengths 2-50 km, "
                   "256x256x12 grid at 0.0015 deg, no land")
    out["plain_fp32_fp16_storage"] = error_stats(win, plain, truth, hours, FP64)
    # the trust limit: particles whose estimated one-interval error exceeds it take the FP32 step
    from wacommplusplus_b200.engine import Engine
    limited = {}
    for limit in (200.0, 50.0):
        e = Engine(local_rank, arithmetic="fp32", storage="fp16", surrogate=1)
        e.set_config(cfg)
        e.load_window(win)
        e.set_surrogate()
        e.set_surrogate_error_limit(limit)
        e.set_particles(start)
        run = fallback = 0
        for t in range(hours):
            e.move_interval(t)
            st = e.surrogate_stats()
            run, fallback = run + st["run"], fallback + st["fallback"]
        got = e.get_particles()
        e.close()
        entry = error_stats(win, got, truth, hours, FP64)
        entry["surrogate_share"] = run / max(1, run + fallback)
        limited[f"{limit:g}_m"] = entry
    out["with_error_limit"] = limited
    return out


def surrogate_leg(args, win, particles, local_rank, world, rank, barrier, dist, exchange):
    """The learned form (config 5 as specified): FP16 forcing storage, the tensor-core surrogate's
    one-interval displacement and the plain stochastic operator every substep (Philox streams),
    device-timed like the headline; beside it, on the same workload, the plain FP32 step with the
    same random walk (the comparator of the >= 3x target) and the deterministic surrogate. Per-
    interval kernel times come from the engine's event ring inside the timed loop."""
    from wacommplusplus_b200.engine import Engine
    from wacommplusplus_b200.types import default_config

    n_intervals = win.T - 1

    def arm(cfg, surrogate, **options):
        e = Engine(local_rank, surrogate=int(surrogate), **options)
        e.set_config(cfg)
        e.load_window(win)
        if surrogate:
            e.set_surrogate()
        e.set_particles(particles)
        e.concentration_reset(win.T)
        ms, count, kt, launches = timed_run(e, args, n_intervals, exchange, barrier)
        ss = e.surrogate_stats() if surrogate else None
        e.close()
        ms, count = over_ranks(dist, world, ms, count)
        return {"value": count / (ms / 1000.0), "ms_per_step": ms / args.steps,
                "gpu_launches": launches * args.steps}, kt, ss, count / args.steps / world

    rw = default_config(random=True)
    walk, kt, ss, per_step = arm(rw, True, arithmetic="fp32", storage="fp16", rng="philox")
    plain_rw, _, _, _ = arm(rw, False, arithmetic="fp32", storage="fp16", rng="philox")
    det, kt_det, ss_det, _ = arm(default_config(random=False), True, arithmetic="fp32",
                                 storage="fp16")
    step_ms, walk_ms, fallback_ms = (float(x) for x in kt.mean(axis=0))
    run = float(ss["run"])
    peak, peak_kind = measured_peaks("bf16_tflops", 1590.0)
    achieved = run * SURROGATE_FLOP / (step_ms / 1000.0) / 1e12
    hbm, hbm_kind = measured_peaks()
    walk_gbs = per_step * B_ALG / (walk_ms / 1000.0) / 1e9
    per_particle = profile_traffic("surrogate_step_kernel_config3.md",
                                   "traffic_bytes_per_particle_interval")
    out = dict(walk)
    out.update({
        "unit": "particle-steps/s", "storage": "fp16", "rng": "philox",
        "diffusion": "plain stochastic operator per substep (sigma 3.46 m, AKT-scaled vertical), "
                     "surrogate displacement spread evenly over the substeps",
        "moved_by_surrogate_per_step": run, "fallback_per_step": float(ss["fallback"]),
        "vs_plain_random_walk": walk["value"] / plain_rw["value"],
        "plain_random_walk": dict(plain_rw, note="plain FP32 step, same workload, storage, random "
                                                 "walk and Philox streams"),
        "deterministic": dict(det, note="random walk off: the closed-form displacement kernel",
                              kernel_ms=[float(x) for x in kt_det.mean(axis=0)]),
        "kernel_ms": {"step": step_ms, "walk": walk_ms, "fallback": fallback_ms,
                      "timing": "per-interval events inside the timed loop, mean over K"},
        "roofline": {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak, "peak_source": peak_kind,
                     "kernel": "surrogate_step_kernel", "kernel_ms": step_ms,
                     "flop_per_particle_interval": SURROGATE_FLOP,
                     "traffic": None if per_particle is None else per_particle * run},
        "walk_roofline": {"bound": "hbm", "achieved": walk_gbs, "peak": hbm, "unit": "GB/s",
                          "frac": walk_gbs / hbm, "peak_source": hbm_kind,
                          "kernel": "surrogate_walk_kernel", "kernel_ms": walk_ms,
                          "algorithmic_bytes_per_particle_step": B_ALG},
    })
    if rank == 0 and not args.no_errors:
        n = min(len(particles), 1 << 20)
        sub = particles[:n].copy()
        hours = min(24, n_intervals)
        cfg = default_config(random=False)
        truth = run_hours(win, cfg, sub, hours, local_rank, arithmetic="reference")
        got = run_hours(win, cfg, sub, hours, local_rank, surrogate=True, arithmetic="fp32",
                        storage="fp16")
        out["error_m"] = error_stats(win, got, truth, hours, FP64)
        out["error_m_nonuniform"] = nonuniform_error(local_rank)
        out["_truth"] = truth
    return out


def precision_leg(args, win, particles, local_rank, truth, exchange, barrier):
    """The precision form: the plain FP32 step with FP32, FP16 and BF16 forcing storage, each
    device-timed on the full workload (a shorter run) with its 24-hour error on the 1,048,576-
    particle subset against the FP64 kernel; and the FP64 reference-arithmetic kernel's own
    throughput on the full workload."""
    from wacommplusplus_b200.engine import Engine
    from wacommplusplus_b200.types import default_config
    cfg = default_config(random=False)
    n_intervals = win.T - 1
    hours = min(24, n_intervals)
    sub = particles[:len(truth)]
    out = {}
    for storage, arithmetic in (("fp32", "fp32"), ("fp16", "fp32"), ("bf16", "fp32"),
                                ("fp32", "reference")):
        e = Engine(local_rank, arithmetic=arithmetic, storage=storage)
        e.set_config(cfg)
        e.load_window(win)
        e.set_particles(particles)
        steps = min(args.steps, 10 if arithmetic == "fp32" else 4)
        ms, count, kt, _ = timed_run(e, args, n_intervals, exchange, barrier, steps=steps,
                                     warmup=3)
        e.close()
        key = f"{storage}_storage" if arithmetic == "fp32" else "fp64_mode"
        entry = {"value": count / (ms / 1000.0), "ms_per_step": ms / steps, "steps": steps,
                 "kernel_ms": float(kt[:, 0].mean())}
        if arithmetic == "fp32":
            got = run_hours(win, cfg, sub, hours, local_rank, arithmetic="fp32", storage=storage)
            entry["error_m"] = error_stats(win, got, truth, hours, FP64)
        else:
            entry["note"] = "reference arithmetic (FP64, parity to 1e-9 deg), FP32 storage"
        out[key] = entry
    return out


def main():
    parser = argparse.ArgumentParser()
    parser.add_argument("--gpus", type=int, default=1)
    parser.add_argument("--steps", type=int, default=10)
    parser.add_argument("--warmup", type=int, default=3)
    parser.add_argument("--impl", default="ours", choices=["ours", "reference"])
    parser.add_argument("--particles", type=int, default=1 << 24)
    parser.add_argument("--storage", default="fp32", choices=["fp32", "fp16", "bf16"])
    parser.add_argument("--arithmetic", default="fp32", choices=["fp32", "reference"])
    parser.add_argument("--no-e2e", action="store_true")
    parser.add_argument("--no-cpu", action="store_true")
    parser.add_argument("--no-surrogate", action="store_true")
    parser.add_argument("--no-precision", action="store_true")
    parser.add_argument("--no-errors", action="store_true",
                        help="skip the 24-hour position-error runs of the surrogate arm")
    parser.add_argument("--no-realistic", action="store_true",
                        help="skip the realistic-grid key of the default line")
    parser.add_argument("--scenarios", type=int, default=256,
                        help="batched workload: number of scenarios")
    parser.add_argument("--workload", default="precision",
                        choices=["precision", "realistic", "batched"])
    args = parser.parse_args()
    if args.warmup < 3:
        args.warmup = 3

    if args.impl == "reference":
        run_reference(args)
        return
    if args.workload == "realistic":
        run_realistic(args)
        return
    if args.workload == "batched":
        run_batched(args)
        return

    import torch
    import torch.distributed as dist

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local_rank)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local_rank))

    from wacommplusplus_b200.engine import Engine

    win, particles, cfg = workload(args.particles, rank)
    cpu = None
    if rank == 0 and not args.no_cpu:
        threads, how = physical_cores()
        rate, kind, sample = cpu_reference_rate(win, particles, cfg, threads)
        rate1, _, sample1 = cpu_reference_rate(win, particles, cfg, 1, repeats=1, sample=16384)
        cpu = {"value": rate, "unit": "particle-steps/s", "cores": threads,
               "cores_counted_as": how, "kind": kind,
               "sample": f"{sample} particles x 120 substeps, one interval: Particle::move "
                         "(OpenMP dynamic,64) + Concentration::evaluate, one thread per physical "
                         "core (OMP_PLACES=cores, OMP_PROC_BIND=close), median of 3 after a warm-up",
               "value_1core": rate1}

    from wacommplusplus_b200 import sharding

    engine = Engine(local_rank, arithmetic=args.arithmetic, storage=args.storage)
    engine.load_window(win)
    engine.set_config(cfg)
    engine.set_particles(particles)
    engine.concentration_reset(win.T)
    n_intervals = win.T - 1

    def barrier():
        if world > 1:
            dist.barrier()

    def exchange(eng, t):
        # the interval's concentration slice summed over the particle shards (N > 1)
        if world > 1:
            sharding.allreduce_concentration(eng, t + 1)

    sampler = ClockSampler(physical_gpu(local_rank))
    sampler.start()
    # the K intervals are enqueued back to back; the kernels count their particle-steps on the
    # device, read once after the timed region, and the move kernel of every interval is timed by
    # events recorded inside the same loop
    elapsed_ms, steps_total, kt, launches = timed_run(engine, args, n_intervals, exchange, barrier)
    clocks = sampler.stop()
    launches *= args.steps
    per_launch_steps = steps_total / args.steps
    elapsed_ms, steps_total = over_ranks(dist, world, elapsed_ms, steps_total)
    value = steps_total / (elapsed_ms / 1000.0)

    kernel_ms = float(kt[:, 0].mean())
    achieved = per_launch_steps * B_ALG / (kernel_ms / 1000.0) / 1e9
    peak, peak_kind = measured_peaks()
    traffic_per_step = profile_traffic()
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_source": peak_kind,
                "traffic": None if traffic_per_step is None else traffic_per_step * per_launch_steps,
                "kernel": "move_fast_kernel (FP32 step)" if args.arithmetic == "fp32" else "move_soa_kernel (reference arithmetic)",
                "kernel_ms": kernel_ms,
                "kernel_ms_timing": "per-interval events inside the timed loop, mean over K",
                "algorithmic_bytes_per_particle_step": B_ALG}

    e2e = None
    if not args.no_e2e:
        n = len(particles)
        host = torch.empty(n * 64, dtype=torch.uint8, pin_memory=True)
        host.numpy()[:] = particles.view(np.uint8).reshape(-1)
        frame_bytes = win.nbytes_frame
        for s in range(2):
            engine.move_interval_host_ptr(s % n_intervals, host.data_ptr(), n)
            exchange(engine, s % n_intervals)
        # two page-locked staging records, alternating: the record of interval s+2 is copied
        # while interval s computes, and is free again once interval s+1 has returned
        fields = ("zeta", "u", "v", "w", "akt")
        staging = [{k: torch.empty(win.frame(0)[k].shape, dtype=torch.float32,
                                   pin_memory=True).numpy() for k in fields} for _ in range(2)]
        barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e2e_steps = 0.0
        for s in range(args.steps):
            t = (args.warmup + s) % n_intervals
            if t + 2 < win.T:
                f, buf = win.frame(t + 2), staging[s % 2]
                for k in fields:
                    buf[k][...] = f[k]
                engine.upload_frame_async(t + 2, *(buf[k] for k in fields))
            engine.move_interval_host_ptr(t, host.data_ptr(), n)
            exchange(engine, t)
            e2e_steps += engine.stats()["particle_steps"]
        engine.synchronize()
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        if world > 1:
            t = torch.tensor([dt, e2e_steps], dtype=torch.float64, device="cuda")
            mx = t.clone()
            dist.all_reduce(mx, op=dist.ReduceOp.MAX)
            dist.all_reduce(t, op=dist.ReduceOp.SUM)
            dt, e2e_steps = float(mx[0]), float(t[1])
        e2e = {"value": e2e_steps / dt, "unit": "particle-steps/s",
               "h2d_bytes_per_step": n * 64 + frame_bytes, "d2h_bytes_per_step": n * 64,
               "timing": "wall clock around K steps of upload_frame_async (record of the interval after "
                         "next, from page-locked memory) + move_interval_host"}

    engine.close()
    surrogate = precision = None
    if not args.no_surrogate:
        surrogate = surrogate_leg(args, win, particles, local_rank, world, rank, barrier, dist,
                                  exchange)
        truth = surrogate.pop("_truth", None)
        if rank == 0 and not args.no_precision and truth is not None:
            # rank 0 alone, no collectives: the other ranks wait at the final barrier
            precision = precision_leg(args, win, particles, local_rank, truth,
                                      lambda eng, t: None, lambda: None)
    realistic = None
    if rank == 0 and world == 1 and not args.no_realistic:
        # the realistic grid as a second workload of the default line (4,194,304 particles,
        # 3 warm-up and 5 timed intervals; records generated on the device)
        r = realistic_leg(1 << 22, 3, 5, not args.no_cpu)
        realistic = {key: r[key] for key in ("value", "unit", "steps", "warmup", "ms_per_step",
                                             "move_kernel_ms", "roofline", "cpu_baseline",
                                             "gpu_launches", "clocks")}
        realistic["workload"] = r["config"]["workload"]
        realistic["particles_alive_at_timing"] = r["config"]["particles_alive_at_timing"]

    if rank == 0:
        line = {
            "metric": "particle-steps/s", "value": value, "unit": "particle-steps/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": elapsed_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32" if args.arithmetic == "fp32" else "f64",
            "data": "synthetic",
            "config": {"workload": "precision-form analytic grid 128x128x10 (lon 14.00-14.20 E, "
                                   "lat 40.70-40.90 N), 25 hourly records, u=0.2 v=0.1 m/s, "
                                   f"{args.particles} particles per GPU, deterministic midpoint, "
                                   f"dt=30 s, forcing storage {args.storage}, arithmetic "
                                   f"{args.arithmetic}",
                       "l2": "inputs larger than L2 (particle state 1 GiB per GPU)",
                       "concentration": "fused uint32 counts each interval; for N > 1 the "
                                        "interval's grid slice is summed over the shards by an "
                                        "NCCL all-reduce inside the timed region",
                       "parallelism": f"particle shards x{world}, one concentration all-reduce "
                                      "per interval"},
            "roofline": roofline,
            "surrogate": surrogate,
            "precision": precision,
            "realistic": realistic,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": launches,
            "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
