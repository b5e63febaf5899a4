"""Benchmark of the per-generation BRKGA hot path on B200.

Workload (the headline configuration): Euclidean TSP, n = 1000 cities with FP32
coordinates uniform in [0,1)^2 (seeded), population 2048, elite 307 (0.15), mutants 307
(0.15), rho = 0.7; one step = one generation (fused crossover / mutant fill / decode /
tour length kernel + elite-partition sort) of the device-resident solver.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs N independent replicas (one instance per GPU, no collective: islands and
instances are independent units), launched one process per GPU by torch.distributed.run.
One timed step is a stretch of GENS_PER_STEP generations of the device-resident solver
(one evolve call: captured CUDA graphs of 16 generations each), with L2 flushed (a 256 MiB
write) before every step, outside its CUDA-event bracket; inside a step the 16 MB
population stays L2-resident as it does in a solver run.  The JSON line's `value` is
whole-job generations per second with the population resident in HBM;
`l2_flushed_gens_per_s` times single generations with L2 flushed before each.  `e2e` is the
same metric through the C ABI from host buffers: each e2e step is one whole
1000-generation solve (problem upload from pinned memory, create, initialise, evolve, read
the best tour back).  At N = 1 the line also nests the batched (256 island instances),
served (Poisson mixed stream) and 32-seed quality measurements.
"""
from __future__ import annotations

import argparse
import json

import numpy as np
import os
import re
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
for _p in (os.path.join(ROOT, "llm-brkga_b200"), os.path.join(ROOT, "oracle")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = "gens/s TSP n=1000 pop 2048"
N_CITIES, POP, ELITE, MUTANTS, RHO = 1000, 2048, 307, 307, 0.7
E2E_GENERATIONS = 1000
GENS_PER_STEP = 4096  # generations per timed step (about 0.13 s of device work)
SEED_INSTANCE, SEED_GA = 2026, 7
PROFILE = os.path.join(ROOT, "profiles", "row_kernel_tsp_n1000_p2048.md")
HOLD_CYCLES_PER_STEP = 400_000  # ~0.2 ms of device spin per queued step (host enqueue cost)


def workload_config():
    """the headline workload, identical in both arms' lines"""
    return {"workload": f"TSP n={N_CITIES} pop={POP} elite={ELITE} mutants={MUTANTS} rho={RHO}",
            "n": N_CITIES, "population": POP, "elite": ELITE, "mutants": MUTANTS, "rho": RHO}


def instance():
    import numpy as np
    return np.random.default_rng(SEED_INSTANCE).random((N_CITIES, 2), dtype=np.float32)


def algorithmic_bytes_per_generation():
    """bytes the fused row kernel must move for one generation (keys FP32):
    elite rows read + written, each child reads one inherited gene per gene and writes its
    row, each mutant writes its row, fitness written, coordinates read once."""
    n, P, E, M = N_CITIES, POP, ELITE, MUTANTS
    off = P - E - M
    return (2 * E * n + 2 * off * n + M * n) * 4 + P * 4 + n * 8


# ---------------------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index, self.rows, self.proc = index, [], None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm = [float(r[0]) for r in self.rows if len(r) >= 8 and r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if len(r) >= 8 and r[1].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            for i, nm in enumerate(names):
                if len(r) >= 8 and r[4 + i].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def profile_figure(key):
    """a figure of the row kernel's committed ncu summary (`key: value` line), or None"""
    try:
        txt = open(PROFILE).read()
    except OSError:
        return None
    m = re.search(key + r":\s*([0-9.eE+]+)", txt)
    return float(m.group(1)) if m else None


def profile_traffic():
    """DRAM bytes per launch of the row kernel from the committed ncu summary, or None"""
    return profile_figure("traffic_bytes_per_launch")


# ---------------------------------------------------------------------------------------
# CPU baseline: the reference's own generation (its CPU path), or the oracle port
# ---------------------------------------------------------------------------------------
def cpu_baseline(seconds=15.0, max_gens=200):
    code = f"""
import json, os, sys, time
sys.path[:0] = [{os.path.join(ROOT, 'oracle')!r}, {os.path.join(ROOT, 'tests')!r}]
import numpy as np
import oracle as O
xy = np.random.default_rng({SEED_INSTANCE}).random(({N_CITIES}, 2), dtype=np.float32)
budget, max_gens = {seconds}, {max_gens}
if O.ref_available():
    R = O.ref()
    h = R.ref_solver_create(1, {N_CITIES}, xy.ctypes.data, None, None, None, 0.0, {POP}, {ELITE}, {MUTANTS}, {RHO})
    assert h, "reference solver creation failed"
    mode = R.ref_solver_mode(h).decode()
    R.ref_solver_evolve(h, 1)
    gens, t = 0, 0.0
    while t < budget and gens < max_gens:
        t += R.ref_solver_evolve(h, 1)
        gens += 1
    R.ref_solver_destroy(h)
    print(json.dumps(dict(kind="reference", value=gens / t, gens=gens, seconds=t, mode=mode)))
else:
    pb = O.OracleProblem(O.TSP_COORDS, {N_CITIES}, xy=xy)
    pr = O.params({POP}, {ELITE}, {MUTANTS}, {RHO}, 1)
    ld = {N_CITIES}
    pop, fit = O.brkga_init(pb, pr, ld)
    srt = O.sort_fitness(fit)
    gens, t = 0, 0.0
    while t < budget and gens < max_gens:
        t0 = time.perf_counter()
        pop, fit = O.brkga_generation(pb, pr, gens + 1, pop, fit, srt, ld)
        srt = O.sort_fitness(fit)
        t += time.perf_counter() - t0
        gens += 1
    print(json.dumps(dict(kind="port", value=gens / t, gens=gens, seconds=t, mode="cpu")))
"""
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=600)
    if r.returncode != 0:
        raise RuntimeError("CPU baseline failed: " + r.stderr[-2000:])
    d = json.loads(r.stdout.strip().splitlines()[-1])
    return {"value": d["value"], "unit": "gens/s", "cores": 1, "kind": d["kind"],
            "sample": f"{d['gens']} generations of the same workload ({d['seconds']:.1f} s, reference "
                      f"execution mode '{d['mode']}', single-threaded like the reference's CPU path)"}


# ---------------------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------------------
def run_ours(args, rank, world):
    import numpy as np
    import torch

    import brkga_b200 as B

    from brkga_b200.replicas import Replicas, whole_job_rate

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    reps = Replicas(backend="nccl")

    def barrier():
        reps.barrier()
        torch.cuda.synchronize()

    xy = instance()
    pb = B.tsp(xy, device=dev)
    prm = B.params(POP, ELITE, MUTANTS, RHO, E2E_GENERATIONS, seed=reps.seed(SEED_GA), device=dev)
    s = B.Solver(pb, prm)
    s_info = s.info
    s.initialize()
    stream = torch.cuda.ExternalStream(s.stream, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    gps = args.gens_per_step
    for _ in range(args.warmup):
        with torch.cuda.stream(stream):
            flush.fill_(1.0)
        s.evolve(gps)
    s.synchronize()

    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    barrier()
    with ClockSampler(dev) as clocks:
        # hold the stream while the host queues the first steps, so no host gap lands
        # inside an event bracket (the hold itself is outside every bracket)
        with torch.cuda.stream(stream):
            torch.cuda._sleep(HOLD_CYCLES_PER_STEP * 16)
        for i in range(args.steps):
            with torch.cuda.stream(stream):
                flush.fill_(float(i))
                starts[i].record(stream)
            s.evolve(gps)
            with torch.cuda.stream(stream):
                ends[i].record(stream)
        s.synchronize()
        barrier()
    ms = reps.max(sum(a.elapsed_time(b) for a, b in zip(starts, ends)))
    value = whole_job_rate(world, args.steps * gps, ms / 1e3)
    best = float(s.get_best_individual()[2])

    # --- single generations with L2 flushed before each (the population re-read from HBM)
    f_starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    f_ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    with torch.cuda.stream(stream):
        torch.cuda._sleep(HOLD_CYCLES_PER_STEP * args.steps)
    for i in range(args.steps):
        with torch.cuda.stream(stream):
            flush.fill_(float(i))
            f_starts[i].record(stream)
        s.evolve(1)
        with torch.cuda.stream(stream):
            f_ends[i].record(stream)
    s.synchronize()
    f_ms = reps.max(sum(a.elapsed_time(b) for a, b in zip(f_starts, f_ends)))
    flushed_value = whole_job_rate(world, args.steps, f_ms / 1e3)

    # --- dominant kernel alone: the fused row kernel through the generation-step entry point
    ld = (N_CITIES + 3) // 4 * 4
    d_pop = torch.from_numpy(np.random.default_rng(1).random((POP, ld), dtype=np.float32)).to(dev)
    d_fit = torch.rand(POP, device=dev)
    d_srt = torch.zeros(POP, dtype=torch.int32, device=dev)
    B.sort_fitness(d_fit, POP, 1, False, d_srt)
    d_next = torch.zeros_like(d_pop)
    d_nfit = torch.zeros_like(d_fit)
    cur = torch.cuda.current_stream()
    kstarts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    kends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    sstarts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    sends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    for i in range(args.warmup):
        B.generation_step(pb, d_pop, d_fit, d_srt, d_next, d_nfit, POP, ELITE, MUTANTS, RHO, ld, SEED_GA, i + 1,
                          stream=cur)
    torch.cuda.synchronize()
    torch.cuda._sleep(2 * HOLD_CYCLES_PER_STEP * args.steps)
    for i in range(args.steps):
        flush.fill_(float(i))
        kstarts[i].record(cur)
        B.generation_step(pb, d_pop, d_fit, d_srt, d_next, d_nfit, POP, ELITE, MUTANTS, RHO, ld, SEED_GA, i + 1,
                          stream=cur)
        kends[i].record(cur)
        flush.fill_(float(i))
        sstarts[i].record(cur)
        B.sort_fitness(d_nfit, POP, 1, False, d_srt, stream=cur)
        sends[i].record(cur)
    torch.cuda.synchronize()
    row_ms = sum(a.elapsed_time(b) for a, b in zip(kstarts, kends)) / args.steps
    sort_ms = sum(a.elapsed_time(b) for a, b in zip(sstarts, sends)) / args.steps

    # --- end to end through the C ABI from host buffers: one whole solve per step
    e2e = None
    if not args.no_e2e:
        pinned = torch.from_numpy(xy).pin_memory()
        xy_host = pinned.numpy()
        keys = np.zeros(N_CITIES, np.float32)
        perm = np.zeros(N_CITIES, np.int32)
        e2e_steps = max(1, min(args.steps, 5))
        times = []
        phases = {"create_ms": 0.0, "run_ms": 0.0, "get_best_ms": 0.0, "destroy_ms": 0.0}
        for i in range(1 + e2e_steps):
            barrier()
            t0 = time.perf_counter()
            pe = B.tsp(xy_host, device=dev)
            se = B.Solver(pe, B.params(POP, ELITE, MUTANTS, RHO, E2E_GENERATIONS, seed=100 + i, device=dev))
            t1 = time.perf_counter()
            se.run()
            t2 = time.perf_counter()
            k2, p2, f2 = se.get_best_individual()
            t3 = time.perf_counter()
            se.close()
            pe.close()
            barrier()
            t4 = time.perf_counter()
            if i > 0:
                times.append(t4 - t0)
                for key, dt in (("create_ms", t1 - t0), ("run_ms", t2 - t1), ("get_best_ms", t3 - t2),
                                ("destroy_ms", t4 - t3)):
                    phases[key] += 1e3 * dt / e2e_steps
        tt = reps.max(sum(times))
        e2e = {"value": whole_job_rate(world, e2e_steps * E2E_GENERATIONS, tt), "unit": "gens/s",
               "h2d_bytes_per_step": int(xy.nbytes), "d2h_bytes_per_step": int(keys.nbytes + perm.nbytes + 4),
               "step": f"one {E2E_GENERATIONS}-generation solve through brkga_problem_create / brkga_create / "
                       f"brkga_run / brkga_get_best", "ms_per_solve": 1e3 * tt / e2e_steps,
               "phases": {k: round(v, 3) for k, v in phases.items()}}

    peak, peak_kind = measured_peak()
    alg = algorithmic_bytes_per_generation()
    achieved = alg / (row_ms / 1e3) / 1e9
    out = None
    if rank == 0:
        out = {
            "metric": METRIC, "value": value, "unit": "gens/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded uniform coordinates)",
            "config": workload_config(),
            "generations_per_step": gps,
            "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
            "l2": f"flushed (256 MiB write) before every timed step of {gps} generations, outside the timing; "
                  "within a step the population stays L2-resident as in a solver run",
            "l2_flushed_gens_per_s": flushed_value,
            "impl": "ours",
            "e2e": e2e,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": profile_traffic(),
                         "kernel": "bk::row_kernel<256,1> (fused crossover/mutant/decode/tour length), "
                                   "timed through brkga_generation_step",
                         "traffic_note": "DRAM bytes per launch from profiles/row_kernel_tsp_n1000_p2048.md",
                         "engine_tile": {"threads": s_info[0], "groups": s_info[1], "grid": s_info[2],
                                         "coords_in_smem": bool(s_info[3])},
                         "algorithmic_bytes_per_launch": alg, "kernel_ms": row_ms, "peak_kind": peak_kind,
                         "sort_kernel_ms": sort_ms,
                         # the in-block argsort's bound: shared-memory pipe utilisation of the
                         # same kernel (ncu, wavefronts as % of the per-SM peak over the
                         # kernel's elapsed time)
                         "smem": {"wavefront_pct_of_peak": profile_figure("smem_wavefront_pct_of_peak"),
                                  "source": "profiles/row_kernel_tsp_n1000_p2048.md"}},
            "gpu_launches": 2 * args.steps * gps,
            # rows decoded and evaluated per generation: children and mutants (elites keep
            # their fitness, as the reference's host path does)
            "individual_evaluations_per_s": value * (POP - ELITE),
            "clocks": clocks.summary(),
            "best_tour": best,
        }
    s.close()
    reps.close()
    return out


# ---------------------------------------------------------------------------------------
# the other workloads (one JSON line each; the default run measures the headline only)
# ---------------------------------------------------------------------------------------
def _events_time(fn, stream=None):
    import torch
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a.record(stream)
    fn()
    b.record(stream)
    torch.cuda.synchronize()
    return a.elapsed_time(b) / 1e3


def workload_solver(args, name, problem_fn, prm_kwargs, gens, cpu_kind=None, cpu_args=None):
    """gens/s of one device-resident solver run (population resident, L2 warm between
    generations because the whole run is one enqueue) and the reference's CPU path"""
    import torch
    import brkga_b200 as B
    pb = problem_fn()
    s = B.Solver(pb, B.params(**prm_kwargs))
    s.initialize()
    s.evolve(args.warmup)
    s.synchronize()
    stream = torch.cuda.ExternalStream(s.stream)
    with torch.cuda.stream(stream):
        torch.cuda._sleep(HOLD_CYCLES_PER_STEP)
    secs = _events_time(lambda: s.evolve(gens), stream)
    best = s.get_best_individual()[2]
    out = {"metric": f"gens/s {name}", "value": gens / secs, "unit": "gens/s", "generations": gens,
           "best": np.asarray(best, np.float64).tolist(), "workload": name,
           "engine_tile": s.info}
    if cpu_kind is not None and not args.no_cpu:
        out["cpu_baseline"] = cpu_reference(cpu_kind, cpu_args, seconds=10.0)
    return out


def cpu_reference(kind, a, seconds=10.0, max_gens=2000):
    """the reference's own Solver on its CPU path (oracle/_ref), generations per second"""
    code = f"""
import json, sys, time
sys.path[:0] = [{os.path.join(ROOT, 'oracle')!r}]
import numpy as np
import oracle as O
a = {a!r}
if a.get('movrp'):
    rng = np.random.default_rng(a['seed'])
    xy = (rng.random((a['n'] + 1, 2)) * 100.0).astype(np.float32)
    dem = rng.integers(1, 31, a['n'] + 1).astype(np.int32)
    dem[0] = 0
elif a.get('tspj'):
    rng = np.random.default_rng(a['seed'])
    pts = rng.random((a['n'] + 1, 2)) * 100.0
    xy = np.ascontiguousarray(np.sqrt(((pts[:, None, :] - pts[None, :, :]) ** 2).sum(-1)).astype(np.float32))
    xy2 = (1.0 + rng.random((a['n'] + 1, a['n'] + 1)) * 99.0).astype(np.float32)
    xy2[0, :] = 0.0
else:
    xy = np.random.default_rng(a['seed']).random((a['pts'], 2), dtype=np.float32) * np.float32(a.get('scale', 1.0))
    xy2 = np.random.default_rng(a['seed'] + 1).random((a['pts'], 2), dtype=np.float32)
if not O.ref_available():
    print(json.dumps(dict(value=None))); sys.exit(0)
R = O.ref()
if a.get('movrp'):
    h = R.ref_solver_create_movrp(xy, dem, a['n'], a['cap'], a['V'], a['P'], 0.10)
else:
    h = R.ref_solver_create({kind}, a['n'], xy.ctypes.data, xy2.ctypes.data, None, None, 0.0, a['P'], a['E'],
                            a['M'], 0.75 if a.get('tspj') else 0.7)
R.ref_solver_evolve(h, 1)
g, t = 0, 0.0
while t < {seconds} and g < {max_gens}:
    t += R.ref_solver_evolve(h, 1); g += 1
print(json.dumps(dict(value=g / t, gens=g, seconds=t)))
"""
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=900)
    if r.returncode != 0:
        return {"error": r.stderr[-500:]}
    d = json.loads(r.stdout.strip().splitlines()[-1])
    if d.get("value") is None:
        return None
    return {"value": d["value"], "unit": "gens/s", "cores": 1, "kind": "reference",
            "sample": f"{d['gens']} generations ({d['seconds']:.1f} s) of the same workload"}


def workload_external(args):
    """a config that brings its own fitness, as the reference's LLM solver writes them
    (cpp/examples/solve_external.cu: single-machine weighted completion time, n=40, P=256,
    E=51, M=25, rho=0.7, generated-main flow): generations/s with its host
    fitness_function and with its own CUDA kernel, and the reference's CPU solver on the
    same config and instance"""
    exe = os.path.join(ROOT, "llm-brkga_b200", "build", "solve_external")
    gens = args.generations
    out = {"metric": "gens/s LLM-style config, weighted completion time n=40 pop 256", "unit": "gens/s",
           "generations": gens, "workload": "external fitness (BRKGA_EXTERNAL) through the drop-in Solver"}
    for mode in ("host", "gpu"):
        r = subprocess.run([exe, mode, "40", "1", str(gens)], capture_output=True, text=True, timeout=900)
        if r.returncode != 0:
            raise SystemExit(f"solve_external {mode} failed: {r.stderr[-500:]}")
        d = json.loads(r.stdout.strip().splitlines()[-1])
        key = "value" if mode == "host" else "gpu_fitness_value"
        out[key] = gens / d["seconds"]
        out["best_" + mode] = d["best"]
    if not args.no_cpu:
        code = f"""
import json, sys
sys.path[:0] = [{os.path.join(ROOT, 'oracle')!r}]
import oracle as O
if not O.ref_available():
    print(json.dumps(dict(value=None))); sys.exit(0)
R = O.ref()
h = R.ref_solver_create_wct(40, 1, 256, 51, 25, 0.7)
R.ref_solver_evolve(h, 1)
g, t = 0, 0.0
while t < 10.0 and g < {gens}:
    t += R.ref_solver_evolve(h, 1); g += 1
print(json.dumps(dict(value=g / t, gens=g, seconds=t, best=R.ref_solver_best(h))))
"""
        env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
        r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=900)
        if r.returncode == 0:
            d = json.loads(r.stdout.strip().splitlines()[-1])
            if d.get("value") is not None:
                out["cpu_baseline"] = {"value": d["value"], "unit": "gens/s", "cores": 1, "kind": "reference",
                                       "sample": f"{d['gens']} generations ({d['seconds']:.1f} s) of the same config"}
                out["best_reference"] = d["best"]
        else:
            out["cpu_baseline"] = {"error": r.stderr[-500:]}
    return out


def workload_batch(args):
    """256 TSP instances, n ~ U[100,2000], P in {256,512,1024}, 4 islands migrating the 2
    best every 50 generations, 500 generations, in one batch; against the same instances
    solved one after another by the plain solver (timed on a sample)"""
    import torch
    import brkga_b200 as B
    rng = np.random.default_rng(4)
    count, gens = args.instances, args.generations
    ns = rng.integers(100, 2001, count)
    Ps = rng.choice([256, 512, 1024], count)
    probs, prms = [], []
    for i in range(count):
        xy = np.random.default_rng(1000 + i).random((int(ns[i]), 2), dtype=np.float32)
        P = int(Ps[i])
        probs.append(B.tsp(xy))
        prms.append(B.params(P, int(0.15 * P), int(0.15 * P), 0.7, gens, seed=2000 + i, num_islands=4,
                             migration_interval=50, num_migrants=2))
    t0 = time.perf_counter()
    batch = B.Batch(probs, prms)
    batch.synchronize()
    t_create = time.perf_counter() - t0
    secs = _events_time(lambda: (batch.evolve(gens), batch.synchronize()))
    best_b = batch.best()[:, 0]
    batch.close()
    # plain solver, one instance at a time, on a sample of the same instances
    sample = list(range(0, count, max(1, count // 16)))
    tsum = 0.0
    same = 0
    for i in sample:
        s = B.Solver(probs[i], prms[i])
        t = _events_time(lambda: (s.run(), s.synchronize()))
        tsum += t
        same += int(s.get_best_individual()[2] == best_b[i])
        s.close()
    plain_per_instance = tsum / len(sample)
    return {"metric": "instance-generations/s batched TSP islands", "value": count * gens / secs,
            "unit": "instance-gens/s", "instances": count, "generations": gens, "seconds": secs,
            "create_seconds": t_create, "plain_solver_instance_gens_per_s": gens / plain_per_instance,
            "speedup_vs_plain": (count * gens / secs) / (gens / plain_per_instance),
            "sample_results_identical_to_plain": f"{same}/{len(sample)}",
            "elements_per_generation": int(sum(int(p) * int(n) for p, n in zip(Ps, ns)))}


def workload_serve(args):
    """Poisson arrivals: 50% TSP (n ~ U[50,5000], P 512), 30% greedy knapsack (n ~
    U[500,10000], weights/values U{1..100}, capacity half the weight, P 1024), 20%
    bi-objective TSP NSGA-II (n 300, P 512), 500 generations each"""
    import brkga_b200 as B
    rng = np.random.default_rng(5)
    rate, dur, gens = args.rate, args.duration, args.generations
    t, arrivals = 0.0, []
    while True:
        t += rng.exponential(1.0 / rate)
        if t > dur:
            break
        arrivals.append(t)
    reqs = []
    for i, at in enumerate(arrivals):
        u = rng.random()
        if u < 0.5:
            n = int(rng.integers(50, 5001))
            reqs.append((at, dict(kind=B.TSP_COORDS, n=n, coords=rng.random((n, 2), dtype=np.float32)),
                         B.params(512, 76, 76, 0.7, gens, seed=i)))
        elif u < 0.8:
            n = int(rng.integers(500, 10001))
            w = rng.integers(1, 101, n).astype(np.int32)
            v = rng.integers(1, 101, n).astype(np.int32)
            reqs.append((at, dict(kind=B.KNAP_GREEDY, n=n, weights=w, values=v, capacity=0.5 * float(w.sum())),
                         B.params(1024, 153, 153, 0.7, gens, seed=i)))
        else:
            n = 300
            reqs.append((at, dict(kind=B.BITSP_COORDS, n=n, coords=rng.random((n + 1, 2), dtype=np.float32),
                                  coords2=rng.random((n + 1, 2), dtype=np.float32)),
                         B.params(512, 0, 51, 0.7, gens, seed=i)))
    srv = B.Server(max_active=args.max_active, generations_per_tick=args.tick)
    ids, k = [], 0
    t0 = time.perf_counter()
    done = {}
    while len(done) < len(reqs):
        now = time.perf_counter() - t0
        while k < len(reqs) and reqs[k][0] <= now:
            at, kw, prm = reqs[k]
            ids.append(srv.submit(prm=prm, **kw))
            k += 1
        if k < len(reqs) and srv.stats()[1] == 0 and srv.stats()[0] == 0:
            time.sleep(max(0.0, reqs[k][0] - (time.perf_counter() - t0)))
            continue
        srv.step()
        for rid in ids:
            if rid not in done:
                r = srv.poll(rid)
                if r is not None:
                    done[rid] = r
    makespan = time.perf_counter() - t0
    lat = np.array([done[r][3] for r in ids])
    srv.close()
    # plain solver (the drop-in, one request at a time, alone on the GPU) on every k-th
    # request of the same stream; its best must equal the served one (results do not depend
    # on what else shares the GPU)
    every = max(1, args.plain_every)
    sample = list(range(0, len(reqs), every))
    tsum, same = 0.0, 0
    for i in sample:
        _, kw, prm = reqs[i]
        kw = dict(kw)
        kind = kw.pop("kind")
        n = kw.pop("n")
        pb = B.Problem(kind, n, **kw)
        t1 = time.perf_counter()
        s = B.Solver(pb, prm)
        s.run()
        best = s.get_best_individual()[2]
        s.close()
        tsum += time.perf_counter() - t1
        pb.close()
        m = 2 if kind == B.BITSP_COORDS else 1
        served_best = np.asarray(done[ids[i]][1], np.float32).reshape(-1)[:m]
        same += int(np.array_equal(np.asarray(best, np.float32).reshape(-1)[:m], served_best))
    plain = len(sample) / tsum
    kinds = {"tsp": 0, "knapsack": 0, "bitsp": 0}
    for _, kw, _ in reqs:
        kinds["tsp" if kw["kind"] == B.TSP_COORDS else "knapsack" if kw["kind"] == B.KNAP_GREEDY else "bitsp"] += 1
    return {"metric": "served solves/s mixed stream", "value": len(reqs) / makespan, "unit": "solves/s",
            "requests": len(reqs), "mix": kinds, "arrival_rate": rate, "arrival_seconds": dur,
            "makespan_s": makespan,
            "latency_p50_s": float(np.percentile(lat, 50)), "latency_p99_s": float(np.percentile(lat, 99)),
            "plain_solver_solves_per_s": plain, "plain_solver_sample": f"every {every}th request ({len(sample)})",
            "speedup_vs_plain": (len(reqs) / makespan) / plain,
            "sample_results_identical_to_plain": f"{same}/{len(sample)}",
            "generations": gens, "max_active": args.max_active, "tick": args.tick}


def workload_operators(args):
    """Each hot-path operator alone on the headline sizes (TSP n=1000, P=2048; Pareto ranks on
    a 2P = 4096 pool), device-resident buffers, CUDA events with L2 flushed before every
    launch; beside it the reference's own CPU code for the same operator (oracle/_ref, CUDA
    hidden, one thread)"""
    import torch
    import brkga_b200 as B
    dev = torch.device("cuda:0")
    xy = instance()
    pb = B.tsp(xy)
    n, P = N_CITIES, POP
    rng = np.random.default_rng(7)
    keys = (rng.integers(0, 1 << 24, (P, n)) / float(1 << 24)).astype(np.float32)
    d_pop = torch.from_numpy(keys).to(dev)
    d_fit = torch.zeros(P, dtype=torch.float32, device=dev)
    d_srt = torch.zeros(P, dtype=torch.int32, device=dev)
    d_next = torch.zeros_like(d_pop)
    d_nfit = torch.zeros_like(d_fit)
    N2 = 2 * P
    obj = rng.random((N2, 2), dtype=np.float32)
    d_obj = torch.from_numpy(obj).to(dev)
    d_rank = torch.zeros(N2, dtype=torch.int32, device=dev)
    d_cd = torch.zeros(N2, dtype=torch.float32, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    cur = torch.cuda.current_stream()
    pb.evaluate_population(d_pop, d_fit, P, n, stream=cur)
    B.sort_fitness(d_fit, P, 1, False, d_srt, stream=cur)

    def timed(fn, reps=30):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        tot = 0.0
        for i in range(reps):
            flush.fill_(float(i))
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(cur)
            fn()
            b.record(cur)
            b.synchronize()
            tot += a.elapsed_time(b)
        return 1e3 * tot / reps  # us

    gen = [0]

    def generation():
        gen[0] += 1
        B.generation_step(pb, d_pop, d_fit, d_srt, d_next, d_nfit, P, ELITE, MUTANTS, RHO, n, SEED_GA, gen[0],
                          stream=cur)
        B.sort_fitness(d_nfit, P, 1, False, d_srt, stream=cur)

    gpu = {
        "decode + tour length": timed(lambda: pb.evaluate_population(d_pop, d_fit, P, n, stream=cur)),
        "elite partition": timed(lambda: B.sort_fitness(d_fit, P, 1, False, d_srt, stream=cur)),
        "generation (crossover, mutants, decode, tour length, partition)": timed(generation),
        "Pareto ranks + crowding (4096 points)": timed(lambda: (B.pareto_rank(d_obj, N2, 2, d_rank, stream=cur),
                                                               B.crowding(d_obj, d_rank, N2, 2, d_cd, stream=cur))),
    }
    fit_sorted = np.sort(d_fit.cpu().numpy().astype(np.float32))
    cpu = _cpu_operators(xy, keys, fit_sorted, obj)
    rows = []
    for k, g_us in gpu.items():
        c = cpu.get(k) if cpu else None
        rows.append({"operator": k, "gpu_us": round(g_us, 2), "reference_cpu_us": None if c is None else round(c, 1),
                     "ratio": None if c is None else round(c / g_us, 1)})
    return {"metric": "hot-path operators, device time vs the reference's CPU code", "unit": "us per call",
            "sizes": f"TSP n={n} P={P}; Pareto pool {N2} x 2 objectives", "operators": rows,
            "reference_cores": 1, "l2": "flushed before every timed launch"}


def _cpu_operators(xy, keys, fit_sorted, obj):
    """the reference's CPU operators in a child process with CUDA hidden (its CPU path)"""
    import tempfile
    with tempfile.TemporaryDirectory() as td:
        np.save(os.path.join(td, "xy.npy"), xy)
        np.save(os.path.join(td, "keys.npy"), keys)
        np.save(os.path.join(td, "fit.npy"), fit_sorted)
        np.save(os.path.join(td, "obj.npy"), obj)
        code = f"""
import json, sys, time
sys.path[:0] = [{os.path.join(ROOT, 'oracle')!r}]
import numpy as np
import oracle as O
if not O.ref_available():
    print(json.dumps(None)); sys.exit(0)
R = O.ref()
td = {td!r}
xy = np.load(td + '/xy.npy'); keys = np.load(td + '/keys.npy'); fit = np.load(td + '/fit.npy'); obj = np.load(td + '/obj.npy')
P, n = keys.shape
def ev(rows):  # the call also builds the config's distance matrix: timed apart by difference
    f = np.zeros(rows, np.float32)
    k = np.ascontiguousarray(keys[:rows])
    t0 = time.perf_counter(); R.ref_tsp_eval(xy.ctypes.data, None, n, k, rows, f, None)
    return time.perf_counter() - t0
out = {{}}
out['decode + tour length'] = 1e6 * (min(ev(160) for _ in range(2)) - min(ev(32) for _ in range(2))) / 128 * P
out['elite partition'] = 1e6 * R.ref_population_sort_seconds(fit, P, n, 5)
g = [R.ref_generation_seconds(xy, n, P, {ELITE}, {MUTANTS}, {RHO}, 1 + i, np.ascontiguousarray(keys), fit) for i in range(2)]
out['generation (crossover, mutants, decode, tour length, partition)'] = 1e6 * min(g)
N = obj.shape[0]; rank = np.zeros(N, np.int32); cd = np.zeros(N, np.float32)
t0 = time.perf_counter(); R.ref_pareto(np.ascontiguousarray(obj), N, rank, cd); t1 = time.perf_counter()
out['Pareto ranks + crowding (4096 points)'] = 1e6 * (t1 - t0)
print(json.dumps(out))
"""
        env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
        r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=900)
    if r.returncode != 0:
        return None
    return json.loads(r.stdout.strip().splitlines()[-1])


def reference_quality(xy, runs, gens, P=256, E=51, M=25):
    """best tour length of `runs` runs of the reference's own Solver on its CPU path
    (oracle/_ref, CUDA hidden); the reference seeds each run from the clock"""
    code = f"""
import json, sys
sys.path[:0] = [{os.path.join(ROOT, 'oracle')!r}]
import numpy as np
import oracle as O
if not O.ref_available():
    print(json.dumps(None)); sys.exit(0)
R = O.ref()
xy = np.array({xy.tolist()!r}, dtype=np.float32)
out = []
for r in range({runs}):
    h = R.ref_solver_create(1, {len(xy)}, xy.ctypes.data, None, None, None, 0.0, {P}, {E}, {M}, 0.7)
    R.ref_solver_evolve(h, {gens})
    out.append(R.ref_solver_best(h))
    R.ref_solver_destroy(h)
print(json.dumps(out))
"""
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=1800)
    if r.returncode != 0:
        return {"error": r.stderr[-500:]}
    return json.loads(r.stdout.strip().splitlines()[-1])


def _stats(v):
    v = np.asarray(v, np.float64)
    return {"mean": float(v.mean()), "std": float(v.std()), "min": float(v.min()), "max": float(v.max())}


def workload_quality(args, headline_scale=True):
    """Best tour over 32 seeds on the n=52 configuration (coordinates uniform in
    [0,1000)^2 from seed 1, population 256, elite 51, mutants 25, rho 0.7, 500
    generations): this engine (the 32 seeds as one batch, spot-checked against the plain
    solver) beside the reference's own solver on its CPU path (32 runs)"""
    import brkga_b200 as B
    xy = np.random.default_rng(1).random((52, 2), dtype=np.float32) * np.float32(1000)
    runs, gens = 32, args.generations
    pb = B.tsp(xy)
    prms = [B.params(256, 51, 25, 0.7, gens, seed=sd) for sd in range(1, runs + 1)]
    t0 = time.perf_counter()
    batch = B.Batch([pb] * runs, prms)
    batch.evolve(gens)
    batch.synchronize()
    secs = time.perf_counter() - t0
    ours = batch.best()[:, 0].astype(np.float64)
    rel = []
    for i in range(runs):
        keys, _ = batch.best_keys(i)
        pts = xy[np.argsort(keys, kind="stable")].astype(np.float64)
        f64 = float(np.sum(np.sqrt(np.sum((pts - np.roll(pts, -1, axis=0)) ** 2, axis=1))))
        rel.append(abs(ours[i] - f64) / f64)
    batch.close()
    same = 0
    for i in range(0, runs, 8):
        s = B.Solver(pb, prms[i])
        s.run()
        same += int(np.float32(s.get_best_individual()[2]) == np.float32(ours[i]))
        s.close()
    out = {"metric": "best tour over 32 seeds, TSP n=52 pop 256, 500 generations", "unit": "tour length",
           "ours": _stats(ours), "ours_seconds_32_runs": secs, "ours_fp32_vs_fp64_max_rel": max(rel),
           "plain_solver_identical": f"{same}/{len(range(0, runs, 8))}", "generations": gens}
    if headline_scale:
        # the headline scale too, on fewer runs (the reference's CPU path takes about 0.09 s
        # per generation there): TSP n=1000, P=2048, E=M=307, 100 generations, 4 runs each
        xy2 = instance()
        pb2 = B.tsp(xy2)
        big = []
        for sd in range(1, 5):
            s = B.Solver(pb2, B.params(POP, ELITE, MUTANTS, RHO, 100, seed=sd))
            s.run()
            big.append(float(s.get_best_individual()[2]))
            s.close()
        out["tsp1000_pop2048"] = {"ours_100_generations": _stats(big)}
    if not args.no_cpu:
        ref = reference_quality(xy, runs, gens)
        if headline_scale:
            ref_big = reference_quality(xy2, 4, 100, P=POP, E=ELITE, M=MUTANTS)
            if isinstance(ref_big, list):
                out["tsp1000_pop2048"]["reference_100_generations"] = _stats(ref_big)
        if isinstance(ref, list):
            out["reference"] = _stats(ref)
            out["mean_ours_minus_reference_rel"] = (out["ours"]["mean"] - out["reference"]["mean"]) / \
                out["reference"]["mean"]
        else:
            out["reference"] = ref
    return out


def movrp_instance(n, seed):
    """depot and n customers uniform in [0,100)^2, demands uniform in {1..30}, the fleet
    max(3, n // 6) (the reference's estimate) and capacity 1.1 x total demand / fleet"""
    rng = np.random.default_rng(seed)
    xy = (rng.random((n + 1, 2)) * 100.0).astype(np.float32)
    dem = rng.integers(1, 31, n + 1).astype(np.int32)
    dem[0] = 0
    V = max(3, n // 6)
    return xy, dem, int(np.ceil(1.1 * dem.sum() / V)), V


def tspj_instance(c, seed):
    """TSPJ data over the depot and c cities: Euclidean travel times of seeded points in
    [0,100)^2, job durations uniform in [1,100) per (city, job type), depot row zero"""
    rng = np.random.default_rng(seed)
    xy = rng.random((c + 1, 2)) * 100.0
    travel = np.sqrt(((xy[:, None, :] - xy[None, :, :]) ** 2).sum(-1)).astype(np.float32)
    jobs = (1.0 + rng.random((c + 1, c + 1)) * 99.0).astype(np.float32)
    jobs[0, :] = 0.0
    return travel, jobs


def run_workload(args):
    import torch
    torch.cuda.init()
    w = args.workload
    if w == "tsp52":
        # n=52 coordinates uniform [0,1000)^2 from seed 1, P 256, elite 0.20, mutants 0.10
        xy = np.random.default_rng(1).random((52, 2), dtype=np.float32) * np.float32(1000)
        import brkga_b200 as B
        out = workload_solver(args, "TSP n=52 pop 256", lambda: B.tsp(xy),
                              dict(population_size=256, elite_size=51, mutant_size=25, elite_prob=0.7,
                                   max_generations=600, seed=1), 500, 1,
                              dict(seed=1, pts=52, n=52, P=256, E=51, M=25, scale=1000.0))
    elif w == "nsga":
        import brkga_b200 as B
        a = np.random.default_rng(3).random((501, 2), dtype=np.float32)
        b = np.random.default_rng(4).random((501, 2), dtype=np.float32)
        out = workload_solver(args, "NSGA-II bi-TSP n=500 pop 2048", lambda: B.bitsp(a, b),
                              dict(population_size=2048, elite_size=0, mutant_size=204, elite_prob=0.7,
                                   max_generations=600, seed=3), args.generations, 5,
                              dict(seed=3, pts=501, n=500, P=2048, E=0, M=0))
    elif w == "tspj":
        import brkga_b200 as B
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        # TSPJConfig::configure_for_multi_gpu on one GPU at 100 cities (configs/tspj_config.hpp:829-849):
        # population 1000, elite 200, mutants 100, rho 0.75; random 2-opt every 2 generations
        # on 100 elites with 5 moves (core/solver.hpp:166)
        travel, jobs = tspj_instance(100, 11)
        out = workload_solver(args, "TSPJ c=100 pop 1000 (local search on)", lambda: B.tspj(travel, jobs),
                              dict(population_size=1000, elite_size=200, mutant_size=100, elite_prob=0.75,
                                   max_generations=100000, seed=11, local_search_interval=2,
                                   local_search_individuals=100, local_search_moves=5), args.generations, 7,
                              dict(seed=11, tspj=True, n=100, P=1000, E=200, M=100))
    elif w == "movrp":
        import brkga_b200 as B
        # MultiObjectiveVRPConfig at 100 customers: configure_for_size gives population 1500
        # and rho 0.10 (configs/multi_objective_vrp_config.hpp:190-211); NSGA-II
        xy, dem, cap, V = movrp_instance(100, 12)
        out = workload_solver(args, "NSGA-II MO-VRP n=100 pop 1500", lambda: B.movrp(xy, dem, cap, V),
                              dict(population_size=1500, elite_size=300, mutant_size=0, elite_prob=0.10,
                                   max_generations=100000, seed=12), args.generations, "movrp",
                              dict(seed=12, movrp=True, n=100, P=1500, cap=cap, V=V))
    elif w == "operators":
        out = workload_operators(args)
    elif w == "batch":
        out = workload_batch(args)
    elif w == "external":
        out = workload_external(args)
    elif w == "serve":
        out = workload_serve(args)
    elif w == "quality":
        out = workload_quality(args)
    else:
        raise SystemExit(f"unknown workload {w}")
    print(json.dumps(out))


def profile_op(args):
    """only the hot-path kernels through their operator entry points (generation step,
    elite partition), for profiler captures: no engine, no autotuning, no timing"""
    import numpy as np
    import torch

    import brkga_b200 as B
    pb = B.tsp(instance())
    ld = (N_CITIES + 3) // 4 * 4
    d_pop = torch.from_numpy(np.random.default_rng(1).random((POP, ld), dtype=np.float32)).cuda()
    d_fit = torch.rand(POP, device="cuda")
    d_srt = torch.zeros(POP, dtype=torch.int32, device="cuda")
    d_next = torch.zeros_like(d_pop)
    d_nfit = torch.zeros_like(d_fit)
    B.sort_fitness(d_fit, POP, 1, False, d_srt)
    for i in range(args.warmup + args.steps):
        B.generation_step(pb, d_pop, d_fit, d_srt, d_next, d_nfit, POP, ELITE, MUTANTS, RHO, ld, SEED_GA, i + 1)
        B.sort_fitness(d_nfit, POP, 1, False, d_srt)
        d_pop, d_next = d_next, d_pop
        d_fit, d_nfit = d_nfit, d_fit
    torch.cuda.synchronize()
    print(json.dumps({"profile_op": True, "steps": args.steps, "best": float(d_fit.min())}))


def profile_kernels(args):
    """small, fixed launches of one kernel family for profiler captures (no timing):
    rows   - the generation step and elite partition at TSP n=1000, P=2048 (as --profile-op)
    big    - rows beyond shared memory: TSP n=65536, 512 rows (134 MB of keys) evaluated
    knap   - greedy knapsack n=10000, 1024 rows evaluated (BASELINE's largest served knapsack)
    nsga   - NSGA-II bi-objective TSP n=500, P=2048 engine: initialisation + generations"""
    import torch

    import brkga_b200 as B
    what = args.profile_kernels
    rng = np.random.default_rng(3)
    if what == "rows":
        return profile_op(args)
    if what in ("big", "knap"):
        if what == "big":
            n, rows = 65536, 512
            pb = B.tsp(rng.random((n, 2), dtype=np.float32))
        else:
            n, rows = 10000, 1024
            w = rng.integers(1, 101, n).astype(np.int32)
            v = rng.integers(1, 101, n).astype(np.int32)
            pb = B.knapsack(w, v, 0.5 * float(w.sum()))
        keys = torch.from_numpy((rng.integers(0, 1 << 24, (rows, n)) / float(1 << 24)).astype(np.float32)).cuda()
        fit = torch.zeros(rows, dtype=torch.float32, device="cuda")
        for _ in range(args.warmup + args.steps):
            pb.evaluate_population(keys, fit, rows, n)
        torch.cuda.synchronize()
        print(json.dumps({"profile_kernels": what, "steps": args.steps, "best": float(fit.min())}))
        return
    if what == "nsga":
        a = np.random.default_rng(3).random((501, 2), dtype=np.float32)
        b = np.random.default_rng(4).random((501, 2), dtype=np.float32)
        s = B.Solver(B.bitsp(a, b), B.params(2048, 0, 204, 0.7, 10000, seed=3))
        s.initialize()
        s.evolve(args.warmup + args.steps)
        s.synchronize()
        print(json.dumps({"profile_kernels": what, "generations": args.warmup + args.steps}))
        s.close()
        return
    raise SystemExit(f"unknown kernel family {what}")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--profile-op", action="store_true", help="operator kernels only (profiler captures)")
    ap.add_argument("--profile-kernels", choices=["rows", "big", "knap", "nsga"],
                    help="small fixed launches of one kernel family (profiler captures)")
    ap.add_argument("--workload", default="tsp1000",
                    choices=["tsp1000", "tsp52", "nsga", "tspj", "movrp", "operators", "batch", "serve", "quality",
                             "external"])
    ap.add_argument("--generations", type=int, default=500)
    ap.add_argument("--instances", type=int, default=256)
    ap.add_argument("--rate", type=float, default=200.0)
    ap.add_argument("--duration", type=float, default=10.0)
    ap.add_argument("--max-active", type=int, default=256)
    ap.add_argument("--tick", type=int, default=25)
    ap.add_argument("--plain-every", type=int, default=20,
                    help="served stream: the plain solver runs every k-th request")
    ap.add_argument("--gens-per-step", type=int, default=GENS_PER_STEP)
    ap.add_argument("--no-extras", action="store_true",
                    help="headline only: skip the nested batched / served / quality measurements")
    args = ap.parse_args()
    if args.profile_op:
        profile_op(args)
        return
    if args.profile_kernels:
        profile_kernels(args)
        return
    if args.workload != "tsp1000":
        run_workload(args)
        return
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if args.warmup < 3 and args.impl == "ours":
        pass  # allowed for quick profiling runs; the default is 5

    if args.impl == "reference":
        if rank != 0:
            return
        cb = cpu_baseline(seconds=max(5.0, min(60.0, 2.0 * args.steps)), max_gens=max(args.steps, 1) * 4)
        line = {"metric": METRIC, "value": cb["value"], "unit": "gens/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": 1e3 / cb["value"], "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded uniform coordinates)",
                "config": workload_config(), "impl": "reference", "cpu_baseline": cb,
                "e2e": {"value": cb["value"], "unit": "gens/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    out = run_ours(args, rank, world)
    if rank == 0:
        if not args.no_cpu:
            out["cpu_baseline"] = cpu_baseline()
        if world == 1 and not args.no_extras:
            # BASELINE's batched-islands and served-stream configurations, and the 32-seed
            # quality check, measured after the headline (outside its timed region)
            out["batched"] = workload_batch(args)
            out["served"] = workload_serve(args)
            out["quality"] = workload_quality(args, headline_scale=False)
        print(json.dumps(out))


if __name__ == "__main__":
    main()
