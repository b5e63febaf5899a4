"""Benchmark of the per-generation BRKGA hot path on B200.

Workload (the headline configuration): Euclidean TSP, n = 1000 cities with FP32
coordinates uniform in [0,1)^2 (seeded), population 2048, elite 307 (0.15), mutants 307
(0.15), rho = 0.7; one step = one generation (fused crossover / mutant fill / decode /
tour length kernel + elite-partition sort) of the device-resident solver.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs N independent replicas (one instance per GPU, no collective: islands and
instances are independent units), launched one process per GPU by torch.distributed.run.
The JSON line's `value` is whole-job generations per second with the population resident
in HBM; `e2e` is the same metric through the C ABI from host buffers: each e2e step is one
whole 1000-generation solve (problem upload from pinned memory, create, initialise,
evolve, read the best tour back).  L2 is flushed (a 256 MiB write) before every timed
generation, outside its CUDA-event bracket.
"""
from __future__ import annotations

import argparse
import json
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
SEED_INSTANCE, SEED_GA = 2026, 7
PROFILE = os.path.join(ROOT, "profiles", "row_kernel_tsp_n1000_p2048.md")
HOLD_CYCLES_PER_STEP = 400_000  # ~0.2 ms of device spin per queued step (host enqueue cost)


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


def profile_traffic():
    """DRAM bytes per launch of the row kernel from the committed ncu summary, or None"""
    try:
        txt = open(PROFILE).read()
    except OSError:
        return None
    m = re.search(r"traffic_bytes_per_launch:\s*([0-9.eE+]+)", txt)
    return float(m.group(1)) if m else None


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

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    xy = instance()
    pb = B.tsp(xy, device=dev)
    prm = B.params(POP, ELITE, MUTANTS, RHO, E2E_GENERATIONS, seed=SEED_GA + rank, device=dev)
    s = B.Solver(pb, prm)
    s_info = s.info
    s.initialize()
    stream = torch.cuda.ExternalStream(s.stream, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    for _ in range(args.warmup):
        with torch.cuda.stream(stream):
            flush.fill_(1.0)
        s.evolve(1)
    s.synchronize()

    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    barrier()
    with ClockSampler(dev) as clocks:
        # hold the stream while the host queues every timed step, so no host gap lands
        # inside an event bracket (the hold itself is outside every bracket)
        with torch.cuda.stream(stream):
            torch.cuda._sleep(HOLD_CYCLES_PER_STEP * args.steps)
        for i in range(args.steps):
            with torch.cuda.stream(stream):
                flush.fill_(float(i))
                starts[i].record(stream)
            s.evolve(1)
            with torch.cuda.stream(stream):
                ends[i].record(stream)
        s.synchronize()
        barrier()
    ms = sum(a.elapsed_time(b) for a, b in zip(starts, ends))
    if dist is not None:
        t = torch.tensor([ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    value = world * args.steps / (ms / 1e3)
    best = float(s.get_best_individual()[2])

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

    # --- for information: back-to-back generations with L2 left warm (one evolve call)
    warm_gens = 200
    s.synchronize()
    w0, w1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        torch.cuda._sleep(HOLD_CYCLES_PER_STEP)
        w0.record(stream)
    s.evolve(warm_gens)
    with torch.cuda.stream(stream):
        w1.record(stream)
    s.synchronize()
    warm_gens_per_s = warm_gens / (w0.elapsed_time(w1) / 1e3)

    # --- end to end through the C ABI from host buffers: one whole solve per step
    e2e = None
    if not args.no_e2e:
        pinned = torch.from_numpy(xy).pin_memory()
        xy_host = pinned.numpy()
        keys = np.zeros(N_CITIES, np.float32)
        perm = np.zeros(N_CITIES, np.int32)
        e2e_steps = max(1, min(args.steps, 5))
        times = []
        for i in range(1 + e2e_steps):
            barrier()
            t0 = time.perf_counter()
            pe = B.tsp(xy_host, device=dev)
            se = B.Solver(pe, B.params(POP, ELITE, MUTANTS, RHO, E2E_GENERATIONS, seed=100 + i, device=dev))
            se.run()
            k2, p2, f2 = se.get_best_individual()
            se.close()
            pe.close()
            barrier()
            if i > 0:
                times.append(time.perf_counter() - t0)
        tt = sum(times)
        if dist is not None:
            t = torch.tensor([tt], device=dev, dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            tt = float(t.item())
        e2e = {"value": world * e2e_steps * E2E_GENERATIONS / tt, "unit": "gens/s",
               "h2d_bytes_per_step": int(xy.nbytes), "d2h_bytes_per_step": int(keys.nbytes + perm.nbytes + 4),
               "step": f"one {E2E_GENERATIONS}-generation solve through brkga_problem_create / brkga_create / "
                       f"brkga_run / brkga_get_best", "ms_per_solve": 1e3 * tt / e2e_steps}

    peak, peak_kind = measured_peak()
    alg = algorithmic_bytes_per_generation()
    achieved = alg / (row_ms / 1e3) / 1e9
    out = None
    if rank == 0:
        out = {
            "metric": METRIC, "value": value, "unit": "gens/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded uniform coordinates)",
            "config": {"workload": f"TSP n={N_CITIES} pop={POP} elite={ELITE} mutants={MUTANTS} rho={RHO}",
                       "n": N_CITIES, "population": POP, "elite": ELITE, "mutants": MUTANTS, "rho": RHO,
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                       "l2": "flushed (256 MiB write) before every timed generation, outside the timing"},
            "impl": "ours",
            "e2e": e2e,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": profile_traffic(),
                         "kernel": "bk::row_kernel<256,1> (fused crossover/mutant/decode/tour length), "
                                   "timed through brkga_generation_step",
                         "engine_tile": {"threads": s_info[0], "groups": s_info[1], "grid": s_info[2],
                                         "coords_in_smem": bool(s_info[3])},
                         "algorithmic_bytes_per_launch": alg, "kernel_ms": row_ms, "peak_kind": peak_kind,
                         "sort_kernel_ms": sort_ms},
            "gpu_launches": 2 * args.steps,
            "clocks": clocks.summary(),
            "best_tour": best,
            "l2_warm_back_to_back_gens_per_s": warm_gens_per_s,
        }
    s.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return out


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


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--profile-op", action="store_true", help="operator kernels only (profiler captures)")
    args = ap.parse_args()
    if args.profile_op:
        profile_op(args)
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
                "config": {"workload": f"TSP n={N_CITIES} pop={POP} elite={ELITE} mutants={MUTANTS} rho={RHO}",
                           "n": N_CITIES, "population": POP, "elite": ELITE, "mutants": MUTANTS, "rho": RHO},
                "impl": "reference", "cpu_baseline": cb,
                "e2e": {"value": cb["value"], "unit": "gens/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    out = run_ours(args, rank, world)
    if rank == 0:
        if not args.no_cpu:
            out["cpu_baseline"] = cpu_baseline()
        print(json.dumps(out))


if __name__ == "__main__":
    main()
