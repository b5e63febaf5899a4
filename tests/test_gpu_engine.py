"""Whole-run parity on the GPU: the device-resident solver (Solver::run / evolve /
get_best / history, islands with migration, NSGA-II) against the oracle run on the
same seed.  Because every draw is a function of (seed, generation, row, gene) and the
fitness sums follow one fixed order, populations, histories and fronts are bit-exact."""
import numpy as np
import pytest

import instances as I
import oracle as O

pytestmark = pytest.mark.gpu


def B():
    import brkga_b200
    return brkga_b200


def oracle_islands(po, P, E, M, rho, seed, k, interval, migrants, G, ld):
    Pi, Ei, Mi = P // k, E // k, M // k
    pops, fits, srts, hist = [], [], [], []
    for i in range(k):
        pr = O.params(Pi, Ei, Mi, rho, seed, i)
        p, f = O.brkga_init(po, pr, ld)
        pops.append(p)
        fits.append(f)
        srts.append(O.sort_fitness(f, po.maximize))
    best = (max if po.maximize else min)
    hist.append(best(f[s[0]] for f, s in zip(fits, srts)))
    for g in range(1, G + 1):
        for i in range(k):
            pr = O.params(Pi, Ei, Mi, rho, seed, i)
            pops[i], fits[i] = O.brkga_generation(po, pr, g, pops[i], fits[i], srts[i], ld)
            srts[i] = O.sort_fitness(fits[i], po.maximize)
        if k > 1 and interval > 0 and migrants > 0 and g % interval == 0:
            pop = np.ascontiguousarray(np.concatenate(pops))
            fit = np.ascontiguousarray(np.concatenate(fits))
            srt = np.ascontiguousarray(np.concatenate(srts))
            O.migrate(k, Pi, migrants, po.n, ld, po.maximize, pop, fit, srt)
            pops = [pop[i * Pi:(i + 1) * Pi].copy() for i in range(k)]
            fits = [fit[i * Pi:(i + 1) * Pi].copy() for i in range(k)]
            srts = [srt[i * Pi:(i + 1) * Pi].copy() for i in range(k)]
        hist.append(best(f[s[0]] for f, s in zip(fits, srts)))
    ranked_keys = np.concatenate([p[s][:, :po.n] for p, s in zip(pops, srts)])
    ranked_fit = np.concatenate([f[s] for f, s in zip(fits, srts)])
    return ranked_keys, ranked_fit, np.array(hist, np.float32)


@pytest.mark.parametrize("G", [0, 1, 17, 40])
def test_engine_tsp_bit_exact(cuda, G):
    n, P, E, M = 52, 256, 51, 25
    xy = I.tsp_coords(n, seed=1, scale=1000.0)
    pb, po = B().tsp(xy), O.OracleProblem(O.TSP_COORDS, n, xy=xy)
    s = B().Solver(pb, B().params(P, E, M, 0.7, max(G, 1), seed=77))
    s.initialize()
    s.evolve(G)
    keys, fit = s.get_population()
    rk, rf, rh = oracle_islands(po, P, E, M, 0.7, 77, 1, 0, 0, G, 52)
    np.testing.assert_array_equal(keys, rk)
    np.testing.assert_array_equal(fit, rf)
    np.testing.assert_array_equal(s.get_fitness_history(), rh)
    bk, bp, bf = s.get_best_individual()
    np.testing.assert_array_equal(bk, rk[0])
    np.testing.assert_array_equal(bp, O.decode(rk[0])[0])
    assert bf == rf[0]


def test_engine_run_matches_evolve_in_pieces(cuda):
    n = 100
    xy = I.tsp_coords(n, seed=2)
    pb = B().tsp(xy)
    a = B().Solver(pb, B().params(300, 45, 45, 0.7, 50, seed=5))
    a.run()
    b = B().Solver(pb, B().params(300, 45, 45, 0.7, 50, seed=5))
    b.initialize()
    for chunk in (1, 3, 16, 20, 10):
        b.evolve(chunk)
    np.testing.assert_array_equal(a.get_population()[0], b.get_population()[0])
    np.testing.assert_array_equal(a.get_fitness_history(), b.get_fitness_history())


def test_engine_knapsack_greedy(cuda):
    n, P, E, M, G = 400, 128, 19, 19, 12
    w, v, cap = I.knap_items(n, seed=3)
    pb, po = B().knapsack(w, v, cap), O.OracleProblem(O.KNAP_GREEDY, n, w=w, v=v, cap=cap)
    s = B().Solver(pb, B().params(P, E, M, 0.7, G, seed=9))
    s.run()
    keys, fit = s.get_population()
    rk, rf, rh = oracle_islands(po, P, E, M, 0.7, 9, 1, 0, 0, G, 400)
    np.testing.assert_array_equal(keys, rk)
    np.testing.assert_array_equal(fit, rf)
    np.testing.assert_array_equal(s.get_fitness_history(), rh)
    assert np.all(np.diff(rh) >= 0)  # elitism: the best never gets worse (maximise)


@pytest.mark.parametrize("G,interval", [(23, 5), (45, 20)])
def test_engine_islands_migration(cuda, G, interval):
    # (45, 20): runs of 16 generations in one captured graph between migrations
    n, P, E, M, k = 60, 256, 40, 24, 4
    xy = I.tsp_coords(n, seed=4)
    pb, po = B().tsp(xy), O.OracleProblem(O.TSP_COORDS, n, xy=xy)
    prm = B().params(P, E, M, 0.7, G, seed=11, num_islands=k, migration_interval=interval, num_migrants=2)
    s = B().Solver(pb, prm)
    s.run()
    keys, fit = s.get_population()
    rk, rf, rh = oracle_islands(po, P, E, M, 0.7, 11, k, interval, 2, G, 60)
    np.testing.assert_array_equal(keys, rk)
    np.testing.assert_array_equal(fit, rf)
    np.testing.assert_array_equal(s.get_fitness_history(), rh)


def test_engine_set_population_and_continue(cuda):
    n, P, E, M = 30, 64, 10, 6
    xy = I.tsp_coords(n, seed=8)
    pb, po = B().tsp(xy), O.OracleProblem(O.TSP_COORDS, n, xy=xy)
    s = B().Solver(pb, B().params(P, E, M, 0.7, 10, seed=3))
    keys = I.keys(P, n, seed=4)
    s.set_population(keys)
    got_keys, got_fit = s.get_population()
    srt = O.sort_fitness(O.evaluate(po, keys))
    np.testing.assert_array_equal(got_keys, keys[srt])
    s.evolve(3)
    pr = O.params(P, E, M, 0.7, 3)
    pop, fit = keys.copy(), O.evaluate(po, keys)
    ld = 32
    popl = np.zeros((P, ld), np.float32)
    popl[:, :n] = pop
    for g in range(1, 4):
        popl, fit = O.brkga_generation(po, pr, g, popl, fit, srt, ld)
        srt = O.sort_fitness(fit)
    np.testing.assert_array_equal(s.get_population()[0], popl[srt][:, :n])


def test_engine_nsga2_bit_exact(cuda):
    n, P, G = 30, 64, 30
    a, b = I.tsp_coords(n + 1, seed=5), I.tsp_coords(n + 1, seed=6)
    pb, po = B().bitsp(a, b), O.OracleProblem(O.BITSP_COORDS, n, xy=a, xy2=b)
    s = B().Solver(pb, B().params(P, 0, 6, 0.7, G, seed=21, diversity_interval=25))
    s.initialize()
    ld = 32
    pr = O.nsga2_params(P, 6, 0.7, 5.0 / n, 21, 25)
    pop, obj, rank, cd = O.nsga2_init(po, pr, ld)
    for g in range(1, G + 1):
        s.evolve(1)
        O.nsga2_generation(po, pr, g, ld, pop, obj, rank, cd)
        gk, go = s.get_population()
        np.testing.assert_array_equal(gk, pop[:, :n], err_msg=f"generation {g}")
        np.testing.assert_array_equal(go, obj, err_msg=f"generation {g}")
    fobj, fkeys = s.get_pareto_front()
    np.testing.assert_array_equal(fobj, obj[rank == 0])


def test_engine_nsga2_diversity_rebuild(cuda):
    # a tiny instance converges to duplicates quickly, so the diversity pass rebuilds
    n, P, G = 4, 40, 60
    a, b = I.tsp_coords(n + 1, seed=15), I.tsp_coords(n + 1, seed=16)
    pb, po = B().bitsp(a, b), O.OracleProblem(O.BITSP_COORDS, n, xy=a, xy2=b)
    s = B().Solver(pb, B().params(P, 0, 0, 0.7, G, seed=3, diversity_interval=5))
    s.initialize()
    ld = 4
    pr = O.nsga2_params(P, 0, 0.7, 5.0 / n, 3, 5)
    pop, obj, rank, cd = O.nsga2_init(po, pr, ld)
    rebuilt = 0
    for g in range(1, G + 1):
        before = pop.copy()
        s.evolve(1)
        O.nsga2_generation(po, pr, g, ld, pop, obj, rank, cd)
        gk, go = s.get_population()
        np.testing.assert_array_equal(gk, pop[:, :n], err_msg=f"generation {g}")
        rebuilt += int(not np.array_equal(before, pop))
    assert rebuilt > 0


@pytest.mark.parametrize("strides", [(1, 7, 3, 13, 20, 16), (60,)])
def test_engine_nsga2_diversity_strides(cuda, strides):
    # evolve() splits a call into captured runs of 16/8/4/2/1 plain generations and one
    # generation with the diversity pass whenever (g - 1) % interval == 0; uneven calls
    # must give the same populations as single generations
    n, P = 4, 40
    a, b = I.tsp_coords(n + 1, seed=15), I.tsp_coords(n + 1, seed=16)
    pb, po = B().bitsp(a, b), O.OracleProblem(O.BITSP_COORDS, n, xy=a, xy2=b)
    s = B().Solver(pb, B().params(P, 0, 0, 0.7, sum(strides), seed=3, diversity_interval=5))
    s.initialize()
    ld = 4
    pr = O.nsga2_params(P, 0, 0.7, 5.0 / n, 3, 5)
    pop, obj, rank, cd = O.nsga2_init(po, pr, ld)
    g = 0
    for k in strides:
        s.evolve(k)
        for _ in range(k):
            g += 1
            O.nsga2_generation(po, pr, g, ld, pop, obj, rank, cd)
        gk, go = s.get_population()
        np.testing.assert_array_equal(gk, pop[:, :n], err_msg=f"generation {g}")
        np.testing.assert_array_equal(go, obj, err_msg=f"generation {g}")
    assert s.generation == g


def test_invalid_params_rejected(cuda):
    xy = I.tsp_coords(10, seed=1)
    pb = B().tsp(xy)
    for bad in (B().params(0, 0, 0), B().params(10, 0, 2), B().params(10, 8, 4), B().params(10, 2, 2, elite_prob=1.5),
                B().params(10, 2, 2, max_generations=0)):
        with pytest.raises(B().BrkgaError) as ei:
            B().Solver(pb, bad)
        assert ei.value.code == -1


def test_cpp_dropin_program(cuda, tmp_path):
    """the reference-style C++ program (TSPLIB file -> TSPConfig::load_from_file -> Solver)
    gives the same best tour as the Python binding on the same coordinates and seed"""
    import json
    import os
    import subprocess
    exe = os.path.join(os.path.dirname(B().LIB_PATH), "..", "build", "solve_tsp")
    path = str(tmp_path / "inst.tsp")
    r = subprocess.run([exe, path, "52", "1", "256", "51", "25", "60"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    out = json.loads(r.stdout.strip().splitlines()[-1])
    assert sorted(out["tour"]) == list(range(52)) and out["history"] == 61
    xy = []
    for line in open(path):
        parts = line.split()
        if len(parts) == 3 and parts[0].isdigit():
            xy.append((float(parts[1]), float(parts[2])))
    s = B().Solver(B().tsp(np.array(xy, np.float32)), B().params(256, 51, 25, 0.7, 60, seed=7))
    s.run()
    _, perm, fit = s.get_best_individual()
    assert np.float32(out["best"]) == fit
    assert out["tour"] == perm.tolist()


def test_cpp_knapsack_files(cuda, tmp_path):
    """KnapsackConfig::load_from_file reads the reference's text and CSV layouts to the same
    instance, and the drop-in solve equals the Python binding's"""
    import json
    import os
    import subprocess
    exe = os.path.join(os.path.dirname(B().LIB_PATH), "..", "build", "solve_knapsack")
    r = subprocess.run([exe, str(tmp_path), "60", "4", "50"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    out = json.loads(r.stdout.strip().splitlines()[-1])
    rows = [l.split() for l in open(tmp_path / "items.txt") if l.strip() and not l.startswith("#")]
    n, cap = int(rows[0][0]), float(rows[0][1])
    w = np.array([int(a) for a, _ in rows[1:]], np.int32)
    v = np.array([int(b) for _, b in rows[1:]], np.int32)
    assert len(w) == n and cap == out["capacity"]
    s = B().Solver(B().knapsack(w, v, cap, greedy=False), B().params(400, 80, 40, 0.7, 50, seed=5))
    s.run()
    best = s.get_best_individual()[2]
    assert np.float32(out["txt"]) == best and np.float32(out["csv"]) == best
    s.close()


def test_engines_on_host_threads(cuda):
    """solvers driven from several host threads at once (the reference's callers use
    OpenMP / std::async) give the runs they give one at a time; one problem is shared"""
    from concurrent.futures import ThreadPoolExecutor
    xy = I.tsp_coords(80, seed=21)
    pb = B().tsp(xy)

    def run(seed):
        s = B().Solver(pb, B().params(128, 20, 12, 0.7, 30, seed=seed))
        s.run()
        keys, fit = s.get_population()
        hist = s.get_fitness_history()
        s.close()
        return keys, fit, hist

    alone = [run(sd) for sd in range(6)]
    with ThreadPoolExecutor(6) as ex:
        together = list(ex.map(run, range(6)))
    for a, b in zip(alone, together):
        for x, y in zip(a, b):
            np.testing.assert_array_equal(x, y)
    pb.close()
