"""External fitness (BRKGA_EXTERNAL): a config that brings its own fitness -- a host
fitness_function or its own evaluate_population_gpu, as the reference's LLM-written
configs do (core/config.hpp:33-53) -- runs on the engine with the keys, crossover,
mutants and elite partition on the device.  Fed the same fitness as a built-in problem,
an external engine must evolve exactly like the built-in engine on the same seed."""
import json
import os
import subprocess

import numpy as np
import pytest

import instances as I
import oracle as O

pytestmark = pytest.mark.gpu


def B():
    import brkga_b200
    return brkga_b200


class _Cai:
    """a device buffer as a torch tensor (__cuda_array_interface__)"""

    def __init__(self, ptr, shape):
        self.__cuda_array_interface__ = {"shape": shape, "typestr": "<f4", "data": (ptr, False), "version": 3}


def _builtin_run(xy, prm, G):
    s = B().Solver(B().tsp(xy), prm)
    s.initialize()
    s.evolve(G)
    keys, fit = s.get_population()
    return keys, fit, s.get_fitness_history()


@pytest.mark.parametrize("n,P,E,M,G", [(60, 128, 26, 13, 12), (53, 96, 19, 10, 9)])
def test_external_host_fitness_equals_builtin(cuda, n, P, E, M, G):
    # the tour length computed on the host by the oracle, fed through the external path
    xy = I.tsp_coords(n, seed=n)
    po = O.OracleProblem(O.TSP_COORDS, n, xy=xy)
    prm = B().params(P, E, M, 0.7, G, seed=5)
    keys_b, fit_b, hist_b = _builtin_run(xy, prm, G)
    s = B().Solver(B().external(n), prm)
    for _ in range(G + 1):  # the initial population, then G generations
        s.external_step(lambda rows: O.evaluate(po, rows))
    keys_e, fit_e = s.get_population()
    np.testing.assert_array_equal(keys_e, keys_b)
    np.testing.assert_array_equal(fit_e, fit_b)
    np.testing.assert_array_equal(s.get_fitness_history(), hist_b)
    assert s.generation == G
    k, perm, f = s.get_best_individual()
    assert perm is None and f == fit_b[0]
    np.testing.assert_array_equal(k, keys_b[0])


@pytest.mark.parametrize("n", [61, 64])
def test_external_device_fitness_dense_rows(cuda, n):
    # a caller's own device evaluation: dense [P][n] rows in, fitness written in HBM
    import torch
    xy = I.tsp_coords(n, seed=3)
    po = O.OracleProblem(O.TSP_COORDS, n, xy=xy)
    P, E, M, G = 64, 13, 6, 6
    prm = B().params(P, E, M, 0.7, G, seed=9)
    keys_b, fit_b, _ = _builtin_run(xy, prm, G)
    s = B().Solver(B().external(n), prm)
    for g in range(G + 1):
        kp, fp, ld, first, cnt = s.external_begin(dense=True)
        assert ld == n and (first, cnt) == ((0, P) if g == 0 else (E, P - E))
        rows = torch.as_tensor(_Cai(kp, (cnt, n)), device="cuda")
        np.testing.assert_array_equal(rows.cpu().numpy(), s.external_rows())
        fit = torch.as_tensor(_Cai(fp, (cnt,)), device="cuda")
        fit[:] = torch.from_numpy(O.evaluate(po, rows.cpu().numpy())).cuda()
        torch.cuda.synchronize()
        assert s.external_commit()
    keys_e, fit_e = s.get_population()
    np.testing.assert_array_equal(keys_e, keys_b)
    np.testing.assert_array_equal(fit_e, fit_b)


def test_external_maximize(cuda):
    # maximise the tour length: the partition orders fitness descending, the best-fitness
    # history never falls (elitism)
    n, P, E, M, G = 40, 64, 13, 6, 15
    xy = I.tsp_coords(n, seed=2)
    po = O.OracleProblem(O.TSP_COORDS, n, xy=xy)
    s = B().Solver(B().external(n, maximize=True), B().params(P, E, M, 0.7, G, seed=4))
    for _ in range(G + 1):
        s.external_step(lambda rows: O.evaluate(po, rows))
    _, fit = s.get_population()
    assert np.all(np.diff(fit) <= 0)
    h = s.get_fitness_history()
    assert len(h) == G + 1 and np.all(np.diff(h) >= 0) and h[-1] == fit[0]


def test_external_rejections(cuda):
    pb = B().external(20)
    s = B().Solver(pb, B().params(32, 6, 3, 0.7, 5, seed=1))
    for call in (lambda: s.evolve(1), lambda: s.run(), lambda: s.set_population(np.zeros((32, 20), np.float32))):
        with pytest.raises(B().BrkgaError) as ei:
            call()
        assert ei.value.code == -6
    with pytest.raises(B().BrkgaError):  # nothing ranked yet
        s.get_best_individual()
    assert s.external_begin()[3:] == (0, 32)
    with pytest.raises(B().BrkgaError) as ei:  # rows already pending
        s.external_begin()
    assert ei.value.code == -1
    with pytest.raises(ValueError):
        s.external_set_fitness(np.zeros(3, np.float32))
    s.external_set_fitness(np.arange(32, dtype=np.float32))
    s.external_commit()
    with pytest.raises(B().BrkgaError) as ei:  # nothing pending
        s.external_commit()
    assert ei.value.code == -1
    assert s.get_best_individual()[2] == 0.0
    # islands, batches and the device evaluation entry points refuse it
    with pytest.raises(B().BrkgaError) as ei:
        B().Solver(pb, B().params(32, 6, 3, 0.7, 5, seed=1, num_islands=2))
    assert ei.value.code == -6
    with pytest.raises(B().BrkgaError) as ei:
        B().Batch([pb], [B().params(32, 6, 3, 0.7, 5, seed=1)])
    assert ei.value.code == -6
    import torch
    pop = torch.zeros((4, 20), device="cuda")
    fit = torch.zeros(4, device="cuda")
    with pytest.raises(B().BrkgaError) as ei:
        pb.evaluate_population(pop, fit, 4)
    assert ei.value.code == -6
    # initialize restarts: the next begin builds a new initial population
    s.initialize()
    assert s.external_begin()[3:] == (0, 32)
    s.external_set_fitness(np.ones(32, np.float32))
    s.external_commit()
    assert s.generation == 0


def _builtin_nsga(a, b, prm, G, per_generation=None):
    s = B().Solver(B().bitsp(a, b), prm)
    s.initialize()
    out = []
    for _ in range(G):
        s.evolve(1)
        if per_generation:
            out.append(s.get_population())
    return s, out


@pytest.mark.parametrize("n,P,G,div", [(30, 64, 30, 25), (4, 40, 40, 5)])
def test_external_nsga2_equals_builtin(cuda, n, P, G, div):
    # two objectives from the host (the oracle's depot tours), NSGA-II on the device; the
    # tiny instance converges to duplicates, so the diversity pass rebuilds the population
    # and the commit asks for the refill rows' objectives
    a, b = I.tsp_coords(n + 1, seed=n), I.tsp_coords(n + 1, seed=n + 1)
    po = O.OracleProblem(O.BITSP_COORDS, n, xy=a, xy2=b)
    prm = B().params(P, 0, 0, 0.7, G, seed=21, diversity_interval=div)
    sb, per_gen = _builtin_nsga(a, b, prm, G, per_generation=True)
    s = B().Solver(B().external(n, num_objectives=2), prm)
    refills = 0

    def objectives(rows):
        return O.evaluate(po, rows)

    s.external_step(objectives)
    for g in range(G):
        while True:
            _, _, _, first, cnt = s.external_begin()
            assert cnt == (P if first == P else P - first)
            s.external_set_fitness(objectives(s.external_rows()))
            if s.external_commit():
                break
            refills += 1
        keys_e, obj_e = s.get_population()
        np.testing.assert_array_equal(keys_e, per_gen[g][0], err_msg=f"generation {g + 1}")
        np.testing.assert_array_equal(obj_e, per_gen[g][1], err_msg=f"generation {g + 1}")
    if n == 4:
        assert refills > 0
    fo_e, fk_e = s.get_pareto_front()
    fo_b, fk_b = sb.get_pareto_front()
    np.testing.assert_array_equal(fo_e, fo_b)
    np.testing.assert_array_equal(fk_e, fk_b)
    np.testing.assert_array_equal(s.get_fitness_history(), sb.get_fitness_history())


def test_external_cpp_program(cuda):
    """the LLM-style config (host fitness_function, or its own CUDA kernel) with the
    generated main's flow: both evaluations evolve identically, and the best individual's
    fitness equals the config's own fitness of its keys"""
    exe = os.path.join(os.path.dirname(B().LIB_PATH), "..", "build", "solve_external")
    outs = {}
    for mode in ("host", "gpu"):
        r = subprocess.run([exe, mode, "41", "3", "60"], capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr
        assert "Best fitness:" in r.stdout and "Weighted completion time:" in r.stdout
        outs[mode] = json.loads(r.stdout.strip().splitlines()[-1])
        outs[mode].pop("seconds")
    assert outs["host"] == outs["gpu"]
    d = outs["host"]
    assert d["best"] == d["check"] and d["history"] == 61 and d["last"] <= d["first"]
    r = subprocess.run([exe, "host", "41", "3", "60"], capture_output=True, text=True, timeout=300,
                       env=dict(os.environ, QUICK_TEST="10"))
    assert r.returncode == 0 and json.loads(r.stdout.strip().splitlines()[-1])["history"] == 11


def test_external_cpp_program_two_objectives(cuda):
    """the same config with a second weight vector (objective_functions, NSGA-II): the host
    objectives and the config's own two-objective kernel give the same Pareto front, and
    no point of it dominates another"""
    exe = os.path.join(os.path.dirname(B().LIB_PATH), "..", "build", "solve_external")
    outs = {}
    for mode in ("host2", "gpu2"):
        r = subprocess.run([exe, mode, "37", "5", "40"], capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr
        assert "Pareto front size:" in r.stdout
        outs[mode] = json.loads(r.stdout.strip().splitlines()[-1])
        outs[mode].pop("seconds")
    assert outs["host2"] == outs["gpu2"]
    pts = np.array(outs["host2"]["points"])
    assert outs["host2"]["front"] == len(pts) > 0
    for i in range(len(pts)):
        dom = np.all(pts <= pts[i], axis=1) & np.any(pts < pts[i], axis=1)
        assert not dom.any()
