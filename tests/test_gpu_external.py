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
    for _ in range(G + 1):
        kp, fp, ld, first = s.external_begin(dense=True)
        assert ld == n
        rows = torch.as_tensor(_Cai(kp, (P, n)), device="cuda")
        host_rows = s.external_rows()
        np.testing.assert_array_equal(rows[first:].cpu().numpy(), host_rows)
        fit = torch.as_tensor(_Cai(fp, (P,)), device="cuda")
        fit[first:] = torch.from_numpy(O.evaluate(po, rows[first:].cpu().numpy())).cuda()
        torch.cuda.synchronize()
        s.external_commit()
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
    s.external_begin()
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
    _, _, _, first = s.external_begin()
    assert first == 0
    s.external_set_fitness(np.ones(32, np.float32))
    s.external_commit()
    assert s.generation == 0


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
    assert outs["host"] == outs["gpu"]
    d = outs["host"]
    assert d["best"] == d["check"] and d["history"] == 61 and d["last"] <= d["first"]
    r = subprocess.run([exe, "host", "41", "3", "60"], capture_output=True, text=True, timeout=300,
                       env=dict(os.environ, QUICK_TEST="10"))
    assert r.returncode == 0 and json.loads(r.stdout.strip().splitlines()[-1])["history"] == 11
