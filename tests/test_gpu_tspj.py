"""TSPJ on the GPU (TSPJConfig, configs/tspj_config.hpp): two argsorts per chromosome (city
keys, job keys) and the makespan summed in the reference's own sequential order, so
decodes and fitness values equal the oracle's -- and through it the reference's own
fitness function -- bit for bit, on the shared-memory and the global-memory row kernels."""
import numpy as np
import pytest

import instances as I
import oracle as O
from test_gpu_engine import oracle_islands
from test_gpu_ops import B, eval_gpu, run_gen

pytestmark = pytest.mark.gpu


def problems(c, seed):
    travel, jobs = I.tspj_instance(c, seed)
    return B().tspj(travel, jobs), O.OracleProblem(O.TSPJ, 2 * c, mat=travel, mat2=jobs)


@pytest.mark.parametrize("c", [1, 2, 5, 52, 300, 1000, 3000, 8000])
def test_tspj_decode_makespan(cuda, c):
    # c = 8000 (16000 genes) takes the global-memory row kernel
    pb, po = problems(c, seed=c)
    keys = I.keys(6, 2 * c, seed=c + 1)
    keys[1] = I.tied_keys(1, 2 * c, seed=c + 2)[0]  # ties go to the lower index in each half
    fit, perm = eval_gpu(pb, keys, cuda)
    np.testing.assert_array_equal(perm, O.decode_problem(po, keys))
    np.testing.assert_array_equal(fit.view(np.uint32), O.evaluate(po, keys).view(np.uint32))


def test_tspj_generation_step(cuda):
    c = 52
    pb, po = problems(c, seed=3)
    run_gen(cuda, pb, po, 128, 25, 12, 0.75, 5, 3)


def test_tspj_engine_bit_exact(cuda):
    c, P, E, M, G = 40, 200, 40, 20, 15
    pb, po = problems(c, seed=4)
    s = B().Solver(pb, B().params(P, E, M, 0.75, G, seed=8))
    s.run()
    keys, fit = s.get_population()
    rk, rf, rh = oracle_islands(po, P, E, M, 0.75, 8, 1, 0, 0, G, (2 * c + 3) // 4 * 4)
    np.testing.assert_array_equal(keys, rk)
    np.testing.assert_array_equal(fit, rf)
    np.testing.assert_array_equal(s.get_fitness_history(), rh)
    _, perm, best = s.get_best_individual()
    np.testing.assert_array_equal(perm, O.decode_problem(po, rk[0])[0])
    assert best == rf[0]
    s.close()


def test_tspj_batch_equals_standalone(cuda):
    b = B()
    probs, prms = [], []
    for i, c in enumerate([10, 60, 250]):
        travel, jobs = I.tspj_instance(c, seed=60 + i)
        probs.append(b.tspj(travel, jobs))
        prms.append(b.params(96, 19, 9, 0.75, 30, seed=70 + i))
    batch = b.Batch(probs, prms)
    batch.evolve(30)
    best = batch.best()
    for i in range(3):
        s = b.Solver(probs[i], prms[i])
        s.run()
        assert best[i, 0] == s.get_best_individual()[2]
        s.close()
    batch.close()
