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


def test_local_search_op(cuda):
    """brkga_local_search on rows in rank order, against the oracle: same rows changed, same
    keys and makespans"""
    import torch
    c, P, moves = 60, 48, 5
    pb, po = problems(c, seed=30)
    ld = (2 * c + 3) // 4 * 4
    keys = np.zeros((P, ld), np.float32)
    keys[:, :2 * c] = I.keys(P, 2 * c, seed=31)
    fit = O.evaluate(po, keys, ld)
    d_pop = torch.from_numpy(keys.copy()).to(cuda)
    d_fit = torch.from_numpy(fit.copy()).to(cuda)
    B().local_search(pb, d_pop, d_fit, P, moves, 99, 7, ld=ld, island=1)
    ref_pop, ref_fit = keys.copy(), fit.copy()
    O.local_search(po, ref_pop, ref_fit, np.arange(P), P, ld, moves, 99, 7, 1)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(d_pop.cpu().numpy(), ref_pop)
    np.testing.assert_array_equal(d_fit.cpu().numpy(), ref_fit)
    improved = int(np.sum(ref_fit < fit))
    assert 0 < improved < P, improved  # the check sees both outcomes


def oracle_run_ls(po, P, E, M, rho, seed, k, G, ld, interval, count, moves, mig_interval=0, migrants=0):
    """oracle generations with the local search pass after generation g when g - 1 > 0 and
    (g - 1) % interval == 0 (then re-rank), before migration"""
    Pi, Ei, Mi = P // k, E // k, M // k
    prs = [O.params(Pi, Ei, Mi, rho, seed, i) for i in range(k)]
    pops, fits, srts = [], [], []
    for i in range(k):
        p, f = O.brkga_init(po, prs[i], ld)
        pops.append(p)
        fits.append(f)
        srts.append(O.sort_fitness(f))
    hist = [min(f[s[0]] for f, s in zip(fits, srts))]
    cnt = min(count, Ei)
    for g in range(1, G + 1):
        for i in range(k):
            pops[i], fits[i] = O.brkga_generation(po, prs[i], g, pops[i], fits[i], srts[i], ld)
            srts[i] = O.sort_fitness(fits[i])
            if g - 1 > 0 and (g - 1) % interval == 0:
                O.local_search(po, pops[i], fits[i], srts[i], cnt, ld, moves, seed, g, i)
                srts[i] = O.sort_fitness(fits[i])
        if k > 1 and mig_interval > 0 and g % mig_interval == 0:
            pop = np.ascontiguousarray(np.concatenate(pops))
            fit = np.ascontiguousarray(np.concatenate(fits))
            srt = np.ascontiguousarray(np.concatenate(srts))
            O.migrate(k, Pi, migrants, po.n, ld, False, pop, fit, srt)
            pops = [pop[i * Pi:(i + 1) * Pi].copy() for i in range(k)]
            fits = [fit[i * Pi:(i + 1) * Pi].copy() for i in range(k)]
            srts = [srt[i * Pi:(i + 1) * Pi].copy() for i in range(k)]
        hist.append(min(f[s[0]] for f, s in zip(fits, srts)))
    keys = np.concatenate([p[s][:, :po.n] for p, s in zip(pops, srts)])
    fit = np.concatenate([f[s] for f, s in zip(fits, srts)])
    return keys, fit, np.array(hist, np.float32)


@pytest.mark.parametrize("k,G,mig", [(1, 12, 0), (2, 12, 5), (1, 36, 0), (2, 36, 20)])
def test_engine_local_search_bit_exact(cuda, k, G, mig):
    # G = 36: runs of 16 generations in one captured graph, local search inside them
    c, P, E, M = 30, 160, 40, 16
    pb, po = problems(c, seed=40 + k)
    prm = B().params(P, E, M, 0.75, G, seed=5, num_islands=k, migration_interval=mig,
                     num_migrants=2 if mig else 0, local_search_interval=2, local_search_individuals=100,
                     local_search_moves=5)
    s = B().Solver(pb, prm)
    s.run()
    keys, fit = s.get_population()
    rk, rf, rh = oracle_run_ls(po, P, E, M, 0.75, 5, k, G, (2 * c + 3) // 4 * 4, 2, 100, 5, mig, 2)
    np.testing.assert_array_equal(keys, rk)
    np.testing.assert_array_equal(fit, rf)
    np.testing.assert_array_equal(s.get_fitness_history(), rh)
    s.close()


def test_local_search_rejected_in_batches(cuda):
    pb, _ = problems(10, seed=50)
    with pytest.raises(B().BrkgaError) as ei:
        B().Batch([pb], [B().params(32, 6, 3, 0.75, 5, seed=1, local_search_interval=2)])
    assert ei.value.code == -6


def test_cpp_tspj_dropin_program(cuda, tmp_path):
    """the reference-style C++ program (_TT/_JT CSV files -> TSPJConfig::load_from_file ->
    Solver with local search) gives the same best makespan and decode as the Python binding
    on the same matrices and seed"""
    import json
    import os
    import subprocess
    exe = os.path.join(os.path.dirname(B().LIB_PATH), "..", "build", "solve_tspj")
    r = subprocess.run([exe, str(tmp_path), "20", "3", "128", "25", "12", "40"], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr
    out = json.loads(r.stdout.strip().splitlines()[-1])
    travel = np.loadtxt(tmp_path / "synthetic_TT.csv", delimiter=",", dtype=np.float32)
    jobs = np.loadtxt(tmp_path / "synthetic_JT.csv", delimiter=",", dtype=np.float32)
    assert travel.shape == (21, 21) and out["history"] == 41
    s = B().Solver(B().tspj(travel, jobs), B().params(128, 25, 12, 0.7, 40, seed=7, local_search_interval=2))
    s.run()
    _, perm, best = s.get_best_individual()
    assert np.float32(out["best"]) == best
    assert out["perm"] == perm.tolist()
    s.close()
