"""The reference's other GPU problem configs on the engine: job scheduling
(JobSchedulingGPUConfig) and continuous functions (ContinuousOptGPUConfig).  Their
fitness values are sequential float sums in the reference; the GPU adds in the same
order, so job scheduling, sphere and Rosenbrock equal the oracle (pinned bit for bit to
the reference) exactly.  Rastrigin calls cos: the device cosf is not the host's, so it is
held to 1e-5 relative against the FP64 value (and to the oracle's float value)."""
import numpy as np
import pytest

import instances as I
import oracle as O
from test_gpu_engine import oracle_islands
from test_gpu_ops import B, eval_gpu

pytestmark = pytest.mark.gpu

BOUNDS = {0: (-5.12, 5.12), 1: (-5.12, 5.12), 2: (-5.0, 10.0)}


def job_times(n, seed):
    return (1.0 + np.random.default_rng(seed).random(n) * 99.0).astype(np.float32)


@pytest.mark.parametrize("n,M", [(1, 1), (50, 5), (1000, 32), (1000, 70), (3000, 300), (20000, 40)])
def test_jobsched_makespan(cuda, n, M):
    # (20000, 40) runs on the global-memory row kernel
    jt = job_times(n, seed=n + M)
    pb, po = B().jobsched(jt, M), O.OracleProblem(O.JOBSCHED, n, jt=jt, machines=M)
    keys = I.keys(8, n, seed=n)
    keys[0] = 0.0         # every job on machine 0
    keys[1] = 0.99999994  # every job on the last machine
    fit, _ = eval_gpu(pb, keys, cuda)
    np.testing.assert_array_equal(fit.view(np.uint32), O.evaluate(po, keys).view(np.uint32))


@pytest.mark.parametrize("fn", [0, 2])
@pytest.mark.parametrize("n", [1, 2, 30, 1000, 20000])
def test_continuous_exact(cuda, fn, n):
    lo, hi = BOUNDS[fn]
    pb, po = B().continuous(n, lo, hi, fn), O.OracleProblem(O.CONTINUOUS, n, function=fn, lo=lo, hi=hi)
    keys = I.keys(6, n, seed=n + fn)
    fit, _ = eval_gpu(pb, keys, cuda)
    np.testing.assert_array_equal(fit.view(np.uint32), O.evaluate(po, keys).view(np.uint32))


@pytest.mark.parametrize("n", [1, 30, 1000, 20000])
def test_rastrigin_tolerance(cuda, n):
    lo, hi = BOUNDS[1]
    pb, po = B().continuous(n, lo, hi, 1), O.OracleProblem(O.CONTINUOUS, n, function=1, lo=lo, hi=hi)
    keys = I.keys(6, n, seed=n + 11)
    fit, _ = eval_gpu(pb, keys, cuda)
    f64 = O.continuous_f64(po, keys)
    assert np.max(np.abs(fit - f64) / np.maximum(np.abs(f64), 1e-30)) <= 1e-5
    orc = O.evaluate(po, keys)
    assert np.max(np.abs(fit - orc) / np.maximum(np.abs(orc), 1e-30)) <= 1e-5


def test_engine_jobsched_bit_exact(cuda):
    n, M, P, E, Mu, G = 120, 8, 128, 25, 12, 20
    jt = job_times(n, seed=3)
    pb, po = B().jobsched(jt, M), O.OracleProblem(O.JOBSCHED, n, jt=jt, machines=M)
    s = B().Solver(pb, B().params(P, E, Mu, 0.7, G, seed=4))
    s.run()
    keys, fit = s.get_population()
    rk, rf, rh = oracle_islands(po, P, E, Mu, 0.7, 4, 1, 0, 0, G, (n + 3) // 4 * 4)
    np.testing.assert_array_equal(keys, rk)
    np.testing.assert_array_equal(fit, rf)
    np.testing.assert_array_equal(s.get_fitness_history(), rh)
    s.close()


def test_engine_sphere_bit_exact(cuda):
    n, P, E, M, G = 30, 200, 40, 20, 25
    pb = B().continuous(n, -5.12, 5.12, 0)
    po = O.OracleProblem(O.CONTINUOUS, n, function=0, lo=-5.12, hi=5.12)
    s = B().Solver(pb, B().params(P, E, M, 0.7, G, seed=6))
    s.run()
    keys, fit = s.get_population()
    rk, rf, rh = oracle_islands(po, P, E, M, 0.7, 6, 1, 0, 0, G, (n + 3) // 4 * 4)
    np.testing.assert_array_equal(keys, rk)
    np.testing.assert_array_equal(fit, rf)
    assert rh[-1] < rh[0]  # the search makes progress
    s.close()


def test_server_mixed_kinds(cuda):
    """served requests of the new kinds (TSPJ, job scheduling, continuous) give their
    standalone results"""
    b = B()
    travel, jobs = I.tspj_instance(25, seed=7)
    jt = job_times(80, seed=8)
    reqs = [
        (b.tspj(travel, jobs), dict(kind=b.TSPJ, n=25, matrix=travel, matrix2=jobs),
         b.params(96, 19, 9, 0.75, 40, seed=1)),
        (b.jobsched(jt, 6), dict(kind=b.JOBSCHED, n=80, job_times=jt, machines=6), b.params(64, 12, 6, 0.7, 40, seed=2)),
        (b.continuous(20, -5.0, 10.0, 2), dict(kind=b.CONTINUOUS, n=20, function=2, lower=-5.0, upper=10.0),
         b.params(64, 12, 6, 0.7, 40, seed=3)),
    ]
    srv = b.Server(max_active=3, generations_per_tick=8)
    ids = [srv.submit(prm=prm, **kw) for _, kw, prm in reqs]
    done = {}
    for _ in range(200):
        srv.step()
        for rid in ids:
            if rid not in done and srv.poll(rid) is not None:
                done[rid] = srv.poll(rid)
        if len(done) == len(ids):
            break
    for rid, (pb, _, prm) in zip(ids, reqs):
        s = b.Solver(pb, prm)
        s.run()
        assert done[rid][0] == 0 and done[rid][1][0] == s.get_best_individual()[2]
        s.close()
    srv.close()
