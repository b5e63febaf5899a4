"""Batched solving and serving on the GPU.  Each instance's draws are a function of its own
seed, so an instance must give exactly the same result alone (a standalone solver) and in
a batch or in the served mix, whatever else shares the launches."""
import numpy as np
import pytest

import instances as I

pytestmark = pytest.mark.gpu


def B():
    import brkga_b200
    return brkga_b200


def make_mix(seed=0):
    """(problem, params, server-kwargs) for a mix of problem kinds and sizes"""
    b = B()
    out = []
    for i, (n, P) in enumerate([(50, 64), (300, 128), (1200, 96), (17, 40)]):
        xy = I.tsp_coords(n, seed=seed + i)
        out.append((b.tsp(xy), b.params(P, P // 5, P // 10, 0.7, 60, seed=seed + 10 + i),
                    dict(kind=b.TSP_COORDS, n=n, coords=xy)))
    for i, n in enumerate([500, 2100]):
        w, v, cap = I.knap_items(n, seed=seed + 20 + i)
        out.append((b.knapsack(w, v, cap), b.params(100, 15, 15, 0.7, 60, seed=seed + 30 + i),
                    dict(kind=b.KNAP_GREEDY, n=n, weights=w, values=v, capacity=cap)))
    for i, n in enumerate([20, 45]):
        a, c = I.tsp_coords(n + 1, seed=seed + 40 + i), I.tsp_coords(n + 1, seed=seed + 50 + i)
        out.append((b.bitsp(a, c), b.params(32 + 16 * i, 0, 4, 0.7, 60, seed=seed + 60 + i, diversity_interval=25),
                    dict(kind=b.BITSP_COORDS, n=n, coords=a, coords2=c)))
    return out


def alone(problem, prm, gens):
    s = B().Solver(problem, prm)
    s.initialize()
    s.evolve(gens)
    k, p, f = s.get_best_individual()
    s.close()
    return k, np.atleast_1d(np.asarray(f, np.float32))


def test_batch_equals_standalone(cuda):
    mix = make_mix()
    G = 37
    batch = B().Batch([m[0] for m in mix], [m[1] for m in mix])
    batch.evolve(G)
    best = batch.best()
    for i, (pb, prm, _) in enumerate(mix):
        keys, fit = alone(pb, prm, G)
        np.testing.assert_array_equal(best[i, :len(fit)], fit, err_msg=f"instance {i}")
        if pb.num_objectives == 1:
            bk, bf = batch.best_keys(i)
            np.testing.assert_array_equal(bk, keys, err_msg=f"instance {i} keys")
    batch.close()


def test_batch_islands_migration_equals_standalone(cuda):
    b = B()
    probs, prms = [], []
    for i, n in enumerate([120, 400, 60]):
        probs.append(b.tsp(I.tsp_coords(n, seed=70 + i)))
        prms.append(b.params(256, 40, 24, 0.7, 60, seed=80 + i, num_islands=4, migration_interval=5, num_migrants=2))
    batch = b.Batch(probs, prms)
    G = 23
    batch.evolve(10)
    batch.evolve(13)
    best = batch.best()
    for i in range(3):
        _, fit = alone(probs[i], prms[i], G)
        assert best[i, 0] == fit[0]
    batch.close()


def serve_all(server, reqs, max_steps=400):
    done = {}
    for _ in range(max_steps):
        server.step()
        for rid in reqs:
            if rid not in done:
                r = server.poll(rid)
                if r is not None:
                    done[rid] = r
        if len(done) == len(reqs):
            return done
    raise AssertionError(f"served {len(done)} of {len(reqs)}")


def test_server_results_equal_standalone(cuda):
    mix = make_mix(seed=100)
    srv = B().Server(max_active=5, generations_per_tick=16)
    ids = []
    # staggered arrivals: requests join while others are running
    for i, (pb, prm, kw) in enumerate(mix):
        ids.append(srv.submit(prm=prm, **kw))
        if i % 2 == 1:
            srv.step()
    done = serve_all(srv, ids)
    for rid, (pb, prm, kw) in zip(ids, mix):
        code, best, gens, lat = done[rid]
        assert code == 0 and gens == prm.max_generations and lat > 0
        _, fit = alone(pb, prm, prm.max_generations)
        np.testing.assert_array_equal(best[:len(fit)], fit, err_msg=f"request {rid}")
    assert srv.stats() == (0, 0, len(ids))
    srv.close()


def test_server_cancel_stall_and_admission(cuda):
    b = B()
    srv = b.Server(max_active=1, generations_per_tick=10, memory_budget=64 << 20)
    xy = I.tsp_coords(80, seed=1)
    prm = b.params(64, 10, 6, 0.7, 200, seed=3)
    r1 = srv.submit(prm=prm, kind=b.TSP_COORDS, n=80, coords=xy)
    r2 = srv.submit(prm=prm, kind=b.TSP_COORDS, n=80, coords=xy)
    r3 = srv.submit(prm=prm, kind=b.TSP_COORDS, n=80, coords=xy)
    srv.step()  # r1 admitted (one slot)
    assert srv.stats()[:2] == (2, 1)
    srv.cancel(r2)  # still queued
    assert srv.poll(r2)[0] == -5
    srv.step()
    srv.cancel(r1)  # active
    assert srv.poll(r1)[0] == -5
    done = serve_all(srv, [r3])
    assert done[r3][0] == 0 and done[r3][2] == 200
    # stall: a tiny instance stops improving long before its budget
    tiny = srv.submit(prm=b.params(16, 3, 2, 0.7, 5000, seed=4), stall=30, kind=b.TSP_COORDS, n=5,
                      coords=I.tsp_coords(5, seed=2))
    d = serve_all(srv, [tiny], max_steps=1000)
    assert d[tiny][0] == 0 and d[tiny][2] < 5000
    # a request larger than the memory budget is refused at submission
    big = b.params(4096, 600, 600, 0.7, 10, seed=5)
    with pytest.raises(b.BrkgaError) as ei:
        srv.submit(prm=big, kind=b.TSP_COORDS, n=8000, coords=I.tsp_coords(8000, seed=6))
    assert ei.value.code == -7
    # a malformed request is rejected on the host
    with pytest.raises(b.BrkgaError):
        srv.submit(prm=prm, kind=99, n=10)
    srv.close()
