"""MO-VRP on the GPU (MultiObjectiveVRPConfig, configs/multi_objective_vrp_config.hpp): the
row's keys become the reference's biased sort values (a float hash of the whole row), one
argsort gives the visiting order, and one warp splits it into capacity-feasible routes in
the reference's own order of float additions.  Decodes and both objectives must equal the
oracle's -- pinned bit for bit to the reference's decode_solution -- including ties,
overloaded customers and fleets too small for the routes; whole NSGA-II runs must equal
the oracle's generation by generation."""
import numpy as np
import pytest

import instances as I
import oracle as O
from test_gpu_ops import B, eval_gpu

pytestmark = pytest.mark.gpu


def problems(n, seed, vehicles=None, overload=False):
    xy, dem, cap, V = I.movrp_instance(n, seed, vehicles, overload)
    pb = B().movrp(xy, dem, cap, V)
    po = O.OracleProblem(O.MOVRP, n, xy=xy, w=dem, machines=V, vcap=cap)
    return pb, po, dem, cap


@pytest.mark.parametrize("n,V,overload", [(1, None, False), (2, 1, False), (31, 5, False), (31, 2, True),
                                          (300, None, False), (1000, 40, True), (5000, None, False)])
def test_movrp_decode_objectives(cuda, n, V, overload):
    pb, po, dem, cap = problems(n, seed=n + 3, vehicles=V, overload=overload)
    assert pb.num_objectives == 2
    keys = I.keys(8, n, seed=n + 4)
    keys[1] = I.tied_keys(1, n, seed=n + 5)[0]  # ties: the lower index first
    obj, perm = eval_gpu(pb, keys, cuda)
    np.testing.assert_array_equal(perm, O.decode_problem(po, keys))
    np.testing.assert_array_equal(obj.view(np.uint32), O.evaluate(po, keys).view(np.uint32))
    routes = B().movrp_routes(perm[0], dem, cap)
    route_of, count = O.movrp_routes(po, perm[0])
    assert len(routes) == count
    assert [c for r in routes for c in r] == (perm[0] + 1).tolist()


@pytest.mark.parametrize("n", [300, 5000])
def test_movrp_degenerate_keys(cuda, n):
    """rows whose sort values crowd a few buckets (a NaN key makes the row hash, and so
    every value, NaN; huge keys swamp the index offsets) take the bounded fallback sort"""
    pb, po, _, _ = problems(n, seed=n + 9)
    keys = I.degenerate_keys(n, seed=n + 10)
    keys[4] = np.float32(3.0e30)  # every value the same float: ties by index
    obj, perm = eval_gpu(pb, keys, cuda)
    np.testing.assert_array_equal(perm, O.decode_problem(po, keys))
    np.testing.assert_array_equal(obj.view(np.uint32), O.evaluate(po, keys).view(np.uint32))


def test_movrp_engine_nsga2_bit_exact(cuda):
    n, P, G = 40, 64, 20
    pb, po, _, _ = problems(n, seed=8, vehicles=4)
    # the reference's MO-VRP settings: rho 0.10 (configure_for_size, :207-209)
    s = B().Solver(pb, B().params(P, 0, 0, 0.10, G, seed=17, diversity_interval=25))
    s.initialize()
    ld = 40
    pr = O.nsga2_params(P, 0, 0.10, 5.0 / n, 17, 25)
    pop, obj, rank, cd = O.nsga2_init(po, pr, ld)
    gk, go = s.get_population()
    np.testing.assert_array_equal(go, obj)
    for g in range(1, G + 1):
        s.evolve(1)
        O.nsga2_generation(po, pr, g, ld, pop, obj, rank, cd)
        gk, go = s.get_population()
        np.testing.assert_array_equal(gk, pop[:, :n], err_msg=f"generation {g}")
        np.testing.assert_array_equal(go, obj, err_msg=f"generation {g}")
    fobj, fkeys = s.get_pareto_front()
    np.testing.assert_array_equal(fobj, obj[rank == 0])
    s.close()


def test_movrp_engine_captured_runs(cuda):
    """a whole run (captured graphs of 16 generations) equals the same run one generation
    at a time"""
    n, P, G = 60, 96, 40
    pb, _, _, _ = problems(n, seed=9)
    a = B().Solver(pb, B().params(P, 0, 0, 0.10, G, seed=5))
    a.run()
    b = B().Solver(pb, B().params(P, 0, 0, 0.10, G, seed=5))
    b.initialize()
    for _ in range(G):
        b.evolve(1)
    for x, y in zip(a.get_population(), b.get_population()):
        np.testing.assert_array_equal(x, y)
    a.close()
    b.close()


def test_movrp_rejected_in_batches_and_server(cuda):
    pb, _, _, _ = problems(20, seed=9)
    with pytest.raises(B().BrkgaError) as ei:
        B().Batch([pb], [B().params(32, 0, 0, 0.1, 5, seed=1)])
    assert ei.value.code == -6
    xy, dem, cap, V = I.movrp_instance(20, 9)
    srv = B().Server(max_active=2, generations_per_tick=4)
    with pytest.raises(B().BrkgaError) as ei:
        srv.submit(kind=B().MOVRP, n=20, prm=B().params(32, 0, 0, 0.1, 5, seed=1), coords=xy, demands=dem,
                   vehicle_capacity=cap, vehicles=V)
    assert ei.value.code == -6
    srv.close()


def test_movrp_invalid_instances_rejected(cuda):
    xy, dem, cap, V = I.movrp_instance(10, 10)
    bad = dem.copy()
    bad[3] = -1
    for kw in (dict(demands=bad, vehicle_capacity=cap, vehicles=V), dict(demands=dem, vehicle_capacity=0, vehicles=V),
               dict(demands=dem, vehicle_capacity=cap, vehicles=0)):
        with pytest.raises(B().BrkgaError) as ei:
            B().Problem(B().MOVRP, 10, coords=xy, **kw)
        assert ei.value.code == -1


def test_cpp_movrp_dropin_program(cuda, tmp_path):
    """the reference-style C++ program (VRP file -> MultiObjectiveVRPConfig::load_from_file ->
    configure_for_size -> Solver) gives the same first front as the Python binding on the
    instance it wrote, with the reference's NSGA-II settings (rho 0.10, no random offspring)"""
    import json
    import os
    import subprocess
    exe = os.path.join(os.path.dirname(B().LIB_PATH), "..", "build", "solve_movrp")
    r = subprocess.run([exe, str(tmp_path), "31", "5", "3", "128", "60"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    out = json.loads(r.stdout.strip().splitlines()[-1])
    lines = open(tmp_path / "synthetic-n32-k5.vrp").read().splitlines()
    cap = int(next(l for l in lines if l.startswith("CAPACITY")).split(":")[1])
    c0 = lines.index("NODE_COORD_SECTION") + 1
    d0 = lines.index("DEMAND_SECTION") + 1
    xy = np.array([[float(v) for v in l.split()[1:]] for l in lines[c0:c0 + 32]], np.float32)
    dem = np.array([int(l.split()[1]) for l in lines[d0:d0 + 32]], np.int32)
    assert out["vehicles"] == 5 and out["capacity"] == cap
    s = B().Solver(B().movrp(xy, dem, cap, 5), B().params(128, 25, 0, 0.10, 60, seed=7))
    s.run()
    fobj, _ = s.get_pareto_front()
    assert sorted(map(tuple, np.asarray(out["front"], np.float32).tolist())) == sorted(map(tuple, fobj.tolist()))
    s.close()
