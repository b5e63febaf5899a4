"""NSGA-II engines at the sizes they are measured on, bit for bit against the oracle every
generation (core/population.hpp:409-517, core/solver.hpp:751-817).

At P = 2048 the pool holds 4096 points, so every CTA of the eight-CTA peel cluster owns
live columns (512 each): the front exchange through distributed shared memory, the
peel that stops at the cut front, the selection kernel's cut-front sort (up to a
register-resident bitonic of several thousand entries) and the diversity pass all run at
full width.  The bi-objective TSP runs are BASELINE-shaped (n = 500, mutants 10 %); the
tiny-tour run converges into fronts of thousands of duplicates, so the cut front holds
more than 1024 entries; MO-VRP runs at P = 1500 with the reference's 100-customer
settings."""
import numpy as np
import pytest

import instances as I
import oracle as O

pytestmark = pytest.mark.gpu


def B():
    import brkga_b200
    return brkga_b200


def cut_front(po, pr, g, n, ld, pop, obj, rank, cd, P):
    """(rank, entries) of the front the oracle's survivor selection cuts in generation g:
    the first front where the survivors, first-front points counted twice, exceed P"""
    off = O.nsga2_offspring(pr, g, n, ld, pop, rank, cd)
    pool = np.concatenate([obj, O.evaluate(po, off[:, :n])])
    counts = np.bincount(O.pareto_ranks(pool))
    taken = 0
    for f, c in enumerate(counts):
        w = 2 * int(c) if f == 0 else int(c)
        if taken + w > P:
            return f, w
        taken += w
    return None, 0


def run_lockstep(s, po, pr, n, ld, G, P, track_cut=False):
    pop, obj, rank, cd = O.nsga2_init(po, pr, ld)
    gk, go = s.get_population()
    np.testing.assert_array_equal(gk, pop[:, :n], err_msg="initial population")
    np.testing.assert_array_equal(go, obj, err_msg="initial objectives")
    cuts, rebuilt = [], 0
    plain = O.nsga2_params(pr.P, pr.Mn, pr.rho, pr.mut_rate, pr.seed, 0)
    for g in range(1, G + 1):
        if track_cut:
            cuts.append(cut_front(po, pr, g, n, ld, pop, obj, rank, cd, P))
            # the same generation without the diversity pass: a difference means it rebuilt
            shadow = [x.copy() for x in (pop, obj, rank, cd)]
            O.nsga2_generation(po, plain, g, ld, *shadow)
        s.evolve(1)
        O.nsga2_generation(po, pr, g, ld, pop, obj, rank, cd)
        gk, go = s.get_population()
        np.testing.assert_array_equal(gk, pop[:, :n], err_msg=f"keys, generation {g}")
        np.testing.assert_array_equal(go, obj, err_msg=f"objectives, generation {g}")
        if track_cut:
            rebuilt += int(not np.array_equal(shadow[0], pop))
    fobj, fkeys = s.get_pareto_front()
    np.testing.assert_array_equal(fobj, obj[rank == 0])
    np.testing.assert_array_equal(fkeys, pop[rank == 0][:, :n])
    return cuts, rebuilt


def test_nsga2_bitsp_config3_size(cuda):
    """bi-objective TSP, 500 genes (501 points with the depot), P = 2048, 10 % random
    offspring, rho 0.7; the diversity pass is due after generations 1, 6 and 11"""
    n, P, Mn, G = 500, 2048, 204, 12
    a, b = I.tsp_coords(n + 1, seed=5), I.tsp_coords(n + 1, seed=6)
    pb, po = B().bitsp(a, b), O.OracleProblem(O.BITSP_COORDS, n, xy=a, xy2=b)
    s = B().Solver(pb, B().params(P, 0, Mn, 0.7, G, seed=21, diversity_interval=5))
    s.initialize()
    pr = O.nsga2_params(P, Mn, 0.7, 5.0 / n, 21, 5)
    run_lockstep(s, po, pr, n, 500, G, P)
    s.close()
    pb.close()


def test_nsga2_bitsp_large_cut_front(cuda):
    """a 6-city depot tour at P = 2048: the pool collapses into a few objective pairs
    with hundreds of copies, so the cut front holds more than 1024 (up to about 2100)
    entries, and the diversity pass rebuilds the population"""
    n, P, G = 6, 2048, 12
    a, b = I.tsp_coords(n + 1, seed=5), I.tsp_coords(n + 1, seed=6)
    pb, po = B().bitsp(a, b), O.OracleProblem(O.BITSP_COORDS, n, xy=a, xy2=b)
    s = B().Solver(pb, B().params(P, 0, 0, 0.7, G, seed=21, diversity_interval=5))
    s.initialize()
    pr = O.nsga2_params(P, 0, 0.7, 5.0 / n, 21, 5)
    cuts, rebuilt = run_lockstep(s, po, pr, n, 8, G, P, track_cut=True)
    assert max(w for _, w in cuts) > 1024, cuts
    assert any(f == 0 for f, _ in cuts), cuts  # a generation whose first front is cut
    assert rebuilt > 0
    s.close()
    pb.close()


def test_movrp_p1500(cuda):
    """MO-VRP, 100 customers, fleet 16, P = 1500, rho 0.10 (the reference's
    configure_for_size at 100 customers); diversity pass every 4 generations"""
    n, P, G = 100, 1500, 10
    xy, dem, cap, V = I.movrp_instance(n, seed=31, vehicles=16)
    pb = B().movrp(xy, dem, cap, V)
    po = O.OracleProblem(O.MOVRP, n, xy=xy, w=dem, machines=V, vcap=cap)
    s = B().Solver(pb, B().params(P, 0, 0, 0.10, G, seed=13, diversity_interval=4))
    s.initialize()
    pr = O.nsga2_params(P, 0, 0.10, 5.0 / n, 13, 4)
    run_lockstep(s, po, pr, n, 100, G, P)
    s.close()
    pb.close()
