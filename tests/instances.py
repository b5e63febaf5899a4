"""Seeded synthetic instances with the shapes and value distributions of the workloads
(uniform coordinates, uniform integer knapsack items); no dataset is read."""
import numpy as np


def tsp_coords(n, seed, scale=1.0):
    return (np.random.default_rng(seed).random((n, 2), dtype=np.float32) * np.float32(scale)).astype(np.float32)


def knap_items(n, seed, lo=1, hi=100):
    rng = np.random.default_rng(seed)
    w = rng.integers(lo, hi + 1, n, dtype=np.int32)
    v = rng.integers(lo, hi + 1, n, dtype=np.int32)
    cap = np.float32(0.5 * float(w.sum()))
    return w, v, cap


def keys(rows, n, seed):
    """keys in [0,1) drawn on the 24-bit grid the engine itself produces"""
    rng = np.random.default_rng(seed)
    return (rng.integers(0, 1 << 24, (rows, n)).astype(np.float32) / np.float32(1 << 24)).astype(np.float32)


def tied_keys(rows, n, seed, levels=8):
    """keys with many exact ties (ties go to the lower index)"""
    rng = np.random.default_rng(seed)
    return (rng.integers(0, levels, (rows, n)).astype(np.float32) / np.float32(levels)).astype(np.float32)


def wild_keys(rows, n, seed):
    """keys outside [0,1): negatives, values above one, signed zeros, infinities"""
    rng = np.random.default_rng(seed)
    k = (rng.standard_normal((rows, n)) * 3).astype(np.float32)
    flat = k.reshape(-1)
    idx = rng.choice(flat.size, size=max(1, flat.size // 20), replace=False)
    specials = np.array([0.0, -0.0, np.inf, -np.inf, 1.0, 0.5], np.float32)
    flat[idx] = specials[rng.integers(0, specials.size, idx.size)]
    return k


def movrp_instance(n, seed, vehicles=None, overload=False):
    """capacitated VRP over the depot (point 0) and n customers: coordinates uniform in
    [0,100)^2, demands uniform in {1..30} (depot 0), capacity about 1.1 x total demand /
    vehicles (vehicles defaults to max(3, n // 6), the reference's own estimate); with
    overload one customer's demand exceeds the capacity"""
    rng = np.random.default_rng(seed)
    xy = (rng.random((n + 1, 2)) * 100.0).astype(np.float32)
    dem = rng.integers(1, 31, n + 1).astype(np.int32)
    dem[0] = 0
    V = vehicles if vehicles is not None else max(3, n // 6)
    cap = int(np.ceil(1.1 * dem.sum() / V))
    if overload and n >= 2:
        dem[1 + n // 2] = cap + 7
    return xy, dem, cap, V


def tspj_instance(c, seed):
    """TSPJ data over the depot and c cities: travel times = Euclidean distances of seeded
    points in [0,100)^2 (as the reference's *_TT.csv files hold), job durations uniform in
    [1,100) per (city, job type), the depot row zero"""
    rng = np.random.default_rng(seed)
    xy = rng.random((c + 1, 2)) * 100.0
    travel = np.sqrt(((xy[:, None, :] - xy[None, :, :]) ** 2).sum(-1)).astype(np.float32)
    jobs = (1.0 + rng.random((c + 1, c + 1)) * 99.0).astype(np.float32)
    jobs[0, :] = 0.0
    return travel, jobs


def degenerate_keys(n, seed):
    """rows whose keys crowd into a few buckets of a value-range bucket sort: every key equal
    (0, 0.5, 1, -3), keys in [1, 10), negative keys, NaN-heavy rows, infinities and signed
    zeros, four tie levels; the last row is ordinary keys in [0, 1)"""
    rng = np.random.default_rng(seed)
    rows = [np.zeros(n), np.full(n, 0.5), np.full(n, 1.0), np.full(n, -3.0),
            1.0 + 9.0 * rng.random(n), -5.0 * rng.random(n)]
    nan = rng.random(n)
    nan[rng.random(n) < 0.6] = np.nan
    rows.append(nan)
    ext = rng.choice(np.array([np.inf, -np.inf, 0.0, -0.0, 0.3], np.float64), n)
    rows.append(ext)
    rows.append(rng.integers(0, 4, n) / 4.0)
    rows.append(rng.random(n))
    return np.ascontiguousarray(np.array(rows, np.float64).astype(np.float32))
