"""Generate the golden vectors in tests/golden/*.npz by running the reference's own code
(hsaseendran/llm-brkga headers compiled into oracle/_ref/libref.so by oracle/Makefile) on
seeded synthetic inputs.  Run in this container, where the reference tree exists:

    make -C oracle ref && CUDA_VISIBLE_DEVICES= python tests/golden/make_golden.py [name ...]

The reference must see no GPU so that it takes its CPU path.  Inputs are seeded numpy
draws (uniform coordinates and keys, uniform integer knapsack items); nothing is read
from any dataset.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")]

import oracle as O  # noqa: E402
import ref_checks as RC  # noqa: E402


def main():
    assert os.environ.get("CUDA_VISIBLE_DEVICES") == "", "run with CUDA_VISIBLE_DEVICES="
    out = {}
    out["tsp52"] = RC.ref_tsp_case(n=52, rows=16, seed=1, scale=1000.0)
    out["tsp_matrix9"] = RC.ref_tsp_matrix_case(n=9, rows=12, seed=2)
    out["knap200"] = RC.ref_knap_case(n=200, rows=16, seed=3)
    out["bitsp30"] = RC.ref_bitsp_case(n=30, rows=16, seed=4)
    out["pareto300"] = RC.ref_pareto_case(N=300, seed=5, dup=False)
    out["pareto_dup256"] = RC.ref_pareto_case(N=256, seed=6, dup=True)
    out["select"] = RC.ref_select_case(N=200, P=100, seed=7)
    out["generation"] = RC.ref_generation_case(n=20, P=40, E=8, M=4, rho=0.7, seed=8)
    out["nsga_offspring"] = RC.ref_nsga_offspring_case(n=15, P=24, rho=0.7, seed=9)
    out["tspj20"] = RC.ref_tspj_case(c=20, rows=16, seed=10)
    out["movrp31"] = RC.ref_movrp_case(n=31, rows=16, seed=11, vehicles=5)
    out["movrp_penalties60"] = RC.ref_movrp_case(n=60, rows=8, seed=12, vehicles=2, overload=True)
    out["jobsched300"] = RC.ref_job_case(n=300, machines=32, rows=16, seed=13)
    for f, name in enumerate(("sphere", "rastrigin", "rosenbrock")):
        out["cont_" + name + "30"] = RC.ref_cont_case(function=f, n=30, rows=8, seed=14 + f)
    only = sys.argv[1:]  # optional: names of the fixtures to (re)generate
    for name, d in out.items():
        if only and name not in only:
            continue
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **d)
        print(name, {k: v.shape for k, v in d.items()})


if __name__ == "__main__":
    main()
