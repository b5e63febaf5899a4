"""CPU tests of the C-ABI library: it loads, exports every function include/brkga_b200.h
declares, and reports errors through brkga_last_error without needing a GPU."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

import brkga_b200 as B


def test_library_exports_every_header_symbol():
    L = B.lib()
    names = B.header_functions()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_abi_version():
    assert B.lib().brkga_abi_version() == 1


def test_params_default_matches_reference_defaults():
    p = B.Params()
    B.lib().brkga_params_default(C.byref(p))
    # core/config.hpp:78-84
    assert (p.population_size, p.elite_size, p.mutant_size, p.elite_prob, p.max_generations) == (100, 20, 10, 0.7, 1000)


def test_invalid_problem_reports_error():
    d = B.ProblemDesc(99, 10, None, None, None, None, None, None, 0.0)
    h = C.c_void_p()
    code = B.lib().brkga_problem_create(C.byref(d), 0, C.byref(h))
    assert code != 0
    assert B.last_error()


def test_null_arguments_rejected():
    L = B.lib()
    assert L.brkga_evaluate_population(None, None, None, 1, 1, 1, None, None) == -1
    assert "null" in B.last_error()
    assert L.brkga_sort_fitness(None, 4, 1, 0, None, None) == -1
    assert L.brkga_create(None, None, None) == -1
    assert L.brkga_pareto_rank(None, 4, 2, None, None) == -1


def test_header_compiles_as_c():
    hdr = os.path.join(os.path.dirname(B.HEADER_PATH))
    src = '#include "brkga_b200.h"\nint main(void){ brkga_params p; brkga_params_default(&p); return 0; }\n'
    r = subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-fsyntax-only", "-I", hdr, "-x", "c", "-"],
                       input=src, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_product_does_not_reference_the_oracle():
    """the CUDA library and its Python binding never load the oracle or the reference"""
    pkg = os.path.join(B.REPO_DIR, "llm-brkga_b200")
    for root, _, files in os.walk(pkg):
        for f in files:
            if f.endswith((".py", ".cu", ".h", ".cuh", ".hpp", ".cpp")):
                txt = open(os.path.join(root, f)).read()
                assert "liboracle" not in txt and "orc_" not in txt and "libref" not in txt, f


def test_problem_desc_layout_matches_header():
    """the ctypes mirror of brkga_problem_desc has the C struct's size and field offsets"""
    hdr = os.path.dirname(B.HEADER_PATH)
    fields = [f[0] for f in B.ProblemDesc._fields_]
    src = ('#include <stdio.h>\n#include <stddef.h>\n#include "brkga_b200.h"\nint main(void){ printf("%zu", '
           'sizeof(brkga_problem_desc));' + "".join(
               f' printf(" %zu", offsetof(brkga_problem_desc, {f}));' for f in fields) + " return 0; }\n")
    exe = os.path.join(os.environ.get("TMPDIR", "/tmp"), f"desc_layout_{os.getpid()}")
    r = subprocess.run(["gcc", "-std=c99", "-I", hdr, "-x", "c", "-", "-o", exe], input=src, capture_output=True,
                       text=True)
    assert r.returncode == 0, r.stderr
    out = [int(x) for x in subprocess.run([exe], capture_output=True, text=True).stdout.split()]
    os.remove(exe)
    assert out[0] == C.sizeof(B.ProblemDesc)
    assert out[1:] == [getattr(B.ProblemDesc, f).offset for f in fields]


def test_movrp_route_listing():
    """movrp_routes (report formatting of a device-decoded order) splits routes where the
    reference's decode_routes does"""
    import instances as I
    import oracle as O
    for n, V, ov in ((1, None, False), (31, 5, False), (60, 2, True)):
        xy, dem, cap, Vv = I.movrp_instance(n, n, V, ov)
        po = O.OracleProblem(O.MOVRP, n, xy=xy, w=dem, machines=Vv, vcap=cap)
        for perm in O.decode_problem(po, I.keys(4, n, n + 1)):
            routes = B.movrp_routes(perm, dem, cap)
            route_of, count = O.movrp_routes(po, perm)
            assert len(routes) == count
            assert [r for r, rt in enumerate(routes) for _ in rt] == route_of.tolist()
            assert [c for rt in routes for c in rt] == (perm + 1).tolist()
