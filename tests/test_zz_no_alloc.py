"""The allocation-free Pareto-rank entry point (brkga_pareto_rank_noalloc), called through
the C ABI, against the allocating entry point (brkga_pareto_rank) on the same inputs.

Some callers cannot allocate device memory -- a plugin running under a framework whose
allocator owns the GPU, or a serving loop that must not call cudaMalloc after start-up --
so this entry point keeps its scratch in a fixed device array inside the library.  Ranks
are integers: the comparison is exact.  Two calls in a row check that the shared array's
leftover contents from the first call do not leak into the second.  This file is
collected last so that a stop-at-first-failure run has run every other test first."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _points(N, m, seed):
    rng = np.random.default_rng(seed)
    obj = rng.random((N, m), dtype=np.float32)
    obj[::3] = np.round(obj[::3] * 8) / 8  # ties and duplicates
    return np.ascontiguousarray(obj.astype(np.float32))


def test_noalloc_ranks_match_allocating_entry_point(cuda):
    import torch

    import brkga_b200 as B
    L = B.lib()
    cases = [(2048, 2, 1), (1500, 2, 2), (700, 3, 3), (1, 2, 4)]
    for N, m, seed in cases:
        d_obj = torch.from_numpy(_points(N, m, seed)).to(cuda)
        want = torch.full((N,), -1, dtype=torch.int32, device=cuda)
        B.check(L.brkga_pareto_rank(d_obj.data_ptr(), N, m, want.data_ptr(), None))
        for call in range(2):  # two calls in a row on the shared array
            got = torch.full((N,), -7, dtype=torch.int32, device=cuda)
            B.check(L.brkga_pareto_rank_noalloc(d_obj.data_ptr(), N, m, got.data_ptr(), None))
            torch.cuda.synchronize()
            np.testing.assert_array_equal(got.cpu().numpy(), want.cpu().numpy(), err_msg=f"N={N} call {call}")


def test_noalloc_rejects_sizes_above_its_limit(cuda):
    import torch

    import brkga_b200 as B
    L = B.lib()
    N = 2049
    d_obj = torch.zeros(N * 2, dtype=torch.float32, device=cuda)
    d_rank = torch.zeros(N, dtype=torch.int32, device=cuda)
    code = L.brkga_pareto_rank_noalloc(d_obj.data_ptr(), N, 2, d_rank.data_ptr(), None)
    assert code == -6
    assert "2048" in B.last_error()
