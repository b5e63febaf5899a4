"""The multi-GPU form of the path: independent replicas, one process per GPU.

Each rank runs whole instances on its own device; the job's collectives are a barrier
and the maximum of the elapsed time over ranks.  These tests run that plumbing as two
gloo ranks on the CPU, launched the way the driver launches bench.py (torch.distributed.run),
and check the reference arm's rank behaviour under the same launcher."""
import json
import os
import socket
import subprocess
import sys
import textwrap

import pytest

from conftest import ROOT


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def torchrun(args, timeout=300, env_extra=None):
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="", OMP_NUM_THREADS="1")
    env.update(env_extra or {})
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr=127.0.0.1", f"--master-port={free_port()}"] + args
    return subprocess.run(cmd, env=env, capture_output=True, text=True, timeout=timeout, cwd=ROOT)


WORKER = textwrap.dedent("""
    import json, sys
    sys.path.insert(0, {pkg!r})
    from brkga_b200.replicas import Replicas, whole_job_rate
    reps = Replicas(backend="gloo", timeout_s=60)
    assert reps.world == 2 and reps.device == "cpu"
    # rank r "took" 1.5 * (r + 1) seconds for 10 generations
    elapsed = 1.5 * (reps.rank + 1)
    reps.barrier()
    slowest = reps.max(elapsed)
    total = reps.sum(10.0)
    out = dict(rank=reps.rank, slowest=slowest, total=total, seed=reps.seed(7),
               rate=whole_job_rate(reps.world, 10, slowest), leader=reps.leader)
    reps.close()
    with open({out!r} + "/rank%d.json" % out["rank"], "w") as f:
        json.dump(out, f)
""")


def test_two_gloo_replicas(tmp_path):
    script = tmp_path / "worker.py"
    script.write_text(WORKER.format(pkg=os.path.join(ROOT, "llm-brkga_b200"), out=str(tmp_path)))
    r = torchrun([str(script)], timeout=180)
    assert r.returncode == 0, r.stderr[-3000:]
    res = [json.loads((tmp_path / f"rank{k}.json").read_text()) for k in range(2)]
    assert sorted(x["rank"] for x in res) == [0, 1]
    for x in res:
        assert x["slowest"] == 3.0           # the max over ranks, seen by every rank
        assert x["total"] == 20.0
        assert x["rate"] == pytest.approx(2 * 10 / 3.0)
        assert x["leader"] == (x["rank"] == 0)
    assert {x["seed"] for x in res} == {7, 8}  # replicas run different seeds


def test_single_process_needs_no_process_group():
    sys.path.insert(0, os.path.join(ROOT, "llm-brkga_b200"))
    from brkga_b200.replicas import Replicas, whole_job_rate
    env = {k: os.environ.pop(k) for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK") if k in os.environ}
    try:
        reps = Replicas()
        assert reps.world == 1 and reps.dist is None and reps.leader
        assert reps.max(2.5) == 2.5 and reps.sum(4.0) == 4.0
        reps.barrier()
        reps.close()
        with pytest.raises(ValueError):
            whole_job_rate(1, 10, 0.0)
    finally:
        os.environ.update(env)


def test_reference_arm_under_two_ranks():
    """bench.py --impl reference on two ranks: rank 0 alone times the reference's CPU path
    and prints one line; the other rank exits 0 without work"""
    r = torchrun(["bench.py", "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "0"], timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["cores"] >= 1
