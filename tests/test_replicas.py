"""Multi-GPU host logic on CPU: the replica group's barrier / max / sum over two gloo ranks (the
same calls bench.py makes over NCCL), the whole-job rate, and the reference arm's rank-0-only rule."""
import importlib.util
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

from conftest import PKG_DIR, ROOT


def _replicas():
    spec = importlib.util.spec_from_file_location("wfb200_replicas", os.path.join(PKG_DIR, "replicas.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    rep = _replicas()
    g = rep.ReplicaGroup("gloo", timeout_s=30)
    g.barrier()
    # rank r measured (r + 1) * 100 ms for 2 steps of 1000 units each
    slowest = g.max((rank + 1) * 0.1)
    total = g.sum(rank + 1)
    rate = rep.whole_job_rate(1000, 2, g.world, slowest)
    g.barrier()
    g.close()
    out.put((rank, slowest, total, rate))


def test_two_gloo_ranks_agree_on_max_and_sum():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, slowest, total, rate in results:
        assert slowest == pytest.approx(0.2)  # every rank sees the slowest replica
        assert total == 3.0
        assert rate == pytest.approx(1000 * 2 * 2 / 0.2)


def test_single_process_group_is_identity():
    rep = _replicas()
    env = {k: os.environ.pop(k) for k in ("WORLD_SIZE", "RANK") if k in os.environ}
    try:
        g = rep.ReplicaGroup("gloo")
        assert not g.active and g.world == 1 and g.rank == 0
        assert g.max(3.5) == 3.5 and g.sum(2.0) == 2.0
        g.barrier()
        g.close()
    finally:
        os.environ.update(env)
    with pytest.raises(ValueError):
        rep.whole_job_rate(1, 1, 1, 0.0)


def test_reference_arm_runs_on_rank_zero_only():
    """bench.py --impl reference under torchrun: ranks other than 0 exit 0 without work or output."""
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2"],
                       capture_output=True, text=True, timeout=120, env=env)
    assert p.returncode == 0, p.stderr
    assert p.stdout.strip() == ""


def test_bench_gpus_flag_starts_its_own_ranks():
    """`bench.py --gpus 2` without a launcher starts two ranks itself; rank 0 alone prints the line,
    which reports both ranks (the reference arm: rank 0 times the CPU arm, the other exits)."""
    import json
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = {k: v for k, v in os.environ.items() if k not in ("WORLD_SIZE", "RANK", "LOCAL_RANK")}
    out = subprocess.run([sys.executable, os.path.join(root, "bench.py"), "--impl", "reference", "--gpus", "2",
                          "--steps", "1", "--warmup", "3", "--ref-spp", "1"],
                         capture_output=True, text=True, timeout=600, env=env)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [json.loads(l) for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1 and lines[0]["n_gpus"] == 2 and lines[0]["impl"] == "reference"


def test_bench_gpus_flag_must_match_the_launcher():
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ, WORLD_SIZE="3", RANK="0")
    out = subprocess.run([sys.executable, os.path.join(root, "bench.py"), "--impl", "reference", "--gpus", "2"],
                         capture_output=True, text=True, timeout=120, env=env)
    assert out.returncode != 0 and "WORLD_SIZE=3" in out.stderr
