"""The multi-rank paths of bench.py on the CPU: gloo process groups of two ranks and the
torchrun launch of the reference arm (no GPU needed)."""
import argparse
import importlib.util
import json
import os
import socket
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _max_worker(rank, world, port, values, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        out[rank] = _bench().max_over_ranks(values[rank])
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_with_gloo():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    port = _free_port()
    procs = [ctx.Process(target=_max_worker, args=(r, 2, port, [3.5, 7.25], out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    assert dict(out) == {0: 7.25, 1: 7.25}


@pytest.mark.parametrize("workload", ["large", "batched"])
def test_ranks_get_disjoint_reads_of_equal_size(workload):
    b = _bench()
    args = argparse.Namespace(workload=workload, scale=0.0005, p=12)
    if workload == "batched":
        args.scale = 0.0002
    s0, l0, r0, p0 = b.workload_of(args, 0)
    s1, l1, r1, p1 = b.workload_of(args, 1)
    assert p0 == p1
    assert all(np.array_equal(x, y) for x, y in zip(s0, s1))  # the same index on every rank
    import sbwt_gpu_b200 as sg
    assert sg.count_kmers(r0, 31) == sg.count_kmers(r1, 31)  # the same work per rank (weak scaling)
    assert l0.size != l1.size or not np.array_equal(l0, l1)  # each rank its own reads


def test_reference_arm_under_torchrun_prints_one_line():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), os.path.join(ROOT, "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "0", "--scale", "0.001",
           "--cpu-seconds", "1"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [x for x in r.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["value"] > 0 and d["e2e"]["h2d_bytes_per_step"] == 0
    # torchrun's OMP_NUM_THREADS=1 does not reach the reference arm: rank 0 runs on every core
    assert d["cpu_baseline"]["cores"] == len(os.sched_getaffinity(0))


def test_host_threads_per_rank(monkeypatch):
    import bench as b
    cores = len(os.sched_getaffinity(0))
    for impl, world, local, env, want in [("ours", 1, 1, "", ""), ("ours", 2, 2, "1", str(max(1, cores // 2))),
                                          ("reference", 2, 2, "1", str(cores)), ("ours", 2, 2, "3", "3"),
                                          ("ours", 4, 2, "", str(max(1, cores // 2)))]:
        monkeypatch.setenv("OMP_NUM_THREADS", env)
        monkeypatch.setenv("LOCAL_WORLD_SIZE", str(local))
        b.host_threads_per_rank(world, impl)
        assert os.environ["OMP_NUM_THREADS"] == want, (impl, world, env)
