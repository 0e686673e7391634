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


def test_answer_transfer_degrades_with_the_per_rank_thread_split(monkeypatch):
    """Under torchrun each rank of this project's arm gets cores / ranks host threads; with 8 ranks on a
    16-core node that is 2.  The host pipeline then sends the share of chunks that lets the copy engines
    and the 2 expanding threads finish together as u64 answers (72 %), not every chunk (the all-dense form,
    PCIe-bound) and not none (2 threads would expand far slower than PCIe copies).  The shares are the
    measured optima of a sweep on the GPU box (large workload, 16 cores): 0.7 at 2 threads gave 6.6G
    k-mers/s against 6.1G all-dense and 3.0G all-sparse."""
    import bench as b
    import sbwt_gpu_b200 as sg
    monkeypatch.delenv("SBWT_PIPELINE_TRANSFER", raising=False)
    n = 100_200_000  # the large workload's columns
    monkeypatch.setenv("OMP_NUM_THREADS", "1")  # what torchrun sets
    monkeypatch.setenv("LOCAL_WORLD_SIZE", "8")
    monkeypatch.setattr(os, "sched_getaffinity", lambda pid: set(range(16)))
    b.host_threads_per_rank(8, "ours")
    t = int(os.environ["OMP_NUM_THREADS"])
    assert t == 2
    f = sg.pipeline_dense_share(n, t)
    assert f == pytest.approx(0.7)
    assert [sg.pipeline_dense_share(n, x) for x in (3, 4, 5)] == pytest.approx([0.5, 0.3, 0.15])
    monkeypatch.setenv("SBWT_PIPELINE_DENSE_SHARE", "0.42")
    assert sg.pipeline_dense_share(n, 2) == pytest.approx(0.42)
    monkeypatch.delenv("SBWT_PIPELINE_DENSE_SHARE")
    # more threads: all sparse; fewer: a larger dense share; indexes past 2^32 columns: all dense
    assert sg.pipeline_dense_share(n, 16) == 0.0 and sg.pipeline_dense_share(n, 6) == 0.0
    assert sg.pipeline_dense_share(n, 1) >= f > sg.pipeline_dense_share(n, 4) > 0.0
    assert sg.pipeline_dense_share(1 << 33, 16) == 1.0
    monkeypatch.setenv("SBWT_PIPELINE_TRANSFER", "sparse")
    assert sg.pipeline_dense_share(n, 2) == 0.0


@pytest.mark.parametrize("n_parts", [1, 2, 3, 4, 8])
def test_partition_rows_balances_kmers_and_never_splits_a_row(n_parts):
    """sbwt_partition_rows (the split of sbwt_search_reads_host_multi, one range per GPU): contiguous
    ranges covering every row once, each within one row's k-mers of an equal share."""
    import numpy as np
    import sbwt_gpu_b200 as sg
    rng = np.random.default_rng(n_parts)
    k = 31
    lens = rng.choice([0, 10, 31, 150, 151, 2000, 15_000], size=5000, p=[.05, .05, .05, .6, .1, .1, .05])
    rows = np.zeros(lens.size + 1, dtype=np.uint64)
    rows[1:] = np.cumsum(lens)
    b = sg.partition_rows(rows, k, n_parts).astype(np.int64)
    assert b[0] == 0 and b[-1] == lens.size and (np.diff(b) >= 0).all()
    per_row = np.maximum(lens - k + 1, 0)
    counts = np.array([per_row[b[i]:b[i + 1]].sum() for i in range(n_parts)])
    assert counts.sum() == per_row.sum()
    assert np.abs(counts - per_row.sum() / n_parts).max() <= per_row.max()
    # a batch with fewer rows than parts: empty ranges, nothing lost
    few = np.array([0, 200, 400], dtype=np.uint64)
    bf = sg.partition_rows(few, k, 4).astype(np.int64)
    assert bf[0] == 0 and bf[-1] == 2 and (np.diff(bf) >= 0).all()
