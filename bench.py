#!/usr/bin/env python
"""k-mers queried per second on B200 GPUs (one process per GPU).

Default workload (the large configuration): a seeded 100 Mbp genome (41% GC,
i.i.d.) plus 5% of its length as inserted 1-10 kbp repeat copies mutated at
0.1%; SBWT of all its 31-mers; presearch depth p = 12; 10M reads of 150 bp
(10% genome-sampled with 1% substitutions, 90% uniform random) = 1.2G k-mers.

One step = one pass of the search path over the whole batch:
  `value`: letters + row table resident in HBM -> pack -> per-row k-mer table
           -> persistent search kernel -> u64 answers + membership bitmap,
           timed with CUDA events on the launching stream (inputs and outputs,
           1.5 GB + 9.6 GB, are larger than L2; no flush needed);
  `e2e`:   the same through sbwt_search_reads_host with pinned host buffers:
           letters and row starts host->device, answers device->host (as a
           bitmap + the found k-mers' node ids, expanded into the u64 answers
           by the host threads), inside the timed region (host wall clock
           around the synchronous call).
With --gpus N (torchrun), every rank holds a replica of the index and searches
its own 10M reads (weak scaling, no collective on the data path); the time
is the max over ranks.

--impl reference times the reference's search semantics on the host cores:
the reference has no CPU search, so its arm is the C restatement in oracle/
(OpenMP, all host threads), on a bounded sample of the same workload.
"""
import argparse
import json
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

METRIC = "k-mers queried/sec on 1 B200, plain vs learned-prefiltered search, bit-exact"
UNIT = "k-mers/s"
FALLBACK_HBM_GBS = 6650.0
FALLBACK_BF16_TFLOPS = 1590.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--scale", type=float, default=1.0, help="shrinks the workload (tests only)")
    ap.add_argument("--query-scale", type=float, default=1.0,
                    help="shrinks the query batch of the large workload only (the index stays full size)")
    ap.add_argument("--p", type=int, default=12)
    ap.add_argument("--kpt", type=int, default=0)
    ap.add_argument("--tpk", type=int, default=0)
    ap.add_argument("--tpb", type=int, default=0)
    ap.add_argument("--layout", choices=["lines", "poppy", "lines512", "lines2048"], default="lines")
    ap.add_argument("--sb", type=int, default=1024, help="bits in superblock of the poppy layout")
    ap.add_argument("--l2-fetch", type=int, default=0, choices=[0, 32, 64, 128],
                    help="L2 fetch granularity in bytes for the searches (0: leave the device default)")
    ap.add_argument("--window", type=int, default=0, choices=[0, 64, 128, 256], help="run-walk window (0: default)")
    ap.add_argument("--evict", type=int, default=-1, choices=[-1, 0, 1, 2],
                    help="evict-first gathers: 0 by table size, 1 never, 2 always (-1: default)")
    ap.add_argument("--l2-persist", type=int, default=-1, choices=[-1, 0, 1], help="rank lines in the L2 set-aside")
    ap.add_argument("--blocks-per-sm", type=int, default=0, help="resident blocks per SM of the run walk (0: as many as fit)")
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="CPU baseline sample budget")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-prefilter", action="store_true", help="skip the learned-prefilter leg")
    ap.add_argument("--no-autotune", action="store_true", help="skip the autotuned leg")
    ap.add_argument("--no-per-kmer", action="store_true", help="skip the leg that searches every k-mer")
    ap.add_argument("--no-contract", action="store_true", help="skip the leg on the reference's kernel contract")
    ap.add_argument("--no-workloads", action="store_true",
                    help="skip the batched and pangenome workloads measured beside the headline")
    ap.add_argument("--workload-steps", type=int, default=3, help="timed steps of each workload beside the headline")
    ap.add_argument("--search-mode", choices=["every", "skip", "stream"], default="stream",
                    help="main leg: every k-mer searched (as the reference), absent-run skip, or skip + backward steps")
    ap.add_argument("--pf-queries", type=int, default=200_000_000)
    ap.add_argument("--pf-steps", type=int, default=20000)
    ap.add_argument("--workload", choices=["large", "batched", "pangenome"], default="large",
                    help="large (default, the headline); batched = 64 files of uneven reads over the small "
                         "index; pangenome = 20 haplotypes of a 50 Mbp base")
    return ap.parse_args()


MODES = {"every": 0, "skip": 1, "stream": 2}

WORKLOADS = {
    "large": "large: 100 Mbp genome (41% GC) + 5% repeats, SBWT k=31, p=12, "
             "10M reads x 150 bp (10% genome-sampled with 1% subs, 90% random)",
    "batched": "batched: index of the small workload (1 Mbp, k=31); 64 query files, read lengths 70% 150 bp / "
               "20% lognormal(2 kbp, 1.0) / 10% lognormal(15 kbp, 0.8) in [31, 1e5]; 500M k-mers, 30% of reads "
               "genome-sampled with 2% subs; one persistent launch",
    "pangenome": "pangenome: 20 haplotypes of a 50 Mbp base (41% GC), 0.5% SNPs, 0.05% indels of 1-20 bp; SBWT "
                 "of the union k-mer set, k=31, p=14; 2G k-mers from 150 bp and lognormal 10 kbp reads, "
                 "95% negatives",
}


def workload_of(args, rank):
    """(sequences to index, letters, row starts, p) of the selected workload; every rank gets its own reads."""
    from sbwt_gpu_b200 import workloads as wl
    if args.workload == "large":
        genome, letters, rows = workload(args.scale, rank, getattr(args, "query_scale", 1.0))
        return [genome], letters, rows, args.p
    if args.workload == "batched":
        letters, rows = batched_queries(args, rank)
        return [wl.small_workload(seed=1235)["genome"]], letters, rows, 10
    haps, letters, rows = pangenome_workload(args, rank)
    return haps, letters, rows, 14


def batched_queries(args, rank):
    """64 FASTA files of uneven reads over the small workload's genome (500M k-mers), written and read back
    with the project's query reader (sbwt_queries_read_many) as one batch."""
    import sbwt_gpu_b200 as sg
    from sbwt_gpu_b200 import workloads as wl
    genome = wl.small_workload(seed=1235)["genome"]
    d = tempfile.mkdtemp(prefix="sbwt_batched_")
    paths = []
    total = int(500_000_000 * args.scale)
    for f, (lt, rw) in enumerate(wl.uneven_read_files(genome, seed=1237 + 100 * rank, total_kmers=total)):
        path = os.path.join(d, f"q{f:02d}.fa")
        wl.write_fasta(path, lt, rw)
        paths.append(path)
    letters, rows, _, _ = sg.read_queries_many(paths, 31)
    shutil.rmtree(d, ignore_errors=True)
    return letters, rows


def pangenome_workload(args, rank):
    """20 haplotypes of a 50 Mbp base (41% GC; 0.5% SNPs, 0.05% indels of 1-20 bp) and 2G k-mers of queries:
    150 bp reads and 10% lognormal ~10 kbp reads, 5% of the reads copied from a haplotype (95% negatives)."""
    from sbwt_gpu_b200 import workloads as wl
    rng = wl.rng_for(1239)
    base = wl.random_bases(rng, int(50_000_000 * args.scale), gc=0.41)
    haps = wl.haplotypes(rng, base, 20)
    del base
    rrng = wl.rng_for(8000 + rank)
    total = int(2_000_000_000 * args.scale)
    parts, lens, got = [], [], 0
    while got < total:
        long_read = rrng.random() < 0.1
        ln = int(min(100_000, max(31, rrng.lognormal(np.log(10_000), 0.5)))) if long_read else 150
        lens.append(ln)
        got += ln - 30
    lens = np.array(lens, dtype=np.int64)
    lens[-1] -= got - total
    rows = np.zeros(lens.size + 1, dtype=np.uint64)
    rows[1:] = np.cumsum(lens)
    letters = wl.ACGT[rrng.integers(0, 4, size=int(rows[-1]), dtype=np.uint8)]
    pos_rows = np.flatnonzero(rrng.random(lens.size) < 0.05)
    for r in pos_rows.tolist():  # 5% of reads copied from a haplotype
        h = haps[r % 20]
        a, b = int(rows[r]), int(rows[r + 1])
        if b - a <= h.size:
            s0 = int(rrng.integers(0, h.size - (b - a) + 1))
            letters[a:b] = h[s0:s0 + (b - a)]
    return haps, letters, rows


def workload_label(args):
    if args.scale == 1.0 and args.query_scale == 1.0:
        return WORKLOADS[args.workload]
    return f"{args.workload} x{args.scale}" + (f", queries x{args.query_scale}" if args.query_scale != 1.0 else "")


def workload(scale, rank, query_scale=1.0):
    from sbwt_gpu_b200 import workloads as wl
    rng = wl.rng_for(1236)
    n = int(100_000_000 * scale)
    genome = wl.random_bases(rng, n, gc=0.41)
    genome = wl.with_repeats(rng, genome, int(0.05 * n))
    rrng = wl.rng_for(7000 + rank)
    n_reads = max(10, int(10_000_000 * scale * query_scale))
    n_pos = n_reads // 10
    letters, rows = wl.mixed_reads(rrng, genome, n_pos, n_reads - n_pos, 150, 0.01)
    return genome, letters, rows


def measured_bf16():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["bf16_tflops"]), "measured (burst)"
    except Exception:
        return FALLBACK_BF16_TFLOPS, "fallback"


def measured_hbm():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class Clocks:
    """SM clock and clock-event (throttle) reasons of the benchmarked GPU, sampled every 10 ms by a
    host thread through NVML (read-only queries) during the timed region; nvidia-smi's 200 ms loop
    is too coarse for a timed region of tens of milliseconds."""

    def __init__(self, device_index):
        self.dev = device_index
        self.samples = []
        self.thread = None
        self.stop_flag = False

    def _handle(self, nv):
        import torch
        pr = torch.cuda.get_device_properties(self.dev)
        try:  # the GPU of this CUDA device, by PCI address (NVML numbers GPUs its own way)
            return nv.nvmlDeviceGetHandleByPciBusId(f"{pr.pci_domain_id:08x}:{pr.pci_bus_id:02x}:{pr.pci_device_id:02x}.0")
        except Exception:
            return nv.nvmlDeviceGetHandleByIndex(self.dev)

    def start(self):
        import threading
        try:
            import pynvml as nv
            nv.nvmlInit()
            h = self._handle(nv)
            smax = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        except Exception:
            return
        names = {"hw_slowdown": nv.nvmlClocksEventReasonHwSlowdown,
                 "hw_thermal_slowdown": nv.nvmlClocksEventReasonHwThermalSlowdown,
                 "sw_thermal_slowdown": nv.nvmlClocksEventReasonSwThermalSlowdown,
                 "sw_power_cap": nv.nvmlClocksEventReasonSwPowerCap}

        def run():
            while not self.stop_flag:
                try:
                    sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                    bits = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                    self.samples.append((sm, smax, [n for n, b in names.items() if bits & b]))
                except Exception:
                    pass
                time.sleep(0.01)

        self.thread = threading.Thread(target=run, daemon=True)
        self.thread.start()
        t0 = time.perf_counter()
        while not self.samples and time.perf_counter() - t0 < 2.0:  # sampling is live before timing starts
            time.sleep(0.001)

    def stop(self):
        if self.thread is None:
            return None
        self.stop_flag = True
        self.thread.join(timeout=2)
        if len(self.samples) > 1:
            self.samples = self.samples[1:]  # the first sample predates the timed region
        if not self.samples:
            return None
        return {"sm_mhz": statistics.median(x[0] for x in self.samples),
                "sm_max_mhz": max(x[1] for x in self.samples),
                "reasons": sorted({r for x in self.samples for r in x[2]}), "samples": len(self.samples),
                "source": "NVML every 10 ms"}


def cpu_reference(ox, letters, rows, k, p, budget_s, table):
    """The oracle port on a bounded prefix of the reads: (k-mers/s, answers, steps, rows used)."""
    import oracle as orc
    threads = orc.num_threads()
    # calibrate on a small prefix, then size the sample to the budget
    r0 = min(rows.size - 1, 2000)
    t = time.perf_counter()
    a0 = ox.search_reads(letters[: int(rows[r0])], rows[: r0 + 1], k, p, table)
    rate = a0.size / max(time.perf_counter() - t, 1e-6)
    per_row = max(a0.size / max(r0, 1), 1.0)
    want_kmers = rate * budget_s
    nr = int(min(rows.size - 1, max(r0, want_kmers / per_row)))
    sub_rows = rows[: nr + 1]
    sub_letters = letters[: int(sub_rows[-1])]
    t = time.perf_counter()
    ans, steps = ox.search_reads(sub_letters, sub_rows, k, p, table, want_steps=True)
    dt = time.perf_counter() - t
    return ans.size / dt, ans, steps, nr, threads


def walk_model(ans, steps, rows, k, p, stream, max_rows=20000):
    """How the run walk settles the k-mers of the first `max_rows` reads, from per-k-mer oracle answers
    and step counts (right to left per read; a search that fails after m letters settles k-m+1
    k-mers; with `stream`, the k-mer left of a found one takes a backward step): the share of k-mers
    searched from scratch, the share reached by a backward step, and the mean rank-pair steps of a
    search from scratch."""
    import oracle as orc
    searched = back = total = walk_steps = 0
    j0 = 0
    for r in range(min(rows.size - 1, max_rows)):
        n = int(rows[r + 1] - rows[r]) - k + 1
        if n <= 0:
            continue
        if j0 + n > ans.size:
            break
        j = j0 + n - 1
        have = False
        while j >= j0:
            hit = ans[j] != orc.NOT_FOUND
            if stream and have:
                back += 1
                have = hit
                j -= 1
            else:
                searched += 1
                walk_steps += int(steps[j])
                if hit:
                    have = True
                    j -= 1
                else:
                    j -= k - min(max(p, p + int(steps[j])), k) + 1
        j0 += n
        total += n
    return searched / max(total, 1), back / max(total, 1), walk_steps / max(searched, 1)


SECTOR = 32  # bytes: the unit in which L2 misses are filled from DRAM


def dram_model(n_kmers, n_letters, n_rows, searched, back, walk_steps, sizes, l2_bytes, answers=True):
    """Algorithmic DRAM bytes per k-mer of one launch of the run-walking search kernel.
    Compulsory streams: packed letters (2 bits per letter), the row table (row start + first k-mer
    index, 16 B per row), the u64 answers (8 B, written once) and the membership bitmap (1 bit).
    Gathers: one presearch entry per search from scratch, one backward-table entry per backward
    step, and two 32-byte lines per rank-pair step (one when the interval is a single node; two is
    the bound), each a 32-byte sector from DRAM when its table cannot stay in L2 (larger than half
    of it) and L2 traffic otherwise."""
    per = {
        "letters": n_letters / 4.0 / n_kmers,
        "row_table": 16.0 * n_rows / n_kmers,
        "answers": 8.0 if answers else 0.0,
        "bitmap": 0.125,
    }
    gathers = {
        "presearch": (searched, sizes["presearch"]),
        "backward_table": (back, sizes["backward_table"]),
        "lines": (searched * walk_steps * 2.0, sizes["lines"]),
    }
    l2 = {}
    for name, (count, table_bytes) in gathers.items():
        if table_bytes > l2_bytes / 2:
            per[name] = count * SECTOR
        else:
            l2[name] = count * SECTOR
    return sum(per.values()), per, l2


def max_over_ranks(x):
    """Max of a per-rank number over all ranks of the process group (device tensor under NCCL,
    host tensor under gloo)."""
    import torch
    import torch.distributed as dist
    dev = torch.device("cpu") if dist.get_backend() == "gloo" else torch.device("cuda", torch.cuda.current_device())
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def bits_of(ans):
    """Membership bitmap of answers: bit j%32 of word j/32 = answer j is not ~0."""
    import oracle as orc
    nk = ans.size
    b = np.zeros((nk + 31) // 32 * 32, dtype=bool)
    b[:nk] = ans != orc.NOT_FOUND
    return np.packbits(b.reshape(-1, 32)[:, ::-1], axis=1).view(">u4").reshape(-1).astype(np.uint32)


def kernel_traffic(kernel, workload, n_kmers):
    """DRAM bytes of one launch from the committed ncu summary, if it covers this kernel and workload."""
    tp = os.path.join(ROOT, "profiles", "search_kernel_traffic.json")
    try:
        for e in json.load(open(tp))["entries"]:
            if e["kernel"] == kernel and e["workload"] == workload:
                return float(e["dram_bytes_per_kmer"]) * n_kmers, e
    except (OSError, ValueError, KeyError, TypeError):
        pass
    return None, None


def table_sizes(n_columns, p, stream_tables=True):
    """Bytes of the index structures the run walk gathers from: presearch table (8-byte entries below
    2^32 columns), backward table (8 bytes per column) and the 32-byte lines of the four vectors."""
    lpc = (n_columns // 224 + 1 + 7) // 8 * 8
    return {"presearch": (1 << (2 * p)) * (8 if n_columns < (1 << 32) else 16) if p else 0,
            "backward_table": 8 * n_columns if stream_tables else 0,
            "lines": 4 * lpc * 32}


def roofline(kernel, kern_ms, n_kmers, n_letters, n_rows, n_columns, p, searched, back, walk_steps, mean_steps,
             p_steps, dev, peak, peak_kind, traffic_workload, stream_tables=True, answers=True):
    """The `roofline` object of the dominant kernel: walk-aware algorithmic DRAM bytes (dram_model)
    over the kernel's CUDA-event time, against the measured copy bandwidth; the measured DRAM traffic
    of the same kernel (ncu, committed summary) beside it; and the reference's per-k-mer step model
    under its own name."""
    import torch
    l2_bytes = torch.cuda.get_device_properties(dev).L2_cache_size
    sizes = table_sizes(n_columns, p, stream_tables)
    b_kmer, parts, l2 = dram_model(n_kmers, n_letters, n_rows, searched, back, walk_steps, sizes, l2_bytes, answers)
    secs = kern_ms / 1e3
    achieved = n_kmers * b_kmer / secs / 1e9
    traffic, tr = kernel_traffic(kernel, traffic_workload, n_kmers)
    ref_b = 128.0 * mean_steps + 16 + 8 + n_letters / 4.0 / n_kmers
    return {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": traffic, "peak_kind": f"of {peak_kind}", "kernel": kernel, "kernel_ms": kern_ms,
            "units_per_launch": n_kmers, "bytes_per_kmer": b_kmer,
            "bytes_per_kmer_parts": {kk: round(vv, 4) for kk, vv in parts.items()},
            "l2_bytes_per_kmer": {kk: round(vv, 4) for kk, vv in l2.items()},
            "table_bytes": sizes, "l2_cache_bytes": l2_bytes,
            "searched_fraction": searched, "backward_step_fraction": back,
            "steps_per_search": walk_steps, "steps_counted_at_p": p_steps,
            "traffic_per_kmer": traffic / n_kmers if traffic else None,
            "traffic_over_model": traffic / (n_kmers * b_kmer) if traffic else None,
            "dram_frac": (traffic / secs / 1e9 / peak) if traffic else None,
            "traffic_source": tr["source"] if tr else None,
            "reference_step_model": {
                "bytes_per_kmer": ref_b, "mean_steps": mean_steps, "equivalent_GBps": n_kmers * ref_b / secs / 1e9,
                "note": "the reference's work per k-mer (every k-mer searched, one 128-byte line per step, "
                        "presearch entry, answer); the walk skips most of it, so this is a speed-up figure, "
                        "not DRAM use"}}


def host_threads_per_rank(world, impl):
    """torchrun gives every rank OMP_NUM_THREADS=1 unless it is set; the host threads (answer
    expansion, the CPU arms) get their share of the cores instead: all of them for the reference
    arm (rank 0 alone runs), cores / ranks on this node for this project's arm.  Must run before
    the first OpenMP runtime starts in this process."""
    if world <= 1 or os.environ.get("OMP_NUM_THREADS", "") not in ("", "1"):
        return
    cores = len(os.sched_getaffinity(0))
    local = int(os.environ.get("LOCAL_WORLD_SIZE", str(world)))
    os.environ["OMP_NUM_THREADS"] = str(cores if impl == "reference" else max(1, cores // max(local, 1)))


def open_index(sg, seqs, k, p, args, rank, world, local_rank, tag, **kw):
    """The index of a workload: rank 0 builds the SBWT on the GPU and writes the reference's four files;
    every rank loads them.  Returns (index, paths, build seconds, load seconds)."""
    import torch.distributed as dist
    tmpdir = os.environ.get("SBWT_BENCH_DIR") or os.path.join(tempfile.gettempdir(), f"sbwt_bench_{os.getppid()}")
    os.makedirs(tmpdir, exist_ok=True)
    prefix = os.path.join(tmpdir, tag)
    build_s = None
    if rank == 0:
        t = time.perf_counter()
        built = sg.build_sbwt([x.tobytes() for x in seqs], k, device=local_rank)  # the GPU builder
        build_s = time.perf_counter() - t
        sg.write_index_files(prefix, built)
        del built
    if world > 1:
        dist.barrier()
    paths = [f"{prefix}.{c}" for c in "ACGT"]
    t = time.perf_counter()
    ix = sg.Index.load(*paths, k=k, k_presearch=p, device=local_rank, **kw)
    return ix, paths, build_s, time.perf_counter() - t


def timed_search(ix, step, steps, warmup, dev, stream, world=1):
    """Device time of `steps` calls of `step` after `warmup` untimed ones (CUDA events on the launching
    stream, synchronize and barrier on both sides; max over ranks), with the CUDA graph of the
    pack -> k-mer table -> search chain replayed; then a few profiled calls for the per-kernel split.
    Returns (total ms, search-kernel ms per call, our kernel launches per call, clocks)."""
    import torch
    import torch.distributed as dist
    ix.profile(False)
    ix.use_graphs(True)
    for _ in range(max(warmup, 0)):
        step()
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    clocks = Clocks(dev.index if dev.index is not None else 0)
    clocks.start()
    torch.cuda.synchronize(dev)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(steps):
        step()
    ev1.record(stream)
    torch.cuda.synchronize(dev)
    total_ms = ev0.elapsed_time(ev1)
    clk = clocks.stop()
    if world > 1:
        dist.barrier()
        total_ms = max_over_ranks(total_ms)
    # per-kernel split: profiled calls (the graph is not used while profiling)
    ix.profile(True)
    search_ms, launches = [], 0
    for _ in range(min(max(steps, 1), 5)):
        step()
        prof = ix.last_profile()
        search_ms.append(prof["search_ms"])
        launches = prof["launches"]
    ix.profile(False)
    return total_ms, statistics.mean(search_ms), launches, clk


def oracle_check(orc, paths, letters, rows, k, p, seconds, got_fn, stream_mode, runs_form):
    """Answers of a bounded prefix of the batch from the oracle (C restatement of the reference search), compared
    with the device answers; the walk model of the run walk from the same sample."""
    ox = orc.OracleIndex.from_files(paths)
    p_cpu = min(p, 12)  # answers do not depend on p; a CPU table beyond 4^12 entries costs minutes
    table = ox.presearch(p_cpu) if p_cpu else None
    rate, ans, steps, nr, threads = cpu_reference(ox, letters, rows, k, p_cpu, seconds, table)
    got = got_fn(ans.size)
    if not np.array_equal(got, ans):
        raise SystemExit(f"bench: {int((got != ans).sum())} of {ans.size} sampled answers differ from the oracle")
    mean_steps = float(steps.mean())
    searched, back, walk_steps = (walk_model(ans, steps, rows, k, p_cpu, stream_mode) if runs_form
                                  else (1.0, 0.0, mean_steps))
    return {"rate": rate, "ans": ans, "nr": nr, "threads": threads, "p_cpu": p_cpu, "mean_steps": mean_steps,
            "searched": searched, "back": back, "walk_steps": walk_steps}


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    k = 31
    host_threads_per_rank(world, args.impl)

    if args.impl == "reference":
        if rank != 0:
            return 0
        return reference_arm(args, k)

    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=dev)

    import sbwt_gpu_b200 as sg
    import oracle as orc

    seqs, letters, rows, p = workload_of(args, rank)
    n_kmers = sg.count_kmers(rows, k)
    layout = {"lines": sg.SBWT_LAYOUT_LINES, "poppy": sg.SBWT_LAYOUT_POPPY, "lines512": sg.SBWT_LAYOUT_LINES512,
              "lines2048": sg.SBWT_LAYOUT_LINES2048}[args.layout]
    ix, paths, build_s, load_s = open_index(
        sg, seqs, k, p, args, rank, world, local_rank, "ix", layout=layout, bits_in_superblock=args.sb,
        kmers_per_thread=args.kpt, threads_per_kmer=args.tpk, threads_per_block=args.tpb,
        search_mode=MODES[args.search_mode])
    del seqs
    runs_form = args.kpt == 0 and args.search_mode != "every" and (args.tpk <= 1 or args.layout == "poppy")
    kernel = ("search_runs_kernel" + ("<stream>" if args.search_mode == "stream" else "<skip>") if runs_form
              else ("search_queue_kernel" if args.kpt == 0 else "search_kernel"))
    if args.l2_fetch:
        ix.set_l2_fetch_granularity(args.l2_fetch)
    if args.window or args.evict >= 0 or args.l2_persist >= 0 or args.blocks_per_sm:
        ix.set_walk_options(window=args.window or None, evict=args.evict if args.evict >= 0 else None,
                            l2_persist=args.l2_persist if args.l2_persist >= 0 else None,
                            blocks_per_sm=args.blocks_per_sm or None)
    build_times = ix.build_times()  # device ms: rank words (lines), poppy, presearch, backward table
    info = ix.info()

    d_letters = torch.from_numpy(letters).to(dev)
    d_rows = torch.from_numpy(rows.view(np.int64)).to(dev)
    d_ans = torch.empty(n_kmers, dtype=torch.int64, device=dev)
    d_mem = torch.empty((n_kmers + 31) // 32, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev)

    def step():
        ix.search_reads(d_letters, d_rows, d_ans, n_kmers, d_member_bits=d_mem, stream=stream)

    total_ms, kern_ms, launches_per_step, clk = timed_search(ix, step, args.steps, args.warmup, dev, stream, world)
    value = n_kmers * world * args.steps / (total_ms / 1e3)

    def got_u64(n):
        return d_ans[:n].cpu().numpy().view(np.uint64)

    # ---- correctness on a sample + the CPU baseline (rank 0 only, untimed)
    cpu = chk = None
    if rank == 0:
        chk = oracle_check(orc, paths, letters, rows, k, p, args.cpu_seconds, got_u64, args.search_mode == "stream",
                           runs_form)
        cpu = {"value": chk["rate"], "unit": UNIT, "cores": chk["threads"], "kind": "port",
               "sample": f"first {chk['nr']} reads ({chk['ans'].size} k-mers) of the same batch, C restatement of "
                         f"the reference search (the reference has no CPU search), OpenMP schedule(dynamic,4096)"}
    ans = chk["ans"] if chk else None

    # ---- end to end through the host entry point (pinned buffers)
    e2e = None
    if not args.no_e2e:
        e2e = e2e_leg(args, ix, letters, rows, n_kmers, d_ans, ans, dev, world, rank)

    extra = rank == 0 and world == 1  # legs for the record, on one GPU only
    per_kmer = member_only = contract = tuned = None
    if extra and runs_form and not args.no_per_kmer:
        # the same batch with every k-mer searched (the reference's per-k-mer work), for comparison
        ix.set_search_mode(sg.SEARCH_EVERY_KMER)
        tt, km, _, _ = timed_search(ix, step, args.steps, 2, dev, stream)
        ix.set_search_mode(MODES[args.search_mode])
        if not np.array_equal(got_u64(ans.size), ans):
            raise SystemExit("bench: per-k-mer answers differ from the oracle")
        per_kmer = {"value": n_kmers * args.steps / (tt / 1e3), "ms_per_step": tt / args.steps,
                    "search_kernel_ms": km, "kernel": "search_queue_kernel"}
    if extra and runs_form:
        # membership only on the device: no answer array, the kernel writes the bitmap alone
        d_mem2 = torch.zeros_like(d_mem)

        def mstep():
            ix.search_reads(d_letters, d_rows, None, n_kmers, d_member_bits=d_mem2, stream=stream)

        tt, km, _, _ = timed_search(ix, mstep, args.steps, 2, dev, stream)
        full = ans.size // 32
        if not np.array_equal(d_mem2[:full].cpu().numpy().view(np.uint32), bits_of(ans)[:full]):
            raise SystemExit("bench: membership bits differ from the oracle")
        member_only = {"value": n_kmers * args.steps / (tt / 1e3), "ms_per_step": tt / args.steps,
                       "search_kernel_ms": km, "output": "membership bitmap only (no answers)",
                       "roofline": roofline(kernel, km, n_kmers, letters.size, rows.size - 1, info["n_bits"], p,
                                            chk["searched"], chk["back"], chk["walk_steps"], chk["mean_steps"],
                                            chk["p_cpu"], dev, *measured_hbm(), None,
                                            stream_tables=args.search_mode == "stream", answers=False)}
        del d_mem2
    if extra and not args.no_contract:
        contract = contract_leg(sg, ix, letters, rows, d_letters, d_rows, n_kmers, k, ans, args.steps, dev, stream)
    if extra and not args.no_autotune:
        tuned = autotune_leg(ix, letters, rows, d_ans, n_kmers, k, step, ans, args.steps, dev, stream)

    if rank == 0:
        peak, peak_kind = measured_hbm()
        roof = roofline(kernel, kern_ms, n_kmers, letters.size, rows.size - 1, info["n_bits"], p, chk["searched"],
                        chk["back"], chk["walk_steps"], chk["mean_steps"], chk["p_cpu"], dev, peak, peak_kind,
                        args.workload if args.scale == 1.0 and args.query_scale == 1.0 else None,
                        stream_tables=args.search_mode == "stream")
        hits = int((d_ans.cpu().numpy().view(np.uint64) != orc.NOT_FOUND).sum())
    # free the headline batch before the other workloads
    del d_letters, d_rows, d_ans, d_mem
    ix.close()
    torch.cuda.empty_cache()

    workloads = prefilter = None
    if extra and not args.no_workloads and args.workload == "large":
        workloads, prefilter = other_workloads(args, sg, orc, k, dev, stream, rank, world, local_rank)
    elif extra and not args.no_prefilter:
        prefilter = {"flat": prefilter_flat_leg(args, dev, k)}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic (seeded)",
            "config": {
                "workload": workload_label(args),
                "n_kmers_per_gpu": n_kmers, "n_columns": info["n_bits"], "k": k, "p": p,
                "layout": args.layout, "present_kmers": hits, "l2_fetch_bytes": args.l2_fetch or "default",
                "l2": "inputs and outputs larger than L2 (letters %.2f GB, answers %.2f GB); no flush" % (
                    letters.nbytes / 1e9, n_kmers * 8 / 1e9),
                "parallelism": f"replicas x{world}" if world > 1 else "1 GPU",
                "cuda_graph": "pack -> k-mer table -> search chain captured once, replayed every timed step",
                "index_build_s": round(build_s, 2), "index_builder": "gpu (sbwt_build_gpu, incl. host copies)",
                "index_load_s": round(load_s, 2),
                "index_build_device_ms": {kk: round(vv, 3) for kk, vv in build_times.items()},
            },
            "roofline": roof,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": launches_per_step * args.steps,
            "clocks": clk,
            "per_kmer": per_kmer,
            "membership_only": member_only,
            "kernel_contract": contract,
            "autotuned": tuned,
            "workloads": workloads,
            "prefilter": prefilter,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def e2e_leg(args, ix, letters, rows, n_kmers, d_ans, ans, dev, world, rank):
    """`e2e`: the same batch through sbwt_search_reads_host (the public host-buffer entry point): letters and row
    starts host -> device and the answers back into pinned host memory, every step, host wall clock around the
    synchronous calls (max over ranks); membership only beside it."""
    import torch
    import torch.distributed as dist
    h_letters = torch.from_numpy(letters).pin_memory()
    h_rows = torch.from_numpy(rows.view(np.int64)).pin_memory()
    h_ans = torch.empty(n_kmers, dtype=torch.int64).pin_memory()
    ix.profile(False)
    ix.search_reads_host(h_letters, h_rows, h_ans)  # warm-up
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    t = time.perf_counter()
    for _ in range(args.e2e_steps):
        ix.search_reads_host(h_letters, h_rows, h_ans)
    e2e_s = time.perf_counter() - t
    if world > 1:
        e2e_s = max_over_ranks(e2e_s)
    if rank == 0 and not np.array_equal(h_ans[: ans.size].numpy().view(np.uint64), ans):
        raise SystemExit("bench: end-to-end answers differ from the oracle")
    if not torch.equal(h_ans.to(dev), d_ans):  # every answer against the device search's
        raise SystemExit("bench: end-to-end answers differ from the device search's")
    moved = ix.pipeline_bytes()
    mode = os.environ.get("SBWT_PIPELINE_TRANSFER", "") or "auto"
    e2e = {"value": n_kmers * world * args.e2e_steps / e2e_s, "unit": UNIT,
           "h2d_bytes_per_step": int(moved["h2d"]), "d2h_bytes_per_step": int(moved["d2h"]),
           "answer_bytes_per_step": int(n_kmers * 8), "steps": args.e2e_steps,
           "host_threads": int(os.environ.get("OMP_NUM_THREADS", "0")) or len(os.sched_getaffinity(0)),
           "transfer": mode + (": u64 answers" if moved["d2h"] >= n_kmers * 8 else
                               ": bitmap + found node ids (some chunks as u64 answers), expanded by the host threads")}
    del h_ans
    n_words = (n_kmers + 31) // 32
    h_mem = torch.empty(n_words, dtype=torch.int32).pin_memory()
    ix.member_reads_host(h_letters, h_rows, h_mem)  # warm-up
    if world > 1:
        dist.barrier()
    t = time.perf_counter()
    for _ in range(args.e2e_steps):
        ix.member_reads_host(h_letters, h_rows, h_mem)
    m_s = time.perf_counter() - t
    if world > 1:
        m_s = max_over_ranks(m_s)
    if rank == 0:
        full = ans.size // 32
        if not np.array_equal(h_mem[:full].numpy().view(np.uint32), bits_of(ans)[:full]):
            raise SystemExit("bench: end-to-end membership bits differ from the oracle")
    moved = ix.pipeline_bytes()
    e2e["membership_only"] = {"value": n_kmers * world * args.e2e_steps / m_s, "unit": UNIT,
                              "h2d_bytes_per_step": int(moved["h2d"]), "d2h_bytes_per_step": int(moved["d2h"]),
                              "entry_point": "sbwt_search_reads_host_member"}
    return e2e


def contract_leg(sg, ix, letters, rows, d_letters, d_rows, n_kmers, k, ans, steps, dev, stream):
    """The reference's kernel contract (sbwt_search_packed): packed letters + the reference's positions array
    (k-mer j of read r at row_start[r] + i), answers written over the positions."""
    import torch
    lens = torch.from_numpy(np.diff(rows.astype(np.int64))).to(dev)
    cnt = torch.clamp(lens - (k - 1), min=0)
    rs = d_rows[:-1]
    ks = torch.cumsum(cnt, 0) - cnt  # first k-mer index of each row
    d_pos0 = torch.arange(n_kmers, dtype=torch.int64, device=dev) + torch.repeat_interleave(rs - ks, cnt)
    n_words = (letters.size + 32 + 31) // 32
    d_words = torch.empty(n_words, dtype=torch.int64, device=dev)
    sg._lib.lib.sbwt_pack(sg._ptr(d_letters), letters.size, sg._ptr(d_words), sg._stream_ptr(stream))
    d_pos = torch.empty_like(d_pos0)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    c_ms = []
    for it in range(2 + steps):
        d_pos.copy_(d_pos0)
        torch.cuda.synchronize(dev)
        e0.record(stream)
        ix.search_packed(d_words, d_pos, stream=stream)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        if it >= 2:
            c_ms.append(e0.elapsed_time(e1))
    if not np.array_equal(d_pos[: ans.size].cpu().numpy().view(np.uint64), ans):
        raise SystemExit("bench: kernel-contract answers differ from the oracle")
    cm = statistics.mean(c_ms)
    return {"value": n_kmers / (cm / 1e3), "ms_per_call": cm, "entry_point": "sbwt_search_packed",
            "note": "positions array in, answers out in place, as the reference's search kernel"}


def autotune_leg(ix, letters, rows, d_ans, n_kmers, k, step, ans, steps, dev, stream):
    """The tuner picks the run walk's knobs and the presearch depth on a sample, then the batch is timed again."""
    import torch
    import sbwt_gpu_b200 as sg
    ns = min(rows.size - 1, 3_000_000)  # 360M k-mers of the large batch: choices that carry over to the whole batch
    nk_s = sg.count_kmers(rows[: ns + 1], k)
    d_ls = torch.from_numpy(letters[: int(rows[ns])]).to(dev)
    d_rs = torch.from_numpy(rows[: ns + 1].view(np.int64)).to(dev)
    rep = ix.autotune(d_ls, d_rs, d_ans, nk_s, tune_p=True, tune_poppy=True)
    del d_ls, d_rs
    tt, km, _, _ = timed_search(ix, step, steps, 2, dev, stream)
    if not np.array_equal(d_ans[: ans.size].cpu().numpy().view(np.uint64), ans):
        raise SystemExit("bench: autotuned answers differ from the oracle")
    return {"value": n_kmers * steps / (tt / 1e3), "ms_per_step": tt / steps, "search_kernel_ms": km,
            "choice": rep["best"], "candidates": len(rep["candidates"]), "tuned_on_kmers": nk_s,
            "default_ms_on_sample": rep.get("default_ms"), "report": rep.get("candidates")}


def device_leg(ix, sg, orc, paths, letters, rows, k, p, steps, warmup, dev, stream, kernel, workload_key, cpu_s,
               label):
    """One workload on the device as the headline is measured (answers + bitmap, CUDA graph, CUDA events),
    checked against the oracle on a bounded prefix, with its roofline."""
    import torch
    n_kmers = sg.count_kmers(rows, k)
    d_letters = torch.from_numpy(letters).to(dev)
    d_rows = torch.from_numpy(rows.view(np.int64)).to(dev)
    d_ans = torch.empty(n_kmers, dtype=torch.int64, device=dev)
    d_mem = torch.empty((n_kmers + 31) // 32, dtype=torch.int32, device=dev)

    def step():
        ix.search_reads(d_letters, d_rows, d_ans, n_kmers, d_member_bits=d_mem, stream=stream)

    total_ms, km, launches, clk = timed_search(ix, step, steps, warmup, dev, stream)
    chk = oracle_check(orc, paths, letters, rows, k, p, cpu_s, lambda n: d_ans[:n].cpu().numpy().view(np.uint64),
                       True, True)
    full = chk["ans"].size // 32
    if not np.array_equal(d_mem[:full].cpu().numpy().view(np.uint32), bits_of(chk["ans"])[:full]):
        raise SystemExit(f"bench: {label}: membership bits differ from the oracle")
    peak, peak_kind = measured_hbm()
    info = ix.info()
    res = {"workload": label, "value": n_kmers * steps / (total_ms / 1e3), "unit": UNIT, "steps": steps,
           "ms_per_step": total_ms / steps, "n_kmers": n_kmers, "n_columns": info["n_bits"], "p": p,
           "present_kmers": int((d_ans.cpu().numpy().view(np.uint64) != orc.NOT_FOUND).sum()),
           "bit_exact_sample": {"kmers": int(chk["ans"].size), "equal": True},
           "gpu_launches": launches * steps, "clocks": clk,
           "roofline": roofline(kernel, km, n_kmers, letters.size, rows.size - 1, info["n_bits"], p, chk["searched"],
                                chk["back"], chk["walk_steps"], chk["mean_steps"], chk["p_cpu"], dev, peak,
                                peak_kind, workload_key)}
    del d_letters, d_rows, d_ans, d_mem
    torch.cuda.empty_cache()
    return res


def filtered_leg(ix, pf, sg, letters, rows, k, steps, dev, stream, plain_value, label, ans_sample):
    """The same batch of reads behind the learned prefilter (sbwt_search_reads_filtered): k-mers/s against the
    plain search's, the skip rate, false-absent count and equality with the oracle's answers on the sample."""
    import torch
    n_kmers = sg.count_kmers(rows, k)
    d_letters = torch.from_numpy(letters).to(dev)
    d_rows = torch.from_numpy(rows.view(np.int64)).to(dev)
    d_ans = torch.empty(n_kmers, dtype=torch.int64, device=dev)
    d_plain = torch.empty(n_kmers, dtype=torch.int64, device=dev)
    ix.search_reads(d_letters, d_rows, d_plain, n_kmers, stream=stream)
    for _ in range(2):
        skipped = ix.search_reads_filtered(pf, d_letters, d_rows, d_ans, n_kmers, stream=stream)
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        ix.search_reads_filtered(pf, d_letters, d_rows, d_ans, n_kmers, stream=stream, count_skipped=False)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1) / steps
    nf = np.uint64(0xFFFFFFFFFFFFFFFF)
    false_absent = int(((d_plain != -1) & (d_ans == -1)).sum().item())
    equal = bool(torch.equal(d_plain, d_ans))
    sample_equal = bool(np.array_equal(d_ans[: ans_sample.size].cpu().numpy().view(np.uint64), ans_sample))
    if not (equal and sample_equal and false_absent == 0):
        raise SystemExit(f"bench: {label}: prefiltered answers differ (false-absent {false_absent})")
    value = n_kmers / (ms / 1e3)
    negatives = int((d_plain == -1).sum().item())
    # the model alone on the first 4M letters' k-mers: the share it rejects among absent and present ones
    import oracle as orc
    ns = int(np.searchsorted(rows, min(int(rows[-1]), 4_000_000)))
    sk = orc.extract_kmers(letters[: int(rows[ns])], rows[: ns + 1], k)
    d_sk = torch.from_numpy(sk.view(np.int64)).to(dev)
    d_lg = torch.empty(d_sk.numel(), dtype=torch.float32, device=dev)
    pf.logits(d_sk, d_lg)
    absent = (d_plain[: d_sk.numel()] == -1)
    rej = d_lg < 0.0  # the default threshold tau = 0 the prefilters here are trained with
    model_reject_absent = float((rej & absent).sum().item()) / max(int(absent.sum().item()), 1)
    model_reject_present = float((rej & ~absent).sum().item()) / max(int((~absent).sum().item()), 1)
    del d_letters, d_rows, d_ans, d_plain, d_sk, d_lg
    torch.cuda.empty_cache()
    return {"workload": label, "plain_kmers_per_s": plain_value, "prefiltered_kmers_per_s": value,
            "model_reject_rate_absent": model_reject_absent, "model_reject_rate_present": model_reject_present,
            "speedup": value / plain_value, "target_speedup": 1.5, "ms_per_call": ms, "skip_rate": skipped / n_kmers,
            "negative_fraction": negatives / n_kmers, "false_absent": false_absent, "bit_exact": equal,
            "entry_point": "sbwt_search_reads_filtered", "n_kmers": n_kmers, "stats": pf.stats()}


def train_prefilter(sg, ix, args):
    t = time.perf_counter()
    pf = sg.Prefilter.train(ix, steps=args.pf_steps, batch=8192, n_positive=50_000_000, n_negative=50_000_000,
                            seed=4)
    return pf, time.perf_counter() - t


def other_workloads(args, sg, orc, k, dev, stream, rank, world, local_rank):
    """Beside the headline (one GPU): the batched-uneven and pangenome workloads measured like it, and the
    learned prefilter on the small index (single k-mers and reads) and on the pangenome index (retrained)."""
    from sbwt_gpu_b200 import workloads as wl
    steps = max(1, min(args.steps, args.workload_steps))
    out, pf_out = {}, {}
    # ---- batched: index of the small workload, 64 query files of uneven reads, one persistent launch
    small = wl.small_workload(seed=1235)["genome"]
    letters, rows = batched_queries(args, rank)
    ix, paths, _, _ = open_index(sg, [small], k, 10, args, rank, 1, local_rank, "small",
                                 search_mode=sg.SEARCH_STREAM)
    kern = "search_runs_kernel<stream>"
    out["batched"] = device_leg(ix, sg, orc, paths, letters, rows, k, 10, steps, 2, dev, stream, kern,
                                "batched" if args.scale == 1.0 else None, min(args.cpu_seconds, 4.0),
                                WORKLOADS["batched"])
    del letters, rows
    if not args.no_prefilter:
        pf, train_s = train_prefilter(sg, ix, args)
        flat = prefilter_flat_leg(args, dev, k, ix, pf, small)
        flat["train_s"] = round(train_s, 2)
        pf_out["flat"] = flat
        # the reads form on the same index: 150 bp reads, 10% genome-sampled with 1% substitutions, 90% random
        rrng = wl.rng_for(4343)
        n_reads = max(10, int(args.pf_queries * args.scale) // 120)
        letters, rows = wl.mixed_reads(rrng, small, n_reads // 10, n_reads - n_reads // 10, 150, 0.01)
        plain = device_leg(ix, sg, orc, paths, letters, rows, k, 10, steps, 2, dev, stream, kern, None,
                           min(args.cpu_seconds, 2.0), "prefilter reads (small index)")
        ns = min(2000, rows.size - 1)  # oracle sample: the first 2000 reads, or all of a small batch
        ox_ans = orc.OracleIndex.from_files(paths).search_reads(letters[: int(rows[ns])], rows[: ns + 1], k, 10)
        pf_out["batched"] = filtered_leg(ix, pf, sg, letters, rows, k, steps, dev, stream, plain["value"],
                                         f"small index (1 Mbp, k=31, p=10); {n_reads} reads x 150 bp "
                                         "(10% genome-sampled with 1% subs, 90% uniform random)", ox_ans)
        pf.close()
        del letters, rows
    ix.close()
    # ---- pangenome: 20 haplotypes of a 50 Mbp base, 2G k-mers in one persistent launch, p = 14
    haps, letters, rows = pangenome_workload(args, rank)
    ix, paths, build_s, _ = open_index(sg, haps, k, 14, args, rank, 1, local_rank, "pan",
                                       search_mode=sg.SEARCH_STREAM)
    del haps
    out["pangenome"] = device_leg(ix, sg, orc, paths, letters, rows, k, 14, steps, 2, dev, stream, kern,
                                  "pangenome" if args.scale == 1.0 else None, min(args.cpu_seconds, 4.0),
                                  WORKLOADS["pangenome"])
    out["pangenome"]["index_build_s"] = round(build_s, 2)
    if not args.no_prefilter:
        pf, train_s = train_prefilter(sg, ix, args)  # retrained on this index
        ox_ans = orc.OracleIndex.from_files(paths).search_reads(letters[: int(rows[500])], rows[:501], k, 12)
        res = filtered_leg(ix, pf, sg, letters, rows, k, steps, dev, stream, out["pangenome"]["value"],
                           WORKLOADS["pangenome"] + "; prefilter retrained on this index", ox_ans)
        res["train_s"] = round(train_s, 2)
        pf_out["pangenome"] = res
        pf.close()
    ix.close()
    return out, (pf_out or None)


def prefilter_flat_leg(args, dev, k, pix=None, pf=None, genome=None):
    """Plain vs learned-prefiltered search of 200M single k-mers (90% negatives: half uniform random, half
    indexed k-mers with 1-3 substitutions) against the index of the small workload (1 Mbp uniform genome,
    p = 10); the MLP is trained on the GPU (20k Adam steps, batch 8192, 5e7 + 5e7 candidates) unless an index
    and a prefilter trained on it are given."""
    import torch
    import sbwt_gpu_b200 as sg
    from sbwt_gpu_b200 import workloads as wl
    own = pix is None
    train_s = None
    if own:
        genome = wl.small_workload(seed=1235)["genome"]
        built = sg.build_sbwt([genome.tobytes()], k)
        pix = sg.Index.from_bits(built.bits, built.n_bits, k=k, k_presearch=10)
        pf, train_s = train_prefilter(sg, pix, args)
    st = pf.stats()
    kmers = wl.kmer_query_words(wl.rng_for(4242), genome, int(args.pf_queries * args.scale), k, neg_frac=0.9)
    d_k = torch.from_numpy(kmers.view(np.int64)).to(dev)
    del kmers
    plain = torch.empty_like(d_k)
    filt = torch.empty_like(d_k)
    d_l = torch.empty(d_k.numel(), dtype=torch.float32, device=dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(fn, reps):
        for _ in range(2):
            fn()
        torch.cuda.synchronize(dev)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize(dev)
        return e0.elapsed_time(e1) / reps

    n = d_k.numel()
    reps = max(min(args.steps, 5), 3)
    ms_plain = timed(lambda: pix.search_kmers(d_k, plain), reps)
    ms_logits = timed(lambda: pf.logits(d_k, d_l), reps)
    ms_filt = timed(lambda: pix.search_kmers_filtered(pf, d_k, filt), reps)
    skipped = pix.search_kmers_filtered(pf, d_k, filt)
    torch.cuda.synchronize(dev)
    p_np, f_np = plain.cpu().numpy().view(np.uint64), filt.cpu().numpy().view(np.uint64)
    nf = 0xFFFFFFFFFFFFFFFF
    false_absent = int(((p_np != nf) & (f_np == nf)).sum())
    if false_absent or not np.array_equal(p_np, f_np):
        raise SystemExit(f"bench: prefiltered k-mer answers differ (false-absent {false_absent})")
    res = {
        "workload": "prefilter: index of the small workload (1 Mbp uniform genome, k=31, p=10); "
                    f"{n} single k-mers, 90% negatives (half uniform random, half 1-3 substitutions)",
        "plain_kmers_per_s": n / (ms_plain / 1e3), "prefiltered_kmers_per_s": n / (ms_filt / 1e3),
        "speedup": ms_plain / ms_filt, "target_speedup": 1.5, "mlp_kmers_per_s": n / (ms_logits / 1e3),
        "mlp_tflops": n * 2 * (128 * 256 + 256 * 256 + 256) / (ms_logits / 1e3) / 1e12,
        "mlp_tensor_frac": (n * 2 * (128 * 256 + 256 * 256 + 256) / (ms_logits / 1e3) / 1e12) / measured_bf16()[0],
        "mlp_tensor_peak_kind": "of " + measured_bf16()[1],
        "skip_rate": skipped / n, "false_absent": false_absent, "bit_exact": True,
        "present": int((p_np != nf).sum()), "train": st,
    }
    if train_s is not None:
        res["train_s"] = round(train_s, 2)
    del d_k, plain, filt, d_l
    if own:
        pf.close()
        pix.close()
    torch.cuda.empty_cache()
    return res


def reference_arm(args, k):
    """The reference's search on this box: its CPU semantics through the oracle's C restatement (the
    reference has no CPU search) on all host threads, a bounded sample of the batch per step; and, as
    `reference_gpu`, the reference's own CUDA search kernel (its program built for sm_100a, oracle/_ref/search)
    on a 10% sample of the large workload, from the kernel time it prints itself."""
    import oracle as orc
    import sbwt_gpu_b200 as sg
    seqs, letters, rows, p = workload_of(args, 0)
    built = sg.build_sbwt([x.tobytes() for x in seqs], k)
    ox = orc.OracleIndex(built.bits, built.n_bits)
    p_cpu = min(p, 12)  # answers do not depend on p; a CPU table beyond 4^12 entries costs minutes
    table = ox.presearch(p_cpu) if p_cpu else None
    # each step: a bounded sample of the batch sized to ~budget seconds
    budget = max(1.0, min(args.cpu_seconds, 150.0 / max(args.steps + args.warmup, 1)))
    rate, ans, steps, nr, threads = cpu_reference(ox, letters, rows, k, p_cpu, budget, table)
    sub_rows = rows[: nr + 1]
    sub_letters = letters[: int(sub_rows[-1])]
    for _ in range(max(args.warmup - 1, 0)):
        ox.search_reads(sub_letters, sub_rows, k, p_cpu, table)
    t = time.perf_counter()
    for _ in range(args.steps):
        ox.search_reads(sub_letters, sub_rows, k, p_cpu, table)
    dt = time.perf_counter() - t
    value = ans.size * args.steps / dt
    sample = (f"first {nr} reads ({ans.size} k-mers) per step of the {args.workload} workload; C restatement of "
              f"the reference search (the reference has no CPU search), OpenMP, {threads} threads")
    ref_gpu = reference_gpu(args, built, letters, rows, k, p) if args.workload == "large" else None
    del built
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3 / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic (seeded)",
        "config": {"workload": workload_label(args), "k": k, "p": p_cpu},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "reference_gpu": ref_gpu,
    }
    print(json.dumps(line), flush=True)
    return 0


def reference_gpu(args, built, letters, rows, k, p, frac=0.1):
    """The reference's own CUDA search kernel on the first 10% of the reads (1M reads, 120M k-mers) and the
    same index, from its printed "Search in GPU" time; inputs checked against its in-bounds conditions first."""
    import ref_program as rp
    import sbwt_gpu_b200 as sg
    from sbwt_gpu_b200 import workloads as wl
    if not rp.available():
        return {"unavailable": "the reference program was not built here (oracle/_ref/search)"}
    import torch
    if not torch.cuda.is_available():
        return {"unavailable": "no GPU visible to this process"}
    nr = max(8, int((rows.size - 1) * frac * args.scale) // 8 * 8)
    sub_rows = rows[: nr + 1]
    sub_letters = letters[: int(sub_rows[-1])]
    p_ref = min(p, 13)  # the reference caps p at 13 (include/parameters.hpp:255-258)
    try:
        rp.check_safe(built.n_bits, sub_letters, sub_rows, k, p_ref)
    except AssertionError as e:
        return {"unavailable": f"inputs outside the reference's in-bounds conditions: {e}"}
    d = tempfile.mkdtemp(prefix="sbwt_refgpu_")
    try:
        sg.write_index_files(os.path.join(d, "ix"), built)
        wl.write_fasta(os.path.join(d, "q.fa"), sub_letters, sub_rows)
        flags = rp.index_flags(os.path.join(d, "ix"), os.path.join(d, "q.fa"), k, p_ref)
        t = time.perf_counter()
        res = rp.time_search(flags)
        res["program_wall_s"] = round(time.perf_counter() - t, 2)
    except (RuntimeError, OSError, subprocess.SubprocessError) as e:
        return {"unavailable": f"the reference program did not run: {str(e)[:300]}"}
    finally:
        shutil.rmtree(d, ignore_errors=True)
    n = int(sg.count_kmers(sub_rows, k))
    res.update({"kmers": n, "reads": nr, "p": p_ref, "flags": " ".join(f for f in flags if not f.startswith("--file")),
                "kmers_per_s": n / (res["search_ms"] / 1e3) if res.get("search_ms") else None,
                "what": "the reference's search kernel (src/search.cpp built for sm_100a), its own CUDA-event time"})
    return res


if __name__ == "__main__":
    sys.exit(main())
