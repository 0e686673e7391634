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


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--scale", type=float, default=1.0, help="shrinks the workload (tests only)")
    ap.add_argument("--p", type=int, default=12)
    ap.add_argument("--kpt", type=int, default=0)
    ap.add_argument("--tpk", type=int, default=0)
    ap.add_argument("--tpb", type=int, default=0)
    ap.add_argument("--layout", choices=["lines", "poppy"], default="lines")
    ap.add_argument("--sb", type=int, default=1024, help="bits in superblock of the poppy layout")
    ap.add_argument("--l2-fetch", type=int, default=0, choices=[0, 32, 64, 128],
                    help="L2 fetch granularity in bytes for the searches (0: leave the device default)")
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="CPU baseline sample budget")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-prefilter", action="store_true", help="skip the learned-prefilter leg")
    ap.add_argument("--no-autotune", action="store_true", help="skip the autotuned leg")
    ap.add_argument("--no-per-kmer", action="store_true", help="skip the leg that searches every k-mer")
    ap.add_argument("--no-contract", action="store_true", help="skip the leg on the reference's kernel contract")
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
        genome, letters, rows = workload(args.scale, rank)
        return [genome], letters, rows, args.p
    if args.workload == "batched":
        import sbwt_gpu_b200 as sg
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
        return [genome], letters, rows, 10
    # pangenome
    rng = wl.rng_for(1239)
    base = wl.random_bases(rng, int(50_000_000 * args.scale), gc=0.41)
    haps = wl.haplotypes(rng, base, 20)
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
    return haps, letters, rows, 14


def workload(scale, rank):
    from sbwt_gpu_b200 import workloads as wl
    rng = wl.rng_for(1236)
    n = int(100_000_000 * scale)
    genome = wl.random_bases(rng, n, gc=0.41)
    genome = wl.with_repeats(rng, genome, int(0.05 * n))
    rrng = wl.rng_for(7000 + rank)
    n_reads = max(10, int(10_000_000 * scale))
    n_pos = n_reads // 10
    letters, rows = wl.mixed_reads(rrng, genome, n_pos, n_reads - n_pos, 150, 0.01)
    return genome, letters, rows


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
    """Share of k-mers the run walk searches from scratch, and share it reaches by a backward step
    (right to left per read; a search that fails after m letters settles k-m+1 k-mers; with
    `stream`, the k-mer left of a found one takes a backward step), from per-k-mer oracle answers
    and step counts of the first `max_rows` reads."""
    import oracle as orc
    searched = back = total = 0
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
                if hit:
                    have = True
                    j -= 1
                else:
                    j -= k - min(max(p, p + int(steps[j])), k) + 1
        j0 += n
        total += n
    return searched / max(total, 1), back / max(total, 1)


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


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    k = 31
    p = args.p
    host_threads_per_rank(world, args.impl)

    if args.impl == "reference":
        if rank != 0:
            return 0
        return reference_arm(args, k, p)

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
    # the index: rank 0 builds the SBWT and writes the reference's files; every rank loads them
    tmpdir = os.environ.get("SBWT_BENCH_DIR") or os.path.join(tempfile.gettempdir(), f"sbwt_bench_{os.getppid()}")
    os.makedirs(tmpdir, exist_ok=True)
    prefix = os.path.join(tmpdir, "ix")
    if rank == 0:
        t = time.perf_counter()
        built = sg.build_sbwt([x.tobytes() for x in seqs], k, device=local_rank)  # the GPU builder
        build_s = time.perf_counter() - t
        paths = sg.write_index_files(prefix, built)
        n_columns = built.n_bits
        del built
    if world > 1:
        dist.barrier()
    paths = [f"{prefix}.{c}" for c in "ACGT"]
    layout = sg.SBWT_LAYOUT_POPPY if args.layout == "poppy" else sg.SBWT_LAYOUT_LINES
    t = time.perf_counter()
    ix = sg.Index.load(*paths, k=k, k_presearch=p, device=local_rank, layout=layout, bits_in_superblock=args.sb,
                       kmers_per_thread=args.kpt, threads_per_kmer=args.tpk, threads_per_block=args.tpb,
                       search_mode=MODES[args.search_mode])
    runs_form = args.kpt == 0 and args.search_mode != "every" and (args.tpk <= 1 or args.layout == "poppy")
    kernel = ("search_runs_kernel" + ("<stream>" if args.search_mode == "stream" else "<skip>") if runs_form
              else ("search_queue_kernel" if args.kpt == 0 else "search_kernel"))
    load_s = time.perf_counter() - t
    if args.l2_fetch:
        ix.set_l2_fetch_granularity(args.l2_fetch)
    build_times = ix.build_times()  # device ms: rank words (lines), poppy, presearch, backward table
    info = ix.info()

    d_letters = torch.from_numpy(letters).to(dev)
    d_rows = torch.from_numpy(rows.view(np.int64)).to(dev)
    d_ans = torch.empty(n_kmers, dtype=torch.int64, device=dev)
    d_mem = torch.empty((n_kmers + 31) // 32, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev)
    ix.profile(True)

    def step():
        ix.search_reads(d_letters, d_rows, d_ans, n_kmers, d_member_bits=d_mem, stream=stream)

    for _ in range(max(args.warmup, 0)):
        step()
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    clocks = Clocks(local_rank)
    clocks.start()
    torch.cuda.synchronize(dev)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    search_ms, launches = [], 0
    ev0.record(stream)
    for _ in range(args.steps):
        step()
        prof = ix.last_profile()  # CUDA events of this step's kernels (on `stream`)
        search_ms.append(prof["search_ms"])
        launches += prof["launches"]
    ev1.record(stream)
    torch.cuda.synchronize(dev)
    total_ms = ev0.elapsed_time(ev1)
    clk = clocks.stop()
    if world > 1:
        dist.barrier()
        total_ms = max_over_ranks(total_ms)
    value = n_kmers * world * args.steps / (total_ms / 1e3)

    # ---- correctness on a sample + the CPU baseline (rank 0 only, untimed)
    cpu = None
    mean_steps = None
    if rank == 0:
        ox = orc.OracleIndex.from_files(paths)
        p_cpu = min(p, 12)  # answers do not depend on p; a CPU table beyond 4^12 entries costs minutes
        table = ox.presearch(p_cpu) if p_cpu else None
        rate, ans, steps, nr, threads = cpu_reference(ox, letters, rows, k, p_cpu, args.cpu_seconds, table)
        got = d_ans[: ans.size].cpu().numpy().view(np.uint64)
        if not np.array_equal(got, ans):
            raise SystemExit(f"bench: {int((got != ans).sum())} of {ans.size} sampled answers differ from the oracle")
        mean_steps = float(steps.mean())
        searched, back = walk_model(ans, steps, rows, k, p_cpu, args.search_mode == "stream") if runs_form else (1.0, 0.0)
        cpu = {"value": rate, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": f"first {nr} reads ({ans.size} k-mers) of the same batch, C restatement of the reference "
                         f"search (the reference has no CPU search), OpenMP schedule(dynamic,4096)"}

    # ---- end to end through the host entry point (pinned buffers)
    e2e = None
    if not args.no_e2e:
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
        d_back = h_ans.to(dev)  # every answer against the device search's (checked against the oracle above)
        if not torch.equal(d_back, d_ans):
            raise SystemExit("bench: end-to-end answers differ from the device search's")
        # bytes that crossed PCIe in the last call: the answers come back as bitmap + group offsets +
        # 32-bit node ids of the found k-mers (sparse, expanded by the host threads), as u64 answers
        # (dense), or both (hybrid; SBWT_PIPELINE_TRANSFER picks one, else by host thread count)
        moved = ix.pipeline_bytes()
        mode = os.environ.get("SBWT_PIPELINE_TRANSFER", "") or "auto"
        e2e = {"value": n_kmers * world * args.e2e_steps / e2e_s, "unit": UNIT,
               "h2d_bytes_per_step": int(moved["h2d"]), "d2h_bytes_per_step": int(moved["d2h"]),
               "answer_bytes_per_step": int(n_kmers * 8),
               "transfer": mode + (": u64 answers" if moved["d2h"] >= n_kmers * 8 else
                                   ": every fourth chunk as u64 answers, the others as bitmap + found node ids"
                                   if mode == "hybrid" else
                                   ": bitmap + found node ids, expanded into the u64 answers by the host threads")}
        # membership only (sbwt_search_reads_host_member): the bitmap crosses the bus, not the answers
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
            want_bits = bits_of(ans)[:full]
            if not np.array_equal(h_mem[:full].numpy().view(np.uint32), want_bits):
                raise SystemExit("bench: end-to-end membership bits differ from the oracle")
        moved = ix.pipeline_bytes()
        e2e["membership_only"] = {"value": n_kmers * world * args.e2e_steps / m_s, "unit": UNIT,
                                  "h2d_bytes_per_step": int(moved["h2d"]),
                                  "d2h_bytes_per_step": int(moved["d2h"]),
                                  "entry_point": "sbwt_search_reads_host_member"}

    # ---- the same batch with every k-mer searched (the reference's per-k-mer work), for comparison
    per_kmer = None
    if runs_form and not args.no_per_kmer and rank == 0:
        ix.profile(True)
        ix.set_search_mode(sg.SEARCH_EVERY_KMER)
        for _ in range(2):
            step()
        torch.cuda.synchronize(dev)
        ev0.record(stream)
        t_ms = []
        for _ in range(args.steps):
            step()
            t_ms.append(ix.last_profile()["search_ms"])
        ev1.record(stream)
        torch.cuda.synchronize(dev)
        tt = ev0.elapsed_time(ev1)
        ix.set_search_mode(MODES[args.search_mode])
        got = d_ans[: ans.size].cpu().numpy().view(np.uint64)
        if not np.array_equal(got, ans):
            raise SystemExit("bench: per-k-mer answers differ from the oracle")
        per_kmer = {"value": n_kmers * args.steps / (tt / 1e3), "ms_per_step": tt / args.steps,
                    "search_kernel_ms": statistics.mean(t_ms), "kernel": "search_queue_kernel"}

    # ---- membership only on the device: no answer array, the kernel writes the bitmap alone
    member_only = None
    if runs_form and rank == 0:
        ix.profile(True)
        d_mem2 = torch.zeros_like(d_mem)

        def mstep():
            ix.search_reads(d_letters, d_rows, None, n_kmers, d_member_bits=d_mem2, stream=stream)

        for _ in range(2):
            mstep()
        torch.cuda.synchronize(dev)
        ev0.record(stream)
        t_ms = []
        for _ in range(args.steps):
            mstep()
            t_ms.append(ix.last_profile()["search_ms"])
        ev1.record(stream)
        torch.cuda.synchronize(dev)
        tt = ev0.elapsed_time(ev1)
        full = ans.size // 32
        if not np.array_equal(d_mem2[:full].cpu().numpy().view(np.uint32), bits_of(ans)[:full]):
            raise SystemExit("bench: membership bits differ from the oracle")
        member_only = {"value": n_kmers * args.steps / (tt / 1e3), "ms_per_step": tt / args.steps,
                       "search_kernel_ms": statistics.mean(t_ms), "output": "membership bitmap only (no answers)"}
        del d_mem2

    # ---- the reference's kernel contract (sbwt_search_packed): packed letters + the reference's
    # positions array (k-mer j of read r at row_start[r] + i), answers written over the positions
    contract = None
    if rank == 0 and not args.no_contract:
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
        for it in range(2 + args.steps):
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
        contract = {"value": n_kmers / (cm / 1e3), "ms_per_call": cm, "entry_point": "sbwt_search_packed",
                    "note": "positions array in, answers out in place, as the reference's search kernel"}
        del d_pos, d_pos0, d_words, lens, cnt, rs, ks

    # ---- autotuned leg: the tuner picks shape and presearch depth on a sample, then the batch is timed again
    tuned = None
    if not args.no_autotune and rank == 0:
        ns = min(rows.size - 1, 1_000_000)
        nk_s = sg.count_kmers(rows[: ns + 1], k)
        d_ls = torch.from_numpy(letters[: int(rows[ns])]).to(dev)
        d_rs = torch.from_numpy(rows[: ns + 1].view(np.int64)).to(dev)
        rep = ix.autotune(d_ls, d_rs, d_ans, nk_s, tune_p=True, tune_poppy=True)
        del d_ls, d_rs
        ix.profile(True)
        for _ in range(2):
            step()
        torch.cuda.synchronize(dev)
        ev0.record(stream)
        t_ms = []
        for _ in range(args.steps):
            step()
            t_ms.append(ix.last_profile()["search_ms"])
        ev1.record(stream)
        torch.cuda.synchronize(dev)
        tt = ev0.elapsed_time(ev1)
        got = d_ans[: ans.size].cpu().numpy().view(np.uint64)
        if not np.array_equal(got, ans):
            raise SystemExit("bench: autotuned answers differ from the oracle")
        tuned = {"value": n_kmers * args.steps / (tt / 1e3), "ms_per_step": tt / args.steps,
                 "search_kernel_ms": statistics.mean(t_ms), "choice": rep["best"],
                 "candidates": len(rep["candidates"]), "tuned_on_kmers": nk_s}

    # ---- learned-prefilter leg (the prefilter configuration: index of the small workload, 90% negatives)
    prefilter = None
    if not args.no_prefilter and rank == 0:
        prefilter = prefilter_leg(args, dev, k)

    if rank == 0:
        peak, peak_kind = measured_hbm()
        kern_ms = statistics.mean(search_ms)
        q = (letters.size / 4.0) / n_kmers
        b_kmer = 128.0 * mean_steps + 16 + 8 + q
        achieved = n_kmers * b_kmer / (kern_ms / 1e3) / 1e9
        traffic, tr = kernel_traffic(kernel, args.workload if args.scale == 1.0 else None, n_kmers)
        hits = int((d_ans.cpu().numpy().view(np.uint64) != orc.NOT_FOUND).sum())
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic (seeded)",
            "config": {
                "workload": WORKLOADS[args.workload] if args.scale == 1.0 else f"{args.workload} x{args.scale}",
                "n_kmers_per_gpu": n_kmers, "n_columns": info["n_bits"], "k": k, "p": p,
                "layout": args.layout, "present_kmers": hits, "l2_fetch_bytes": args.l2_fetch or "default",
                "l2": "inputs and outputs larger than L2 (letters %.2f GB, answers %.2f GB); no flush" % (
                    letters.nbytes / 1e9, n_kmers * 8 / 1e9),
                "parallelism": f"replicas x{world}" if world > 1 else "1 GPU",
                "index_build_s": round(build_s, 2), "index_builder": "gpu (sbwt_build_gpu, incl. host copies)", "index_load_s": round(load_s, 2),
                "index_build_device_ms": {kk: round(vv, 3) for kk, vv in build_times.items()},
            },
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_kind": f"of {peak_kind}",
                         "kernel": kernel, "kernel_ms": kern_ms, "bytes_per_kmer_model": b_kmer,
                         "mean_steps": mean_steps, "steps_counted_at_p": p_cpu, "searched_fraction": searched, "backward_step_fraction": back,
                         "dram_frac": (traffic / (kern_ms / 1e3) / 1e9 / peak) if traffic else None,
                         "traffic_source": tr["source"] if tr else None},
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": launches,
            "clocks": clk,
            "per_kmer": per_kmer,
            "membership_only": member_only,
            "kernel_contract": contract,
            "autotuned": tuned,
            "prefilter": prefilter,
        }
        print(json.dumps(line), flush=True)
    ix.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def prefilter_leg(args, dev, k):
    """Plain vs learned-prefiltered search of 200M single k-mers (90% negatives: half uniform random, half
    indexed k-mers with 1-3 substitutions) against the index of the small workload (1 Mbp uniform genome,
    p = 10); the MLP is trained on the GPU (20k Adam steps, batch 8192, 5e7 + 5e7 candidates)."""
    import torch
    import sbwt_gpu_b200 as sg
    from sbwt_gpu_b200 import workloads as wl
    w = wl.small_workload(seed=1235)
    built = sg.build_sbwt([w["genome"].tobytes()], k)
    pix = sg.Index.from_bits(built.bits, built.n_bits, k=k, k_presearch=10)
    t = time.perf_counter()
    pf = sg.Prefilter.train(pix, steps=args.pf_steps, batch=8192, n_positive=50_000_000, n_negative=50_000_000,
                            seed=4)
    train_s = time.perf_counter() - t
    st = pf.stats()
    kmers = wl.kmer_query_words(wl.rng_for(4242), w["genome"], args.pf_queries, k, neg_frac=0.9)
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
    reps = max(args.steps, 3)
    ms_plain = timed(lambda: pix.search_kmers(d_k, plain), reps)
    ms_logits = timed(lambda: pf.logits(d_k, d_l), reps)
    ms_filt = timed(lambda: pix.search_kmers_filtered(pf, d_k, filt), reps)
    skipped = pix.search_kmers_filtered(pf, d_k, filt)
    torch.cuda.synchronize(dev)
    p_np, f_np = plain.cpu().numpy().view(np.uint64), filt.cpu().numpy().view(np.uint64)
    nf = 0xFFFFFFFFFFFFFFFF
    false_absent = int(((p_np != nf) & (f_np == nf)).sum())
    res = {
        "workload": "prefilter: index of the small workload (1 Mbp uniform genome, k=31, p=10); "
                    f"{n} single k-mers, 90% negatives (half uniform random, half 1-3 substitutions)",
        "plain_kmers_per_s": n / (ms_plain / 1e3), "prefiltered_kmers_per_s": n / (ms_filt / 1e3),
        "speedup": ms_plain / ms_filt, "mlp_kmers_per_s": n / (ms_logits / 1e3),
        "mlp_tflops": n * 2 * (128 * 256 + 256 * 256 + 256) / (ms_logits / 1e3) / 1e12,
        "skip_rate": skipped / n, "false_absent": false_absent, "bit_exact": bool(np.array_equal(p_np, f_np)),
        "present": int((p_np != nf).sum()), "train_s": round(train_s, 2), "train": st,
    }
    pf.close()
    pix.close()
    return res


def reference_arm(args, k, p):
    import oracle as orc
    import sbwt_gpu_b200 as sg
    seqs, letters, rows, p = workload_of(args, 0)
    built = sg.build_sbwt([x.tobytes() for x in seqs], k)
    ox = orc.OracleIndex(built.bits, built.n_bits)
    del built
    p = min(p, 12)  # answers do not depend on p; a CPU table beyond 4^12 entries costs minutes
    table = ox.presearch(p) if p else None
    # each step: a bounded sample of the batch sized to ~budget seconds
    budget = max(1.0, min(args.cpu_seconds, 150.0 / max(args.steps + args.warmup, 1)))
    rate, ans, steps, nr, threads = cpu_reference(ox, letters, rows, k, p, budget, table)
    sub_rows = rows[: nr + 1]
    sub_letters = letters[: int(sub_rows[-1])]
    for _ in range(max(args.warmup - 1, 0)):
        ox.search_reads(sub_letters, sub_rows, k, p, table)
    t = time.perf_counter()
    for _ in range(args.steps):
        ox.search_reads(sub_letters, sub_rows, k, p, table)
    dt = time.perf_counter() - t
    value = ans.size * args.steps / dt
    sample = (f"first {nr} reads ({ans.size} k-mers) per step of the large workload; C restatement of the "
              f"reference search (the reference has no CPU search), OpenMP, {threads} threads")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3 / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic (seeded)",
        "config": {"workload": WORKLOADS[args.workload] if args.scale == 1.0 else f"{args.workload} x{args.scale}",
                   "k": k, "p": p},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
