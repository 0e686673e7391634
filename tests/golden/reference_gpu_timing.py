"""Times the reference's own CUDA search kernel (oracle/_ref/search: the
reference program built for sm_100a) on the large benchmark workload, from
the kernel time the reference itself prints ("Search in GPU: X ms",
include/epicseq/kmer_search.hpp:167-169; CUDA events around the kernel,
include/gpu/search_and_presearch_launchers.hpp:41,53-54).

    python tests/golden/reference_gpu_timing.py [--scale S] [--out FILE] [--cli]

With --cli both programs also store their answers (the reference's stdout
format) and the wall time of each whole program run is recorded: the
reference's build/search against this project's sbwt_search, same flags,
same index files and query file; the two outputs must be byte-identical.

The inputs satisfy the reference's in-bounds conditions (make_golden.check_safe):
150 bp ACGT reads, a k-mer count that is a multiple of 64 with
--threads-per-block=64, p = 12, n not a multiple of 4096.  The answers are
not printed (--do-not-store-results).  Test infrastructure only.
"""
import argparse
import json
import os
import re
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--scale", type=float, default=1.0)
    ap.add_argument("--out", default=None)
    ap.add_argument("--cli", action="store_true", help="also time both programs end to end with stored results")
    args = ap.parse_args()
    import bench
    import make_golden
    import sbwt_gpu_b200 as sg
    from sbwt_gpu_b200 import workloads as wl
    genome, letters, rows = bench.workload(args.scale, 0)
    built = sg.build_sbwt([genome.tobytes()], 31)
    make_golden.check_safe(built.n_bits, letters, rows, 31, 12)
    d = tempfile.mkdtemp(prefix="sbwt_ref_")
    sg.write_index_files(os.path.join(d, "ix"), built)
    n_bits = built.n_bits
    del built, genome
    wl.write_fasta(os.path.join(d, "queries.fa"), letters, rows)
    flags = make_golden.small_workload_flags(d)
    flags = [f for f in flags if not f.startswith("--k-presearch")] + ["--k-presearch=12", "--do-not-store-results"]
    env = dict(os.environ, MALLOC_PERTURB_="255")
    r = subprocess.run([make_golden.REF_SEARCH] + flags, capture_output=True, env=env, timeout=3600)
    err = r.stderr.decode(errors="replace")
    if r.returncode != 0 or make_golden.reference_failed(r.stderr):
        print(err[-3000:])
        raise SystemExit("the reference reported an error")

    def grab(pattern):
        m = re.search(pattern, err)
        return float(m.group(1)) if m else None

    n_kmers = int((rows[1:] - rows[:-1]).astype("int64").sum() - (rows.size - 1) * 30)
    res = {
        "workload": f"large x{args.scale}", "n_kmers": n_kmers, "n_columns": n_bits,
        "search_ms": grab(r"Search in GPU: ([0-9.]+) ms"),
        "presearch_ms": grab(r"Presearch takes ([0-9.]+) ms"),
        "pack_ms": grab(r"IN GPU: ([0-9.]+) ms"),
        "total_per_query_ns": grab(r"Total per query: ([0-9.]+) ns"),
        "flags": " ".join(f for f in flags if not f.startswith("--file")),
    }
    res["search_kmers_per_s"] = n_kmers / (res["search_ms"] / 1e3) if res["search_ms"] else None
    if args.cli:
        res["cli"] = time_programs(d, flags, env)
    line = json.dumps(res)
    print(line)
    if args.out:
        with open(args.out, "w") as f:
            f.write(line + "\n")


def time_programs(d, flags, env):
    """Wall time of each program writing its answers to a file, and the outputs' SHA-256."""
    import hashlib
    import time
    import sbwt_gpu_b200 as sg
    import make_golden
    store = [f for f in flags if f != "--do-not-store-results"]
    out = {}
    for name, exe in (("reference", make_golden.REF_SEARCH), ("ours", sg.CLI_PATH)):
        path = os.path.join(d, f"{name}.out")
        with open(path, "wb") as f:
            t = time.perf_counter()
            r = subprocess.run([exe] + store, stdout=f, stderr=subprocess.PIPE, env=env, timeout=3600)
            wall = time.perf_counter() - t
        if r.returncode != 0 or (name == "reference" and make_golden.reference_failed(r.stderr)):
            raise SystemExit(f"{name} failed: {r.stderr.decode(errors='replace')[-2000:]}")
        h = hashlib.sha256()
        with open(path, "rb") as f:
            for block in iter(lambda: f.read(1 << 24), b""):
                h.update(block)
        out[name] = {"wall_s": wall, "bytes": os.path.getsize(path), "sha256": h.hexdigest(),
                     "stderr_tail": r.stderr.decode(errors="replace")[-600:]}
        os.remove(path)
    out["identical"] = out["reference"]["sha256"] == out["ours"]["sha256"]
    return out


if __name__ == "__main__":
    main()
