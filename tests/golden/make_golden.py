"""Golden fixtures produced by the reference program itself.

The reference ships no tests or fixtures, so its answers are pinned by running
its own program (oracle/_ref/search: src/search.cpp built for sm_100a by
oracle/Makefile) on seeded inputs and recording its stdout.

    python tests/golden/make_golden.py prepare   # CPU: write the inputs under tests/golden/cases/
    python tests/golden/make_golden.py run OUT   # on a B200: run the reference on every case into OUT/
    python tests/golden/make_golden.py collect OUT  # CPU: store OUT/<case>.out as fixtures

Every case keeps the reference's in-bounds conditions (checked by
`check_safe`): all reads are ACGT, '\\n'-terminated and at least k long; the
k-mer count is a multiple of 64 and --threads-per-block=64, so no search
thread runs past the positions buffer (include/epicseq/search_caller.hpp:
84-86, include/gpu/search_kernel.hpp:65); 5 <= p <= 13 so 4^p is a multiple
of the block (include/presearch.hpp:38-42); the column count n is not a
multiple of 4096, so rank(n) reads a basic block inside the padded vector
(include/bit_vector.hpp:104).  The reference leaves the bytes past ceil(n/8)
of the last word uninitialised (include/bit_vector.hpp:119-124); the run
sets MALLOC_PERTURB_=255, which makes glibc hand out zero-filled memory.
"""
import gzip
import hashlib
import re
import json
import os
import shutil
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
from ref_program import REF_SEARCH, check_safe, reference_failed  # noqa: E402

CASES = os.path.join(HERE, "cases")

# name: (seed, genome bp, reads, read length, k, p (0 = --without-presearch), SB, rank structure, shuffles)
SPECS = {
    "sb1024_poppy_p10": (11, 40_000, 96, 150, 31, 10, 1024, "poppy", False),
    "sb256_cum_p7": (12, 30_000, 96, 150, 31, 7, 256, "cum-poppy", False),
    "sb2048_poppy_shuffles_p12": (13, 50_000, 96, 150, 31, 12, 2048, "poppy", True),
    "sb4096_poppy_nopre": (14, 35_000, 96, 150, 31, 0, 4096, "poppy", False),
    "sb512_cum_k25_p9": (15, 30_000, 96, 150, 25, 9, 512, "cum-poppy", False),
    "sb1024_cum_shuffles_k32_p13": (16, 45_000, 128, 150, 32, 13, 1024, "cum-poppy", True),
    "sb2048_cum_k15_p5": (17, 20_000, 64, 100, 15, 5, 2048, "cum-poppy", False),
}


# The small workload (1,000,000 bp genome, 10,000 reads of 150 bp,
# k=31, p=10), regenerated from its seed wherever it is needed; only the
# SHA-256 of the reference's output is stored (small_workload.json).
SMALL_SEED = 1235
SMALL_JSON = os.path.join(HERE, "small_workload.json")


def write_small_workload(d):
    """Writes the small workload's index files and query FASTA into d; returns (n_bits, letters, rows)."""
    import sbwt_gpu_b200 as sg
    from sbwt_gpu_b200 import workloads as wl
    w = wl.small_workload(seed=SMALL_SEED)
    built = sg.build_sbwt([w["genome"].tobytes()], w["k"])
    check_safe(built.n_bits, w["letters"], w["row_starts"], w["k"], w["p"])
    os.makedirs(d, exist_ok=True)
    sg.write_index_files(os.path.join(d, "ix"), built)
    wl.write_fasta(os.path.join(d, "queries.fa"), w["letters"], w["row_starts"])
    return built.n_bits, w["letters"], w["row_starts"]


def small_workload_flags(d):
    return [f"--file-a={d}/ix.A", f"--file-c={d}/ix.C", f"--file-g={d}/ix.G", f"--file-t={d}/ix.T",
            f"--file-queries={d}/queries.fa", "--k=31", "--k-presearch=10", "--threads-per-block=64"]


def case_flags(name, cases=CASES):
    seed, gbp, nreads, rl, k, p, sb, rs, sh = SPECS[name]
    d = os.path.join(cases, name)
    flags = [f"--file-a={d}/ix.A", f"--file-c={d}/ix.C", f"--file-g={d}/ix.G", f"--file-t={d}/ix.T",
             f"--file-queries={d}/queries.fa", f"--k={k}", f"--bits-in-superblock={sb}",
             f"--rank-structure={rs}", "--threads-per-block=64"]
    flags.append(f"--k-presearch={p}" if p else "--without-presearch")
    if sh:
        flags.append("--with-shuffles")
    return flags


def prepare():
    import sbwt_gpu_b200 as sg
    from sbwt_gpu_b200 import workloads as wl
    for name, (seed, gbp, nreads, rl, k, p, sb, rs, sh) in SPECS.items():
        rng = wl.rng_for(seed)
        gl = gbp
        while True:  # n must not be a multiple of 4096
            genome = wl.random_bases(rng, gl)
            built = sg.build_sbwt([genome.tobytes()], k)
            if built.n_bits % 4096:
                break
            gl += 1
        letters, rows = wl.mixed_reads(rng, genome, nreads // 2, nreads - nreads // 2, rl, 0.01)
        check_safe(built.n_bits, letters, rows, k, p)
        d = os.path.join(CASES, name)
        os.makedirs(d, exist_ok=True)
        sg.write_index_files(os.path.join(d, "ix"), built)
        wl.write_fasta(os.path.join(d, "queries.fa"), letters, rows)
        with open(os.path.join(d, "case.json"), "w") as f:
            json.dump({"k": k, "p": p, "bits_in_superblock": sb, "rank_structure": rs, "with_shuffles": sh,
                       "n_bits": built.n_bits, "n_kmers": int((np.diff(rows.astype(np.int64)) - k + 1).sum())},
                      f, indent=1)
        print(name, "n =", built.n_bits)


def run(out_dir):
    os.makedirs(out_dir, exist_ok=True)
    env = dict(os.environ, MALLOC_PERTURB_="255")
    c1 = os.path.join(out_dir, "small_workload_inputs")
    write_small_workload(c1)
    jobs = [(name, case_flags(name)) for name in SPECS] + [("small_workload", small_workload_flags(c1))]
    for name, flags in jobs:
        with open(os.path.join(out_dir, f"{name}.out"), "wb") as fo, \
                open(os.path.join(out_dir, f"{name}.err"), "wb") as fe:
            rc = subprocess.run([REF_SEARCH] + flags, stdout=fo, stderr=fe, env=env, timeout=300).returncode
        print(name, "rc", rc)
    shutil.rmtree(c1)


def collect(out_dir):
    for name in SPECS:
        src = os.path.join(out_dir, f"{name}.out")
        err = open(os.path.join(out_dir, f"{name}.err"), "rb").read()
        if reference_failed(err):
            raise SystemExit(f"{name}: the reference reported an error")
        data = open(src, "rb").read()
        with open(os.path.join(CASES, name, "reference.out.gz"), "wb") as raw, \
                gzip.GzipFile(fileobj=raw, mode="wb", mtime=0) as f:
            f.write(data)
        meta_p = os.path.join(CASES, name, "case.json")
        meta = json.load(open(meta_p))
        meta["reference_sha256"] = hashlib.sha256(data).hexdigest()
        json.dump(meta, open(meta_p, "w"), indent=1)
        print(name, len(data), "bytes")
    err = open(os.path.join(out_dir, "small_workload.err"), "rb").read()
    if reference_failed(err):
        raise SystemExit("small workload: the reference reported an error")
    data = open(os.path.join(out_dir, "small_workload.out"), "rb").read()
    json.dump({"seed": SMALL_SEED, "bytes": len(data), "lines": data.count(b"\n"),
               "minus_ones": data.count(b"-1 "), "reference_sha256": hashlib.sha256(data).hexdigest()},
              open(SMALL_JSON, "w"), indent=1)
    print("small_workload", len(data), "bytes")


if __name__ == "__main__":
    cmd = sys.argv[1]
    if cmd == "prepare":
        prepare()
    elif cmd == "run":
        run(sys.argv[2])
    elif cmd == "collect":
        collect(sys.argv[2])
    else:
        raise SystemExit(__doc__)
