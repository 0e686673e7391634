"""The reference program (oracle/_ref/search: the reference's src/search.cpp
built for sm_100a by oracle/Makefile) as a checker and as the reference-GPU
baseline.  Test and baseline infrastructure only: the product never runs it.

Every input handed to it keeps the reference's in-bounds conditions
(`check_safe`): all reads are ACGT, '\\n'-terminated and at least k long; the
k-mer count is a multiple of 64 and --threads-per-block=64, so no search
thread runs past the positions buffer (include/epicseq/search_caller.hpp:
84-86, include/gpu/search_kernel.hpp:65); 5 <= p <= 13 so 4^p is a multiple
of the block (include/presearch.hpp:38-42); the column count n is not a
multiple of 4096, so rank(n) reads a basic block inside the padded vector
(include/bit_vector.hpp:104).  The reference leaves the bytes past ceil(n/8)
of the last word uninitialised (include/bit_vector.hpp:119-124); runs set
MALLOC_PERTURB_=255, which makes glibc hand out zero-filled memory.
"""
import os
import re
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_SEARCH = os.path.join(HERE, "_ref", "search")


def available():
    return os.path.isfile(REF_SEARCH) and os.access(REF_SEARCH, os.X_OK)


def check_safe(n_bits, letters, rows, k, p):
    """Raises AssertionError unless the reference program stays in bounds on these inputs."""
    lens = np.diff(rows.astype(np.int64))
    n_kmers = int((lens - k + 1).sum())
    assert (lens >= k).all(), "every read must be at least k long"
    assert n_kmers % 64 == 0, "the k-mer count must be a multiple of 64"
    assert n_bits % 4096 != 0, "n must not be a multiple of 4096"
    assert p == 0 or 5 <= p <= 13
    assert set(np.unique(letters).tolist()) <= set(b"ACGT")


def reference_failed(err):
    """The reference's error reports (include/gpu/cuda.hpp:67-84, search_caller.hpp:68-71)."""
    return (b"did not succeed" in err or re.search(rb"CUDA error \d+ \(", err) is not None
            or re.search(rb"Last CUDA error code [1-9]", err) is not None)


def index_flags(prefix, queries, k, p):
    """The reference's flags (include/parameters.hpp:13-37) for index files prefix.{A,C,G,T} and a query file."""
    return [f"--file-a={prefix}.A", f"--file-c={prefix}.C", f"--file-g={prefix}.G", f"--file-t={prefix}.T",
            f"--file-queries={queries}", f"--k={k}", "--threads-per-block=64",
            f"--k-presearch={p}" if p else "--without-presearch"]


def time_search(flags, timeout=1800):
    """Runs the reference program with its answers not stored and returns the times it prints itself:
    "Search in GPU: X ms" (CUDA events around its search kernel, include/epicseq/kmer_search.hpp:167-169,
    include/gpu/search_and_presearch_launchers.hpp:41,53-54), the presearch and packing times, and the end
    of its stderr.  Raises RuntimeError if it reports an error."""
    env = dict(os.environ, MALLOC_PERTURB_="255")
    r = subprocess.run([REF_SEARCH] + flags + ["--do-not-store-results"], capture_output=True, env=env,
                       timeout=timeout)
    err = r.stderr.decode(errors="replace")
    if r.returncode != 0 or reference_failed(r.stderr):
        raise RuntimeError("the reference program reported an error: " + err[-2000:])

    def grab(pattern):
        m = re.search(pattern, err)
        return float(m.group(1)) if m else None

    return {"search_ms": grab(r"Search in GPU: ([0-9.]+) ms"),
            "presearch_ms": grab(r"Presearch takes ([0-9.]+) ms"),
            "pack_ms": grab(r"IN GPU: ([0-9.]+) ms"),
            "total_per_query_ns": grab(r"Total per query: ([0-9.]+) ns"),
            "stderr_tail": err[-1500:]}
