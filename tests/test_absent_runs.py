"""The absent-run lemma behind the run-walking search kernel, checked on the
CPU oracle: when the search of the k-mer at j fails after m letters, every
k-mer of the same row starting in [j+m-k, j] is absent.  A right-to-left walk
that uses it answers exactly as the per-k-mer search."""
import numpy as np
import pytest

import oracle as orc
import sbwt_gpu_b200 as sg
from sbwt_gpu_b200 import workloads as wl


def _case(seed, k, n_genome=30_000):
    rng = wl.rng_for(seed)
    genome = wl.random_bases(rng, n_genome)
    built = sg.build_sbwt([genome.tobytes()], k)
    letters, rows = wl.mixed_reads(rng, genome, 60, 60, 150, 0.02)
    return built, letters, rows


def _walk(ans, steps, rows, k, p):
    """The kernel's run walk, over per-k-mer oracle results: start at the row's
    last k-mer; a failure after m = p + steps letters settles k-m+1 k-mers."""
    out = np.full(ans.size, orc.NOT_FOUND, dtype=np.uint64)
    searched = 0
    j0 = 0
    for r in range(rows.size - 1):
        n = int(rows[r + 1] - rows[r]) - k + 1
        if n <= 0:
            continue
        j = j0 + n - 1
        while j >= j0:
            searched += 1
            if ans[j] != orc.NOT_FOUND:
                out[j] = ans[j]
                j -= 1
            else:
                m = max(p, p + int(steps[j]))  # the failing prefix length (p alone: empty entry)
                j -= k - min(m, k) + 1
        j0 += n
    return out, searched


@pytest.mark.parametrize("k,p", [(31, 10), (31, 0), (21, 8), (9, 4)])
def test_absent_prefix_settles_its_kmers(k, p):
    built, letters, rows = _case(77 + k, k)
    ox = orc.OracleIndex(built.bits, built.n_bits)
    ans, steps = ox.search_reads(letters, rows, k, p, want_steps=True)
    j0 = 0
    checked = 0
    for r in range(rows.size - 1):
        n = int(rows[r + 1] - rows[r]) - k + 1
        if n <= 0:
            continue
        a = ans[j0:j0 + n]
        s = steps[j0:j0 + n]
        for j in np.flatnonzero(a == orc.NOT_FOUND):
            m = min(k, p + int(s[j]))
            lo = max(0, j + m - k)
            assert (a[lo:j + 1] == orc.NOT_FOUND).all(), (r, j, m)
            checked += 1
        j0 += n
    assert checked > 1000


@pytest.mark.parametrize("k,p", [(31, 10), (31, 0), (31, 12), (13, 13)])
def test_right_to_left_walk_matches_every_kmer(k, p):
    built, letters, rows = _case(91 + p, k)
    ox = orc.OracleIndex(built.bits, built.n_bits)
    ans, steps = ox.search_reads(letters, rows, k, p, want_steps=True)
    out, searched = _walk(ans, steps, rows, k, p)
    assert np.array_equal(out, ans)
    if k - p >= 8:
        assert searched < 0.6 * ans.size  # half the reads are random: most of their k-mers are settled
