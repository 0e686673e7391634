"""The batched-uneven and pangenome workload shapes at reduced scale,
bit for bit against the oracle (needs a B200)."""
import numpy as np
import pytest

import oracle as orc
import sbwt_gpu_b200 as sg
from sbwt_gpu_b200 import workloads as wl

pytestmark = pytest.mark.gpu


def _search(ix, letters, rows, dev):
    import torch
    nk = sg.count_kmers(rows, ix.info()["k"])
    d_ans = torch.empty(max(nk, 1), dtype=torch.int64, device=dev)
    ix.search_reads(torch.from_numpy(letters).to(dev), torch.from_numpy(rows.view(np.int64)).to(dev), d_ans, nk)
    torch.cuda.synchronize()
    return d_ans.cpu().numpy().view(np.uint64)[:nk]


def test_batched_uneven_files_one_launch(cuda, tmp_path):
    """64 query files, read lengths from the 150 bp / lognormal 2 kbp / lognormal 15 kbp mixture."""
    rng = wl.rng_for(31)
    genome = wl.random_bases(rng, 300_000)
    built = sg.build_sbwt([genome.tobytes()], 31)
    paths = []
    for f, (letters, rows) in enumerate(wl.uneven_read_files(genome, seed=32, total_kmers=3_000_000, n_files=64)):
        p = str(tmp_path / f"q{f:02d}.fa")
        wl.write_fasta(p, letters, rows)
        paths.append(p)
    letters, rows, nk, file_rows = sg.read_queries_many(paths, 31)
    assert nk == 3_000_000
    lens = np.diff(rows.astype(np.int64))
    assert lens.max() > 5000 and (lens == 150).mean() > 0.5  # the mixture is there
    ox = orc.OracleIndex(built.bits, built.n_bits)
    want = ox.search_reads(letters, rows, 31, 10)
    with sg.Index.from_bits(built.bits, built.n_bits, k=31, k_presearch=10) as ix:
        got = _search(ix, letters, rows, cuda)
        host = ix.search_reads_host(letters, rows)
    assert np.array_equal(got, want)
    assert np.array_equal(host, want)
    assert 0.05 < (want != orc.NOT_FOUND).mean() < 0.6


def test_pangenome_union_index(cuda):
    """20 haplotypes with SNPs and indels; the index holds the union of their k-mers."""
    rng = wl.rng_for(51)
    base = wl.random_bases(rng, 100_000, gc=0.41)
    haps = wl.haplotypes(rng, base, 20)
    built = sg.build_sbwt([h.tobytes() for h in haps], 31)
    keys, dk, _ = orc.independent_sbwt([h.tobytes() for h in haps], 31)
    assert built.n_kmers == keys.size and built.n_dummies == dk.size
    # queries: reads sampled from the haplotypes (positives) and random reads (negatives)
    reads = [wl.sampled_reads(rng, haps[i % 20], 20, 150, 0.0) for i in range(20)]
    pos = np.concatenate(reads)
    # reads with 1% and 3% substitutions: found stretches broken by absent ones (backward steps, then
    # fresh searches after each substitution)
    subs = np.concatenate([wl.sampled_reads(rng, haps[i % 20], 10, 150, 0.01 if i % 2 else 0.03) for i in range(20)])
    neg = wl.uniform_reads(rng, 200, 150)
    q = np.concatenate([pos, subs, neg])
    letters = np.ascontiguousarray(q).reshape(-1)
    rows = np.arange(q.shape[0] + 1, dtype=np.uint64) * np.uint64(150)
    ox = orc.OracleIndex(built.bits, built.n_bits)
    want = ox.search_reads(letters, rows, 31, 12)
    with sg.Index.from_bits(built.bits, built.n_bits, k=31, k_presearch=12) as ix:
        got = _search(ix, letters, rows, cuda)
    assert np.array_equal(got, want)
    n_pos = pos.shape[0] * 120
    assert (got[:n_pos] != orc.NOT_FOUND).all()  # every haplotype k-mer is indexed
    sub_hits = (got[n_pos:n_pos + subs.shape[0] * 120] != orc.NOT_FOUND).mean()
    assert 0.2 < sub_hits < 0.95  # substituted reads mix found and absent k-mers


def test_search_reads_host_multi_replicas(cuda):
    """sbwt_search_reads_host_multi: the rows split into contiguous ranges of near-equal k-mer counts, one
    index replica per range, each writing its own slice of the answers.  Only one GPU is visible here, so
    the replicas share it (their pipelines are independent: no replica waits on another); the answers
    equal the oracle's for 1, 2 and 3 replicas, and a non-replica is refused."""
    rng = wl.rng_for(61)
    genome = wl.random_bases(rng, 150_000)
    built = sg.build_sbwt([genome.tobytes()], 31)
    files = list(wl.uneven_read_files(genome, seed=62, total_kmers=600_000, n_files=4))
    letters = np.concatenate([lt for lt, _ in files])
    rows, off = [np.zeros(1, dtype=np.uint64)], 0
    for lt, rw in files:
        rows.append(rw[1:].astype(np.uint64) + np.uint64(off))
        off += lt.size
    rows = np.concatenate(rows)
    want = orc.OracleIndex(built.bits, built.n_bits).search_reads(letters, rows, 31, 10)
    ixs = [sg.Index.from_bits(built.bits, built.n_bits, k=31, k_presearch=10) for _ in range(3)]
    try:
        for n in (1, 2, 3):
            got = sg.search_reads_host_multi(ixs[:n], letters, rows)
            assert np.array_equal(got, want), n
        other = sg.build_sbwt([genome[:50_000].tobytes()], 31)
        with sg.Index.from_bits(other.bits, other.n_bits, k=31, k_presearch=10) as bad:
            with pytest.raises(sg.SbwtError, match="not a replica"):
                sg.search_reads_host_multi([ixs[0], bad], letters, rows)
    finally:
        for ix in ixs:
            ix.close()
