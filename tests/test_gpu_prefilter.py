"""The learned prefilter: tensor-core kernels vs the FP32 oracle, and the
sandwich guarantees (no indexed k-mer reported absent, answers identical to
the plain search).  Needs a B200.

Tolerances: the GPU and the oracle round to BF16 at the same points and
differ only in FP32 accumulation order, so a value near a BF16 rounding tie
can land one BF16 step (2^-8 relative) apart.  Logits must agree within
2e-2 absolute + 2e-2 relative; every gradient tensor within 2e-2 of the
oracle's in relative L2 norm.
"""
import numpy as np
import pytest

import mlp_oracle as mo
import oracle as orc
import sbwt_gpu_b200 as sg
from sbwt_gpu_b200 import workloads as wl

pytestmark = pytest.mark.gpu


def _rand_kmers(rng, n, k):
    mask = np.uint64(((1 << (2 * k)) - 1) << (64 - 2 * k)) if k < 32 else np.uint64(0xFFFFFFFFFFFFFFFF)
    return rng.integers(0, 2**63, size=n, dtype=np.int64).astype(np.uint64) * np.uint64(2) & mask


@pytest.mark.parametrize("k", [31, 15, 32])
def test_fused_inference_matches_oracle(cuda, k):
    rng = np.random.default_rng(k)
    theta = mo.init_like(seed=k, k=k)
    kmers = _rand_kmers(rng, 1000, k)  # not a multiple of the 128-row tile
    got = sg.mlp_logits(k, theta, kmers)
    want, _ = mo.forward(theta, kmers, k)
    assert np.allclose(got, want, rtol=2e-2, atol=2e-2), np.abs(got - want).max()


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


@pytest.mark.parametrize("n", [256, 2048])
def test_training_gradients_match_oracle(cuda, n):
    rng = np.random.default_rng(n)
    k = 31
    theta = mo.init_like(seed=n, k=k)
    kmers = _rand_kmers(rng, n, k)
    labels = (rng.random(n) < 0.4).astype(np.uint8)
    loss, g = sg.mlp_gradients(k, theta, kmers, labels)
    wl_, wg = mo.loss_and_grad(theta, kmers, labels, k)
    assert abs(loss - wl_) < 1e-3 * max(1.0, abs(wl_))
    for name, a, b in [("W1", 0, 32768), ("b1", 32768, 33024), ("W2", 33024, 98560), ("b2", 98560, 98816),
                       ("w3", 98816, 99072), ("b3", 99072, 99073)]:
        assert _rel(g[a:b], wg[a:b]) < 2e-2, (name, _rel(g[a:b], wg[a:b]))
    assert not g[0:32768].reshape(256, 128)[:, 4 * k:].any()  # padded inputs get no gradient


@pytest.fixture(scope="module")
def trained(cuda):
    # A GC-rich genome: uniform random negatives differ from indexed k-mers in
    # composition, which the network can learn; membership in a uniform random
    # k-mer set carries no such signal.
    rng = wl.rng_for(4040)
    k = 31
    genome = wl.random_bases(rng, 60_000, gc=0.9)
    built = sg.build_sbwt([genome.tobytes()], k)
    ix = sg.Index.from_bits(built.bits, built.n_bits, k=k, k_presearch=10)
    pf = sg.Prefilter.train(ix, steps=400, batch=2048, n_positive=400_000, n_negative=400_000, seed=9)
    yield {"ix": ix, "pf": pf, "genome": genome, "built": built, "k": k}
    pf.close()
    ix.close()


def test_training_reduces_loss(trained):
    st = trained["pf"].stats()
    assert st["final_loss"] < 0.9 * st["first_loss"]
    # half of the negatives (uniform random) are separable by composition; the
    # mutated half is not: about 0.75 is reachable, 0.5 is chance
    assert st["train_accuracy"] > 0.65
    assert 0.3 < st["label_positive_fraction"] < 0.7
    assert st["n_indexed_kmers"] == trained["built"].n_kmers
    assert st["bloom_bits"] >= 1024


def test_sandwich_is_bit_exact_and_never_drops_an_indexed_kmer(trained, cuda):
    import torch
    ix, pf, k = trained["ix"], trained["pf"], trained["k"]
    rng = wl.rng_for(5)
    letters, rows = wl.kmer_queries(rng, trained["genome"], 20_000, k, neg_frac=0.9)
    kmers = orc.extract_kmers(letters, rows, k)
    d_k = torch.from_numpy(kmers.view(np.int64)).to(cuda)
    plain = torch.empty_like(d_k)
    filt = torch.full_like(d_k, -5)
    ix.search_kmers(d_k, plain)
    skipped = ix.search_kmers_filtered(pf, d_k, filt)
    torch.cuda.synchronize()
    p, f = plain.cpu().numpy().view(np.uint64), filt.cpu().numpy().view(np.uint64)
    assert np.array_equal(p, f)
    ox = orc.OracleIndex(trained["built"].bits, trained["built"].n_bits)
    words = np.append(kmers, np.uint64(0))  # one padding word after the last k-mer
    assert np.array_equal(p, ox.search_positions(words, np.arange(kmers.size, dtype=np.uint64) * np.uint64(32), k, 10))
    assert skipped > 0
    # every indexed k-mer passes the sandwich (false-absent = 0)
    keys, dk, _ = orc.independent_sbwt([trained["genome"].tobytes()], k)
    g = trained["genome"]
    all_rows = np.array([0, g.size], dtype=np.uint64)
    all_kmers = orc.extract_kmers(g, all_rows, k)
    d_all = torch.from_numpy(all_kmers.view(np.int64)).to(cuda)
    out = torch.empty_like(d_all)
    ix.search_kmers_filtered(pf, d_all, out)
    torch.cuda.synchronize()
    assert (out.cpu().numpy().view(np.uint64) != orc.NOT_FOUND).all()


def test_prefilter_logits_api(trained, cuda):
    import torch
    pf, k = trained["pf"], trained["k"]
    theta = pf.params()
    rng = np.random.default_rng(3)
    kmers = _rand_kmers(rng, 777, k)
    d_k = torch.from_numpy(kmers.view(np.int64)).to(cuda)
    d_l = torch.empty(777, dtype=torch.float32, device=cuda)
    pf.logits(d_k, d_l)
    torch.cuda.synchronize()
    want, _ = mo.forward(theta, kmers, k)
    assert np.allclose(d_l.cpu().numpy(), want, rtol=2e-2, atol=2e-2)


def _auc(pos, neg):
    """Probability that a positive's logit exceeds a negative's (ties count half)."""
    allv = np.concatenate([pos, neg])
    ranks = np.argsort(np.argsort(allv, kind="mergesort"), kind="mergesort").astype(np.float64) + 1
    return (ranks[: pos.size].sum() - pos.size * (pos.size + 1) / 2) / (pos.size * neg.size)


def test_trained_network_gains_over_the_untrained_one(trained, cuda):
    """What training buys over the same sandwich with the untrained (initial) network, at the
    same threshold and Bloom settings: the trained network separates indexed k-mers from random
    ones (AUC) and sends far fewer indexed k-mers to the backup Bloom filter, so the filter that
    keeps the sandwich exact is many times smaller for the same false-positive rate.  (The
    untrained network rejects about half of everything at random, so its sandwich skips a
    similar share of a 90%-negative query set, but only by carrying most of the index in its
    Bloom filter.)"""
    import torch
    ix, pf, k = trained["ix"], trained["pf"], trained["k"]
    with sg.Prefilter.train(ix, steps=0, batch=2048, n_positive=400_000, n_negative=400_000, seed=9) as base:
        g = trained["genome"]
        pos = orc.extract_kmers(g, np.array([0, g.size], dtype=np.uint64), k)[:20_000]
        neg = _rand_kmers(np.random.default_rng(8), 20_000, k)
        out = {}
        for name, f in (("trained", pf), ("untrained", base)):
            d = torch.from_numpy(np.concatenate([pos, neg]).view(np.int64)).to(cuda)
            lg = torch.empty(d.numel(), dtype=torch.float32, device=cuda)
            f.logits(d, lg)
            torch.cuda.synchronize()
            lg = lg.cpu().numpy()
            rng = wl.rng_for(5)
            letters, rows = wl.kmer_queries(rng, g, 20_000, k, neg_frac=0.9)
            qk = torch.from_numpy(orc.extract_kmers(letters, rows, k).view(np.int64)).to(cuda)
            ans = torch.empty_like(qk)
            skipped = ix.search_kmers_filtered(f, qk, ans)
            out[name] = {"auc": _auc(lg[: pos.size], lg[pos.size:]), "skip": skipped / qk.numel(),
                         "rejected_indexed": f.stats()["n_rejected_indexed"]}
    t, u = out["trained"], out["untrained"]
    assert t["auc"] > 0.95 and t["auc"] > u["auc"] + 0.2, out
    assert t["rejected_indexed"] < 0.25 * u["rejected_indexed"], out
    assert t["skip"] > 0.3 and u["skip"] > 0, out


def _concat_files(files):
    letters = np.concatenate([lt for lt, _ in files])
    rows, off = [np.zeros(1, dtype=np.uint64)], 0
    for lt, rw in files:
        rows.append(rw[1:].astype(np.uint64) + np.uint64(off))
        off += lt.size
    return letters, np.concatenate(rows)


def _filtered_vs_oracle(ix, pf, built, letters, rows, k, p, cuda, monkeypatch=None, chunk=None):
    import torch
    if chunk is not None:
        monkeypatch.setenv("SBWT_FILTER_CHUNK_KMERS", str(chunk))
    nk = sg.count_kmers(rows, k)
    d_l = torch.from_numpy(letters).to(cuda)
    d_r = torch.from_numpy(rows.view(np.int64)).to(cuda)
    filt = torch.full((nk,), -5, dtype=torch.int64, device=cuda)
    bits = torch.full(((nk + 31) // 32,), -1, dtype=torch.int32, device=cuda)
    skipped = ix.search_reads_filtered(pf, d_l, d_r, filt, nk, d_member_bits=bits)
    only = torch.full(((nk + 31) // 32,), -1, dtype=torch.int32, device=cuda)  # membership only
    ix.search_reads_filtered(pf, d_l, d_r, None, nk, d_member_bits=only)
    torch.cuda.synchronize()
    want = orc.OracleIndex(built.bits, built.n_bits).search_reads(letters, rows, k, p)
    got = filt.cpu().numpy().view(np.uint64)
    assert np.array_equal(got, want)  # bit-exact, so no indexed k-mer is reported absent
    full = nk // 32
    hit = np.zeros((nk + 31) // 32 * 32, dtype=bool)
    hit[:nk] = want != orc.NOT_FOUND
    want_bits = np.packbits(hit.reshape(-1, 32)[:, ::-1], axis=1).view(">u4").reshape(-1).astype(np.uint32)
    assert np.array_equal(bits.cpu().numpy().view(np.uint32)[:full], want_bits[:full])
    assert np.array_equal(only.cpu().numpy().view(np.uint32)[:full], want_bits[:full])
    return skipped, nk, want


def test_filtered_reads_batched_uneven_shape(trained, cuda, monkeypatch):
    """The prefiltered search of reads (sbwt_search_reads_filtered) on the batched-uneven shape: 64 files of
    150 bp / lognormal 2 kbp / lognormal 15 kbp reads, 30% genome reads with 2% substitutions, in one batch;
    the inference runs in several chunks (a small chunk size), and the answers equal the oracle's."""
    ix, pf, k = trained["ix"], trained["pf"], trained["k"]
    files = list(wl.uneven_read_files(trained["genome"], seed=77, total_kmers=400_000, n_files=64))
    letters, rows = _concat_files(files)
    skipped, nk, want = _filtered_vs_oracle(ix, pf, trained["built"], letters, rows, k, 10, cuda, monkeypatch,
                                            chunk=50_000)
    assert 0 < skipped < nk
    assert skipped <= int((want == orc.NOT_FOUND).sum())


def test_filtered_reads_pangenome_shape(cuda):
    """Pangenome shape: union index of 20 haplotypes, a prefilter trained on that index, 150 bp and
    lognormal ~10 kbp reads with 95% random reads; answers equal the oracle's."""
    rng = wl.rng_for(52)
    k = 31
    base = wl.random_bases(rng, 40_000, gc=0.41)
    haps = wl.haplotypes(rng, base, 20)
    built = sg.build_sbwt([h.tobytes() for h in haps], k)
    lens = [150 if rng.random() < 0.9 else int(min(30_000, max(31, rng.lognormal(np.log(10_000), 0.5))))
            for _ in range(600)]
    rows = np.zeros(len(lens) + 1, dtype=np.uint64)
    rows[1:] = np.cumsum(lens)
    letters = wl.ACGT[rng.integers(0, 4, size=int(rows[-1]), dtype=np.uint8)]
    for r in np.flatnonzero(rng.random(len(lens)) < 0.05).tolist():
        h = haps[r % 20]
        a, b = int(rows[r]), int(rows[r + 1])
        s0 = int(rng.integers(0, h.size - (b - a) + 1)) if b - a <= h.size else 0
        if b - a <= h.size:
            letters[a:b] = wl.substitute(rng, h[s0:s0 + (b - a)].copy()[None, :], 0.01)[0]
    with sg.Index.from_bits(built.bits, built.n_bits, k=k, k_presearch=12) as ix:
        with sg.Prefilter.train(ix, steps=300, batch=2048, n_positive=300_000, n_negative=300_000, seed=3) as pf:
            skipped, nk, want = _filtered_vs_oracle(ix, pf, built, letters, rows, k, 12, cuda)
    assert 0 < skipped < nk


def test_sandwich_holds_when_the_index_has_more_kmers_than_the_training_set(cuda):
    """The backup Bloom filter covers every indexed k-mer the model rejects, also when the index has more
    k-mers than the training set has samples (the count of indexed k-mers must not use the training
    labels' buffer).  With tau far above any logit the model rejects every k-mer, so the filter must
    hold all of them and the answers must still equal the oracle's."""
    rng = wl.rng_for(57)
    k = 31
    genome = wl.random_bases(rng, 300_000)
    built = sg.build_sbwt([genome.tobytes()], k)
    letters, rows = wl.mixed_reads(rng, genome, 400, 400, 150, 0.01)
    with sg.Index.from_bits(built.bits, built.n_bits, k=k, k_presearch=10) as ix:
        with sg.Prefilter.train(ix, steps=5, batch=2048, n_positive=4096, n_negative=4096, seed=5,
                                tau=1e9) as pf:
            st = pf.stats()
            assert st["n_train"] == 8192 < built.n_bits // 10
            assert st["n_rejected_indexed"] == st["n_indexed_kmers"] > 250_000
            skipped, nk, want = _filtered_vs_oracle(ix, pf, built, letters, rows, k, 10, cuda)
    assert (want != orc.NOT_FOUND).any() and 0 < skipped < nk
