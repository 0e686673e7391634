"""The host SBWT builder (product code, CPU only) against the SBWT definition."""
import os

import numpy as np
import pytest

import oracle as orc
import sbwt_gpu_b200 as sg
from sbwt_gpu_b200 import workloads as wl

ORDER = {"$": 0, "A": 1, "C": 2, "G": 3, "T": 4}


def strings_sbwt(seqs, k):
    """The SBWT by its definition on plain strings (tiny inputs only)."""
    K = set()
    for s in seqs:
        for i in range(len(s) - k + 1):
            w = s[i:i + k]
            if all(ch in "ACGT" for ch in w):
                K.add(w)
    suffixes = {x[1:] for x in K}
    nodes = set(K)
    nodes.add("$" * k)
    for x in K:
        if x[:-1] not in suffixes:
            for i in range(k):
                nodes.add("$" * (k - i) + x[:i])
    order = sorted(nodes, key=lambda v: [ORDER[ch] for ch in reversed(v)])
    index = {v: i for i, v in enumerate(order)}
    bits = np.zeros((4, len(order)), dtype=bool)
    seen = set()
    for v in order:
        suf = v[1:]
        if suf in seen:
            continue
        seen.add(suf)
        for c, ch in enumerate("ACGT"):
            if suf + ch in index:
                bits[c, index[v]] = True
    return order, bits


def unpack(words, n):
    w = np.asarray(words, dtype=np.uint64)
    out = np.zeros(n, dtype=bool)
    for p in range(n):
        out[p] = (int(w[p // 64]) >> (63 - p % 64)) & 1
    return out


@pytest.mark.parametrize("k", [3, 4, 7, 12])
@pytest.mark.parametrize("seed", [1, 2, 3])
def test_builder_matches_definition(k, seed):
    rng = np.random.default_rng(seed * 100 + k)
    seqs = ["".join(rng.choice(list("ACGT"), size=int(rng.integers(k, 60)))) for _ in range(int(rng.integers(1, 6)))]
    seqs.append("ACGTNACGTACGT"[: 4 + k])  # a k-mer holding N is skipped
    order, want = strings_sbwt(seqs, k)
    built = sg.build_sbwt(seqs, k)
    assert built.n_bits == len(order)
    for c in range(4):
        assert np.array_equal(unpack(built.bits[c], built.n_bits), want[c]), (c, seqs)
    # every non-root node has exactly one incoming 1
    assert sum(int(b.sum()) for b in want) == len(order) - 1


def test_builder_cycle_and_repeats():
    # a cyclic k-mer set has no source: the index is the root plus the k-mers
    k = 4
    s = "ACGTTGCA" * 4
    order, want = strings_sbwt([s], k)
    built = sg.build_sbwt([s], k)
    assert built.n_bits == len(order)
    for c in range(4):
        assert np.array_equal(unpack(built.bits[c], built.n_bits), want[c])


def test_builder_counts_match_independent_numpy():
    rng = wl.rng_for(5)
    g = wl.random_bases(rng, 200_000, gc=0.41)
    g = wl.with_repeats(rng, g, 10_000)
    built = sg.build_sbwt([g.tobytes()], 31)
    keys, dk, _ = orc.independent_sbwt([g.tobytes()], 31)
    assert built.n_kmers == keys.size
    assert built.n_dummies == dk.size
    ox = orc.OracleIndex(built.bits, built.n_bits)
    assert int(ox.C[4]) == built.n_bits  # 1 root + one incoming 1 per other node


def test_file_writer_round_trip(tmp_path):
    rng = wl.rng_for(8)
    g = wl.random_bases(rng, 5000)
    built = sg.build_sbwt([g.tobytes()], 31)
    paths = sg.write_index_files(str(tmp_path / "ix"), built)
    for c, path in enumerate(paths):
        words, n = orc.read_words(path)
        assert n == built.n_bits
        assert os.path.getsize(path) == 8 + (n + 7) // 8
        nw = (n + 63) // 64
        assert np.array_equal(words[:nw], built.bits[c][:nw])
        assert not words[nw:].any()


def test_builder_rejects_bad_k():
    with pytest.raises(sg.SbwtError):
        sg.build_sbwt(["ACGT"], 2)
    with pytest.raises(sg.SbwtError):
        sg.build_sbwt(["ACGT"], 33)
    with pytest.raises(sg.SbwtError, match="no k-mer"):
        sg.build_sbwt(["ACG"], 5)
