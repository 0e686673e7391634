"""The CPU oracle, pinned against the reference's own code and fixtures (no GPU).

* rank structures: word for word against the reference's RankDataStructures
  compiled from its sources (oracle/_ref/ref_rank), for every superblock size
  and rank-structure kind the reference supports;
* search answers: against the stdout of the reference program itself
  (tests/golden/, produced by tests/golden/make_golden.py on a B200);
* search semantics: against the independent k-mer-set oracle.
"""
import gzip
import hashlib
import json
import os

import numpy as np
import pytest

import oracle as orc
import sbwt_gpu_b200 as sg
from sbwt_gpu_b200 import workloads as wl

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = sorted(os.listdir(os.path.join(GOLDEN, "cases")))


def _random_vector_file(tmp_path, n, density, seed, name="v"):
    rng = np.random.default_rng(seed)
    bits = rng.random(n) < density
    nbytes = (n + 7) // 8
    packed = np.packbits(bits)  # MSB first within each byte = the reference's file layout
    path = str(tmp_path / name)
    with open(path, "wb") as f:
        f.write(int(n).to_bytes(8, "little"))
        f.write(packed[:nbytes].tobytes())
    return path, bits


@pytest.mark.skipif(not orc.ref_rank_available(), reason="reference sources not built here")
@pytest.mark.parametrize("n", [1, 63, 64, 65, 255, 4095, 4096, 4097, 70_001, 1 << 20])
@pytest.mark.parametrize("sb,kind", orc.SB_KINDS)
def test_rank_build_matches_reference_code(tmp_path, n, sb, kind):
    path, _ = _random_vector_file(tmp_path, n, 0.3, n + sb)
    ref = orc.ref_rank(path, sb, kind, tmp_path)
    words, nb = orc.read_words(path)
    assert nb == n == ref["n"]
    assert np.array_equal(words, ref["words"])
    L0, L12, ones = orc.rank_build(words, n, sb, kind)
    assert np.array_equal(L0, ref["L0"])
    assert np.array_equal(L12, ref["L12"])
    assert ones == ref["ones"]


@pytest.mark.parametrize("sb,kind", orc.SB_KINDS)
def test_oracle_rank_is_popcount_prefix(tmp_path, sb, kind):
    n = 9_000
    path, bits = _random_vector_file(tmp_path, n, 0.45, sb * 7 + kind)
    words, _ = orc.read_words(path)
    ix = orc.OracleIndex([words] * 4, n, sb, kind)
    prefix = np.concatenate([[0], np.cumsum(bits)])
    for i in list(range(0, 300)) + list(range(n - 300, n + 1)) + [1023, 1024, 1025, 4095, 4096, 4097]:
        assert ix.rank(0, i) == prefix[i], i


def test_file_errors(tmp_path):
    short = tmp_path / "short"
    short.write_bytes(b"\x01\x02")
    assert orc.file_bits(str(short)) == -2
    zero = tmp_path / "zero"
    zero.write_bytes((0).to_bytes(8, "little"))
    assert orc.file_bits(str(zero)) == -3
    trunc = tmp_path / "trunc"
    trunc.write_bytes((100).to_bytes(8, "little") + b"\xff" * 5)
    assert orc.file_bits(str(trunc)) == -4
    assert orc.file_bits(str(tmp_path / "missing")) == -1


def test_read_queries_reference_semantics():
    k = 5
    data = b">h1\nACGTACGT\n>h2\nAC\n\nNNNNNNN\nacgtAC\n"
    letters, starts, nk = orc.read_queries(data, k)
    assert letters.tobytes() == b"ACGTACGTACNNNNNNNacgtAC"
    assert starts.tolist() == [0, 8, 10, 17, 23]
    assert nk == (8 - 4) + 0 + (7 - 4) + (6 - 4)
    # a final line without '\n' loses its last letter (kmer_search.hpp:328)
    letters, starts, nk = orc.read_queries(b">x\nACGTAC", k)
    assert letters.tobytes() == b"ACGTA" and starts.tolist() == [0, 5] and nk == 1
    # '\r' is a letter; '>' only counts at the start of a line
    letters, starts, nk = orc.read_queries(b"AC>GT\r\n", 3)
    assert letters.tobytes() == b"AC>GT\r" and nk == 4


def test_pack_layout():
    letters = np.frombuffer(b"ACGTNacgtx" * 7, dtype=np.uint8)
    words = orc.pack(letters)
    code = {ord("A"): 0, ord("C"): 1, ord("G"): 2, ord("T"): 3, ord("a"): 0, ord("c"): 1, ord("g"): 2, ord("t"): 3}
    assert words.size == (letters.size + 32 + 31) // 32
    for j, ch in enumerate(letters.tolist()):
        got = (int(words[j // 32]) >> (62 - 2 * (j % 32))) & 3
        assert got == code.get(ch, 0)
    assert int(words[-1]) == 0 or letters.size % 32 != 0


def test_oracle_search_matches_independent_definition():
    rng = wl.rng_for(99)
    for k, p in [(31, 10), (31, 0), (17, 6), (32, 12), (5, 3), (3, 0)]:
        genome = wl.random_bases(rng, 6000)
        built = sg.build_sbwt([genome.tobytes()], k)
        ox = orc.OracleIndex(built.bits, built.n_bits)
        letters, rows = wl.mixed_reads(rng, genome, 20, 20, 90, 0.02)
        ans = ox.search_reads(letters, rows, k, p)
        keys, dk, _ = orc.independent_sbwt([genome.tobytes()], k)
        want = orc.independent_answers(keys, dk, orc.query_colex_keys(orc.extract_kmers(letters, rows, k), k))
        assert np.array_equal(ans, want), (k, p)


@pytest.mark.parametrize("case", CASES)
def test_oracle_matches_reference_program_output(case):
    d = os.path.join(GOLDEN, "cases", case)
    ref_path = os.path.join(d, "reference.out.gz")
    if not os.path.exists(ref_path):
        pytest.skip("fixture not generated yet")
    meta = json.load(open(os.path.join(d, "case.json")))
    ref = gzip.open(ref_path).read()
    assert hashlib.sha256(ref).hexdigest() == meta["reference_sha256"]
    kind = orc.POPPY if meta["rank_structure"] == "poppy" else orc.CUM_POPPY
    ox = orc.OracleIndex.from_files([os.path.join(d, f"ix.{c}") for c in "ACGT"], meta["bits_in_superblock"], kind)
    letters, rows, nk = orc.read_queries(open(os.path.join(d, "queries.fa"), "rb").read(), meta["k"])
    ans = ox.search_reads(letters, rows, meta["k"], meta["p"])
    assert orc.format_answers(rows, meta["k"], ans) == ref


def test_oracle_matches_reference_program_small_workload(tmp_path):
    meta_p = os.path.join(GOLDEN, "small_workload.json")
    if not os.path.exists(meta_p):
        pytest.skip("fixture not generated yet")
    import make_golden
    meta = json.load(open(meta_p))
    n, letters, rows = make_golden.write_small_workload(str(tmp_path))
    ox = orc.OracleIndex.from_files([str(tmp_path / f"ix.{c}") for c in "ACGT"])
    l2, r2, nk = orc.read_queries(open(tmp_path / "queries.fa", "rb").read(), 31)
    assert np.array_equal(l2, letters) and np.array_equal(r2, rows)
    ans = ox.search_reads(letters, rows, 31, 10)
    text = orc.format_answers(rows, 31, ans)
    assert hashlib.sha256(text).hexdigest() == meta["reference_sha256"]
