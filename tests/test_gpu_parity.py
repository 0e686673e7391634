"""CUDA path vs the oracle, bit for bit, through the C ABI (needs a B200)."""
import gzip
import hashlib
import json
import os
import subprocess

import numpy as np
import pytest

import oracle as orc
import sbwt_gpu_b200 as sg
from sbwt_gpu_b200 import workloads as wl

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = sorted(os.listdir(os.path.join(GOLDEN, "cases")))


def _t(a, dev):
    import torch
    a = np.ascontiguousarray(a)
    if a.dtype == np.uint64:
        a = a.view(np.int64)
    return torch.from_numpy(a).to(dev)


def _u64(t):
    return t.cpu().numpy().view(np.uint64)


@pytest.fixture(scope="module")
def small(cuda):
    rng = wl.rng_for(4242)
    k = 31
    genome = wl.random_bases(rng, 120_000)
    built = sg.build_sbwt([genome.tobytes()], k)
    letters, rows = wl.mixed_reads(rng, genome, 300, 300, 150, 0.01)
    return {"k": k, "genome": genome, "built": built, "letters": letters, "rows": rows}


def run_reads(ix, letters, rows, dev, n_kmers=None, member=False):
    import torch
    nk = sg.count_kmers(rows, ix.info()["k"]) if n_kmers is None else n_kmers
    d_ans = torch.full((max(nk, 1),), -7, dtype=torch.int64, device=dev)
    d_mem = torch.zeros(((nk + 31) // 32 + 1,), dtype=torch.int32, device=dev) if member else None
    ix.search_reads(_t(letters, dev), _t(rows, dev), d_ans, nk, d_member_bits=d_mem)
    torch.cuda.synchronize()
    out = _u64(d_ans)[:nk]
    return (out, d_mem.cpu().numpy().view(np.uint32)) if member else out


@pytest.mark.parametrize("sb,kind", orc.SB_KINDS)
def test_gpu_rank_build_matches_reference_layout(small, sb, kind):
    b = small["built"]
    ox = orc.OracleIndex(b.bits, b.n_bits, sb, kind)
    with sg.Index.from_bits(b.bits, b.n_bits, k=31, k_presearch=0) as ix:
        for c in range(4):
            L0, L12 = ix.rank_structures(sb, kind, c)
            assert np.array_equal(L0, ox.L0[c]), (sb, kind, c)
            assert np.array_equal(L12, ox.L12[c]), (sb, kind, c)


def test_c_array(small):
    b = small["built"]
    ox = orc.OracleIndex(b.bits, b.n_bits)
    with sg.Index.from_bits(b.bits, b.n_bits, k=31) as ix:
        assert ix.info()["C"] == [int(x) for x in ox.C]


@pytest.mark.parametrize("p", [1, 2, 5, 9, 12])
def test_presearch_table_matches_oracle(small, p):
    b = small["built"]
    ox = orc.OracleIndex(b.bits, b.n_bits)
    with sg.Index.from_bits(b.bits, b.n_bits, k=31, k_presearch=p) as ix:
        lefts, rights = ix.presearch_table()
    wl_, wr = ox.presearch(p)
    assert np.array_equal(lefts, wl_)
    assert np.array_equal(rights, wr)


@pytest.mark.parametrize("p", [13, 14])
def test_deep_presearch_table_matches_oracle_on_a_sample(small, p):
    """p = 13 and 14 (the depths the autotuner and the pangenome workload use): the whole GPU table is
    exported; the oracle restates 2M sampled entries plus both ends of the table."""
    b = small["built"]
    ox = orc.OracleIndex(b.bits, b.n_bits)
    with sg.Index.from_bits(b.bits, b.n_bits, k=31, k_presearch=p) as ix:
        lefts, rights = ix.presearch_table()
    n = 1 << (2 * p)
    assert lefts.size == n and rights.size == n
    rng = np.random.default_rng(p)
    idx = np.concatenate([np.arange(1024, dtype=np.uint64), np.arange(n - 1024, n, dtype=np.uint64),
                          rng.integers(0, n, size=2_000_000, dtype=np.uint64)])
    wl_, wr = ox.presearch_at(p, idx)
    assert np.array_equal(lefts[idx], wl_)
    assert np.array_equal(rights[idx], wr)
    # every non-empty entry lies inside the index
    ne = lefts <= rights
    assert ne.any() and int(rights[ne].max()) < b.n_bits


def test_search_packed_reference_contract(small, cuda):
    b, k = small["built"], small["k"]
    ox = orc.OracleIndex(b.bits, b.n_bits)
    words = orc.pack(small["letters"])
    pos = orc.positions(small["rows"], k)
    want = ox.search_positions(words, pos, k, 10)
    with sg.Index.from_bits(b.bits, b.n_bits, k=k, k_presearch=10) as ix:
        d_words = _t(words, cuda)
        d_pos = _t(pos, cuda)
        ix.search_packed(d_words, d_pos)
        import torch
        torch.cuda.synchronize()
        assert np.array_equal(_u64(d_pos), want)


def test_pack_kernel_matches_oracle(cuda):
    import torch
    rng = np.random.default_rng(3)
    for n in [0, 1, 31, 32, 33, 1000, 4097]:
        letters = rng.choice(np.frombuffer(b"ACGTacgtNnRX\r>", dtype=np.uint8), size=n)
        want = orc.pack(letters)
        from ctypes import c_void_p
        for off in (0, 3):  # aligned (16-byte loads) and unaligned (byte loads)
            buf = torch.zeros(n + 64, dtype=torch.uint8, device=cuda)
            if n:
                buf[off:off + n] = _t(letters, cuda)
            d_words = torch.full((want.size,), -1, dtype=torch.int64, device=cuda)
            rc = sg._lib.lib.sbwt_pack(c_void_p(buf.data_ptr() + off), n, c_void_p(d_words.data_ptr()), None)
            assert rc == 0
            torch.cuda.synchronize()
            assert np.array_equal(_u64(d_words), want), (n, off)


SHAPES = [(0, 1)] + [(kpt, tpk) for kpt in (1, 2, 3, 4, 6, 8) for tpk in (1, 2, 4)]


@pytest.mark.parametrize("kpt,tpk", SHAPES)
def test_search_reads_line_layout_all_shapes(small, cuda, kpt, tpk):
    b, k = small["built"], small["k"]
    ox = orc.OracleIndex(b.bits, b.n_bits)
    want = ox.search_reads(small["letters"], small["rows"], k, 10)
    with sg.Index.from_bits(b.bits, b.n_bits, k=k, k_presearch=10) as ix:
        ix.configure(sg.SBWT_LAYOUT_LINES, kmers_per_thread=kpt, threads_per_kmer=tpk, threads_per_block=128)
        got = run_reads(ix, small["letters"], small["rows"], cuda)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("sb,kind", orc.SB_KINDS)
@pytest.mark.parametrize("shuffles,kpt", [(0, 0), (0, 2), (1, 2)])
def test_search_reads_poppy_layout(small, cuda, sb, kind, shuffles, kpt):
    b, k = small["built"], small["k"]
    ox = orc.OracleIndex(b.bits, b.n_bits)
    want = ox.search_reads(small["letters"], small["rows"], k, 8)
    with sg.Index.from_bits(b.bits, b.n_bits, k=k, k_presearch=8) as ix:
        ix.configure(sg.SBWT_LAYOUT_POPPY, bits_in_superblock=sb, rank_structure=kind, with_shuffles=shuffles,
                     kmers_per_thread=kpt)
        got = run_reads(ix, small["letters"], small["rows"], cuda)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("p", [0, 1, 4, 7, 10, 13, 15])
def test_answers_do_not_depend_on_p(small, cuda, p):
    b, k = small["built"], small["k"]
    ox = orc.OracleIndex(b.bits, b.n_bits)
    want = ox.search_reads(small["letters"], small["rows"], k, 0)
    with sg.Index.from_bits(b.bits, b.n_bits, k=k, k_presearch=p) as ix:
        got = run_reads(ix, small["letters"], small["rows"], cuda)
    assert np.array_equal(got, want)


def test_member_bits(small, cuda):
    b, k = small["built"], small["k"]
    with sg.Index.from_bits(b.bits, b.n_bits, k=k, k_presearch=10) as ix:
        ans, bits = run_reads(ix, small["letters"], small["rows"], cuda, member=True)
    nk = ans.size
    want = np.zeros((nk + 31) // 32 * 32, dtype=bool)
    want[:nk] = ans != orc.NOT_FOUND
    w = want.reshape(-1, 32).astype(np.uint64)
    words = (w << np.arange(32, dtype=np.uint64)).sum(axis=1).astype(np.uint32)  # bit j%32 of word j/32
    assert np.array_equal(bits[: words.size], words)


@pytest.mark.parametrize("k,p", [(3, 0), (3, 3), (4, 2), (9, 5), (17, 8), (25, 9), (31, 31), (32, 12), (32, 0)])
def test_k_and_p_range(cuda, k, p):
    rng = wl.rng_for(1000 + k)
    genome = wl.random_bases(rng, 8000)
    built = sg.build_sbwt([genome.tobytes()], k)
    letters, rows = wl.mixed_reads(rng, genome, 40, 40, 70, 0.02)
    ox = orc.OracleIndex(built.bits, built.n_bits)
    want = ox.search_reads(letters, rows, k, min(p, 15))
    keys, dk, _ = orc.independent_sbwt([genome.tobytes()], k)
    assert np.array_equal(want, orc.independent_answers(keys, dk, orc.query_colex_keys(
        orc.extract_kmers(letters, rows, k), k)))
    with sg.Index.from_bits(built.bits, built.n_bits, k=k, k_presearch=min(p, 15)) as ix:
        got = run_reads(ix, letters, rows, cuda)
    assert np.array_equal(got, want)


def test_ragged_rows_and_odd_bytes(small, cuda):
    """Reads shorter than k, empty reads, N and lowercase letters, one-letter reads."""
    b, k = small["built"], small["k"]
    rng = np.random.default_rng(11)
    g = small["genome"]
    parts = [g[100:400], np.frombuffer(b"ACG", np.uint8), np.zeros(0, np.uint8), g[5000:5031],
             np.frombuffer(b"NNNNNNNNNNNNNNNNNNNNNNNNNNNNNNNNNNNNNN", np.uint8),
             np.frombuffer(g[7000:7100].tobytes().lower(), np.uint8), g[9000:9030], np.frombuffer(b"A", np.uint8),
             rng.choice(np.frombuffer(b"ACGTN", np.uint8), size=500)]
    letters = np.concatenate(parts)
    rows = np.zeros(len(parts) + 1, dtype=np.uint64)
    rows[1:] = np.cumsum([p.size for p in parts])
    ox = orc.OracleIndex(b.bits, b.n_bits)
    want = ox.search_reads(letters, rows, k, 10)
    with sg.Index.from_bits(b.bits, b.n_bits, k=k, k_presearch=10) as ix:
        got = run_reads(ix, letters, rows, cuda)
        host = ix.search_reads_host(letters, rows)
    assert np.array_equal(got, want)
    assert np.array_equal(host, want)
    assert (want[: 300 - k + 1] != orc.NOT_FOUND).all()  # an exact genome substring is present


def test_n_kmers_smaller_than_rows_hold(small, cuda):
    b, k = small["built"], small["k"]
    ox = orc.OracleIndex(b.bits, b.n_bits)
    want = ox.search_reads(small["letters"], small["rows"], k, 10)
    with sg.Index.from_bits(b.bits, b.n_bits, k=k, k_presearch=10) as ix:
        got = run_reads(ix, small["letters"], small["rows"], cuda, n_kmers=1000)
    assert np.array_equal(got, want[:1000])


def test_search_reads_host_pinned_and_pageable(small, cuda):
    import torch
    b, k = small["built"], small["k"]
    ox = orc.OracleIndex(b.bits, b.n_bits)
    want = ox.search_reads(small["letters"], small["rows"], k, 10)
    with sg.Index.from_bits(b.bits, b.n_bits, k=k, k_presearch=10) as ix:
        got = ix.search_reads_host(small["letters"], small["rows"])
        assert np.array_equal(got, want)
        pl = torch.from_numpy(small["letters"]).pin_memory()
        pr = torch.from_numpy(small["rows"].view(np.int64)).pin_memory()
        pa = torch.empty(want.size, dtype=torch.int64).pin_memory()
        ix.search_reads_host(pl, pr, pa)
        assert np.array_equal(pa.numpy().view(np.uint64), want)


def test_small_workload_full(cuda, tmp_path):
    import make_golden
    n, letters, rows = make_golden.write_small_workload(str(tmp_path))
    paths = [str(tmp_path / f"ix.{c}") for c in "ACGT"]
    ox = orc.OracleIndex.from_files(paths)
    want = ox.search_reads(letters, rows, 31, 10)
    with sg.Index.load(*paths, k=31, k_presearch=10) as ix:
        got = run_reads(ix, letters, rows, cuda)
        host = ix.search_reads_host(letters, rows)
    assert np.array_equal(got, want)
    assert np.array_equal(host, want)
    meta_p = os.path.join(GOLDEN, "small_workload.json")
    if os.path.exists(meta_p):
        text = sg.format_answers(rows, 31, got)
        assert hashlib.sha256(text).hexdigest() == json.load(open(meta_p))["reference_sha256"]


@pytest.mark.parametrize("fmt,batch", [("fasta", 0), ("fastq", 0), ("fastq", 100_000), ("fasta", 77_777)])
def test_cli_streams_fasta_and_fastq(cuda, tmp_path, fmt, batch):
    """The CLI reads its query file on a thread of its own in batches of whole reads while the
    previous batch is searched; FASTQ input (no reference counterpart) gives the same output as the
    FASTA file of the same reads.  On the small workload (1.2M k-mers), over up to ~20 batches, the
    output's SHA-256 equals that of the reference program's output on the FASTA file."""
    import make_golden
    n, letters, rows = make_golden.write_small_workload(str(tmp_path))
    q = str(tmp_path / "queries.fa")
    if fmt == "fastq":
        q = str(tmp_path / "queries.fq")
        wl.write_fastq(q, letters, rows)
    flags = [f if not f.startswith("--file-queries=") else f"--file-queries={q}"
             for f in make_golden.small_workload_flags(str(tmp_path))]
    env = dict(os.environ)
    if batch:
        env["SBWT_CLI_BATCH_LETTERS"] = str(batch)
    r = subprocess.run([sg.CLI_PATH] + flags, capture_output=True, timeout=300, env=env)
    assert r.returncode == 0, r.stderr.decode()
    want = orc.format_answers(rows, 31, orc.OracleIndex.from_files([str(tmp_path / f"ix.{c}") for c in "ACGT"])
                              .search_reads(letters, rows, 31, 10))
    assert r.stdout == want
    meta_p = os.path.join(GOLDEN, "small_workload.json")
    if os.path.exists(meta_p):
        assert hashlib.sha256(r.stdout).hexdigest() == json.load(open(meta_p))["reference_sha256"]


@pytest.mark.parametrize("case", CASES)
def test_cli_matches_reference_program(case, cuda):
    d = os.path.join(GOLDEN, "cases", case)
    meta = json.load(open(os.path.join(d, "case.json")))
    import make_golden
    flags = make_golden.case_flags(case, os.path.join(GOLDEN, "cases"))
    ref_path = os.path.join(d, "reference.out.gz")
    if os.path.exists(ref_path):
        want = gzip.open(ref_path).read()
    else:
        kind = orc.POPPY if meta["rank_structure"] == "poppy" else orc.CUM_POPPY
        ox = orc.OracleIndex.from_files([os.path.join(d, f"ix.{c}") for c in "ACGT"], meta["bits_in_superblock"],
                                        kind)
        letters, rows, _ = orc.read_queries(open(os.path.join(d, "queries.fa"), "rb").read(), meta["k"])
        want = orc.format_answers(rows, meta["k"], ox.search_reads(letters, rows, meta["k"], meta["p"]))
    for layout in ("lines", "poppy"):
        r = subprocess.run([sg.CLI_PATH] + flags + [f"--layout={layout}"], capture_output=True, timeout=300)
        assert r.returncode == 0, r.stderr.decode()
        assert r.stdout == want, (case, layout)


def test_index_load_errors(tmp_path, cuda):
    b = sg.build_sbwt(["ACGTACGTTTGACCA" * 3], 5)
    paths = sg.write_index_files(str(tmp_path / "ix"), b)
    other = sg.build_sbwt(["ACGTACGTTTGACCAGG" * 3], 5)
    p2 = sg.write_index_files(str(tmp_path / "other"), other)
    with pytest.raises(sg.SbwtError, match="different lengths"):
        sg.Index.load(paths[0], paths[1], paths[2], p2[3], k=5, k_presearch=0)
    with pytest.raises(sg.SbwtError):
        sg.Index.load(paths[0], paths[1], paths[2], str(tmp_path / "missing"), k=5)
    bad = tmp_path / "bad"
    bad.write_bytes((10_000).to_bytes(8, "little") + b"\0" * 10)
    with pytest.raises(sg.SbwtError):
        sg.Index.load(str(bad), str(bad), str(bad), str(bad), k=5)


def test_autotune_keeps_answers_and_picks_a_shape(small, cuda):
    import torch
    b, k = small["built"], small["k"]
    ox = orc.OracleIndex(b.bits, b.n_bits)
    want = ox.search_reads(small["letters"], small["rows"], k, 10)
    with sg.Index.from_bits(b.bits, b.n_bits, k=k, k_presearch=10) as ix:
        d_ans = torch.empty(want.size, dtype=torch.int64, device=cuda)
        rep = ix.autotune(_t(small["letters"], cuda), _t(small["rows"], cuda), d_ans, want.size, tune_p=True,
                          tune_poppy=True)
        assert rep["best"]["ms"] > 0 and rep["default_ms"] > 0 and len(rep["candidates"]) >= 15
        layouts = {c["layout"] for c in rep["candidates"]}
        assert {"lines", "lines512", "lines2048", "poppy"} <= layouts
        if any(c["layout"] == "lines" and c["window"] != 128 for c in rep["candidates"]) or \
                rep["best"]["layout"] == "lines":  # the windows are a knob of the 32-byte line layout
            assert {c["window"] for c in rep["candidates"]} >= {64, 128, 256}
        assert {c["p"] for c in rep["candidates"]} >= {8, 10, 12, 14}
        got = run_reads(ix, small["letters"], small["rows"], cuda)
        # with the per-k-mer kernel's register shapes as well
        rep2 = ix.autotune(_t(small["letters"], cuda), _t(small["rows"], cuda), d_ans, want.size, tune_shapes=True)
        assert sum(1 for c in rep2["candidates"] if c["kmers_per_thread"] > 0) >= 36
        got2 = run_reads(ix, small["letters"], small["rows"], cuda)
    assert np.array_equal(got, want)
    assert np.array_equal(got2, want)


def test_graph_replay_matches(small, cuda):
    import torch
    b, k = small["built"], small["k"]
    ox = orc.OracleIndex(b.bits, b.n_bits)
    want = ox.search_reads(small["letters"], small["rows"], k, 10)
    s = torch.cuda.Stream(device=cuda)
    with sg.Index.from_bits(b.bits, b.n_bits, k=k, k_presearch=10) as ix:
        ix.use_graphs(True)
        d_l, d_r = _t(small["letters"], cuda), _t(small["rows"], cuda)
        for rep in range(3):
            d_ans = torch.full((want.size,), -1, dtype=torch.int64, device=cuda)
            with torch.cuda.stream(s):
                ix.search_reads(d_l, d_r, d_ans, want.size, stream=s)
            s.synchronize()
            assert np.array_equal(_u64(d_ans), want), rep
        # same buffers again: the captured graph is replayed
        d_ans.fill_(-1)
        ix.search_reads(d_l, d_r, d_ans, want.size, stream=s)
        s.synchronize()
        assert np.array_equal(_u64(d_ans), want)
        ix.presearch(7)  # the index changed: the graph is re-captured
        d_ans.fill_(-1)
        ix.search_reads(d_l, d_r, d_ans, want.size, stream=s)
        s.synchronize()
        assert np.array_equal(_u64(d_ans), want)


def test_l2_fetch_granularity(small, cuda):
    b = small["built"]
    with sg.Index.from_bits(b.bits, b.n_bits, k=31) as ix:
        for v in (32, 64, 128):
            ix.set_l2_fetch_granularity(v)
        with pytest.raises(sg.SbwtError):
            ix.set_l2_fetch_granularity(48)


def test_many_files_one_batch(small, cuda, tmp_path):
    b, k = small["built"], small["k"]
    ox = orc.OracleIndex(b.bits, b.n_bits)
    rng = wl.rng_for(77)
    paths, wants = [], []
    for f in range(5):
        letters, rows = wl.mixed_reads(rng, small["genome"], 10 + f, 10, 60 + 40 * f, 0.01)
        p = str(tmp_path / f"q{f}.fa")
        wl.write_fasta(p, letters, rows)
        paths.append(p)
        wants.append(ox.search_reads(letters, rows, k, 10))
    letters, rows, nk, file_rows = sg.read_queries_many(paths, k)
    with sg.Index.from_bits(b.bits, b.n_bits, k=k, k_presearch=10) as ix:
        got = run_reads(ix, letters, rows, cuda)
    assert np.array_equal(got, np.concatenate(wants))


def _row_mixture(rng, genome, k):
    """Rows of every length class the run walk cuts differently: shorter than k, exactly k
    (one k-mer), a window and a bit, long genome substrings (every k-mer present), random
    and mutated reads, and many one-k-mer rows in a row."""
    parts = []
    for n in [k - 1, k, k + 1, 2 * k, k + 33, k + 64, 1000, 5000]:
        s = int(rng.integers(0, genome.size - n))
        parts.append(genome[s:s + n])
        parts.append(wl.random_bases(rng, n))
        mut = genome[s:s + n].copy()
        hits = rng.random(n) < 0.02
        mut[hits] = rng.choice(np.frombuffer(b"ACGT", np.uint8), size=int(hits.sum()))
        parts.append(mut)
    for _ in range(300):
        s = int(rng.integers(0, genome.size - k))
        parts.append(genome[s:s + k] if rng.random() < 0.5 else wl.random_bases(rng, k))
    letters = np.concatenate(parts)
    rows = np.zeros(len(parts) + 1, dtype=np.uint64)
    rows[1:] = np.cumsum([p.size for p in parts])
    return letters, rows


@pytest.mark.parametrize("k,p", [(31, 10), (31, 0), (31, 13), (5, 3), (5, 5), (32, 12), (12, 6), (3, 2)])
@pytest.mark.parametrize("layout", [sg.SBWT_LAYOUT_LINES, sg.SBWT_LAYOUT_POPPY, sg.SBWT_LAYOUT_LINES512,
                                    sg.SBWT_LAYOUT_LINES2048])
def test_run_walk_modes_equal_per_kmer_search(cuda, k, p, layout):
    """The right-to-left run walk (absent-run skip, and skip + backward steps) answers
    exactly as the per-k-mer search and the oracle, bitmap included."""
    _check_run_walk(cuda, k, p, layout)


@pytest.mark.parametrize("k,p", [(31, 10), (5, 3), (32, 12)])
@pytest.mark.parametrize("layout", [sg.SBWT_LAYOUT_LINES, sg.SBWT_LAYOUT_POPPY, sg.SBWT_LAYOUT_LINES512])
def test_run_walk_64bit_index_form(cuda, monkeypatch, k, p, layout):
    """Batches below 4G letters walk with 32-bit k-mer and letter indices; larger ones with
    64-bit indices.  SBWT_RUN_INDEX64=1 puts a small batch on the 64-bit form."""
    monkeypatch.setenv("SBWT_RUN_INDEX64", "1")
    _check_run_walk(cuda, k, p, layout)


def _check_run_walk(cuda, k, p, layout):
    rng = wl.rng_for(2000 + k * 17 + p)
    genome = wl.random_bases(rng, 60_000)
    built = sg.build_sbwt([genome.tobytes()], k)
    letters, rows = _row_mixture(rng, genome, k)
    ox = orc.OracleIndex(built.bits, built.n_bits)
    want = ox.search_reads(letters, rows, k, p)
    if k >= 12:
        assert 0.05 < (want != orc.NOT_FOUND).mean() < 0.95
    got = {}
    with sg.Index.from_bits(built.bits, built.n_bits, k=k, k_presearch=p) as ix:
        ix.configure(layout, kmers_per_thread=0)
        for mode in (sg.SEARCH_STREAM, sg.SEARCH_SKIP_ABSENT, sg.SEARCH_EVERY_KMER):
            ix.set_search_mode(mode)
            got[mode] = run_reads(ix, letters, rows, cuda, member=True)
        ix.set_search_mode(sg.SEARCH_STREAM)
        half = run_reads(ix, letters, rows, cuda, n_kmers=want.size // 2 + 7)
    nk = want.size
    bits = np.zeros((nk + 31) // 32 * 32, dtype=bool)
    bits[:nk] = want != orc.NOT_FOUND
    words = (bits.reshape(-1, 32).astype(np.uint64) << np.arange(32, dtype=np.uint64)).sum(axis=1).astype(np.uint32)
    for mode, (ans, mem) in got.items():
        assert np.array_equal(ans, want), mode
        assert np.array_equal(mem[: words.size], words), mode
    assert np.array_equal(half, want[: nk // 2 + 7])


def _node_bytes_cpu(seqs, k):
    """First letter and group-start flag of every node, from the SBWT definition."""
    keys, dk, dl = orc.independent_sbwt(seqs, k)
    key = np.concatenate([dk, keys])
    ln = np.concatenate([dl, np.full(keys.size, k, dtype=np.int64)])
    order = np.lexsort((ln, key))
    key, ln = key[order], ln[order]
    first = np.where(ln >= k, (key & np.uint64(3)).astype(np.int64) + 1, 0)
    suf = key >> np.uint64(2)  # letters 1..k-1
    sl = np.minimum(ln, k - 1)
    start = np.ones(key.size, dtype=bool)
    start[1:] = (suf[1:] != suf[:-1]) | (sl[1:] != sl[:-1])
    return (first | (start.astype(np.int64) << 3)).astype(np.uint8)


@pytest.mark.parametrize("k", [3, 7, 31, 32])
def test_node_bytes_match_the_sbwt_definition(cuda, k):
    rng = wl.rng_for(3100 + k)
    seqs = [wl.random_bases(rng, 20_000).tobytes(), wl.random_bases(rng, 3_000).tobytes()]
    built = sg.build_sbwt(seqs, k)
    want = _node_bytes_cpu(seqs, k)
    assert want.size == built.n_bits
    with sg.Index.from_bits(built.bits, built.n_bits, k=k, k_presearch=min(k, 8)) as ix:
        got = ix.node_bytes()
    assert np.array_equal(got, want)


def test_search_mode_default_param(cuda):
    p = sg.default_params()
    assert p.search_mode == sg.SEARCH_STREAM


def _bits_of(ans):
    nk = ans.size
    b = np.zeros((nk + 31) // 32 * 32, dtype=bool)
    b[:nk] = ans != orc.NOT_FOUND
    return (b.reshape(-1, 32).astype(np.uint64) << np.arange(32, dtype=np.uint64)).sum(axis=1).astype(np.uint32)


@pytest.mark.parametrize("mode", [0, 1, 2])
def test_membership_only_device_and_host(small, cuda, mode):
    """Answers NULL + bitmap (device entry point) and the host membership pipeline, every mode,
    with chunks whose first k-mer is not a multiple of 32."""
    import torch
    b, k = small["built"], small["k"]
    rng = np.random.default_rng(5)
    lens = rng.integers(20, 400, size=3000)
    g = small["genome"]
    parts = [g[s:s + n] if i % 3 else wl.random_bases(rng, int(n)) for i, (s, n) in
             enumerate(zip(rng.integers(0, g.size - 400, size=lens.size), lens))]
    letters = np.concatenate(parts)
    rows = np.zeros(len(parts) + 1, dtype=np.uint64)
    rows[1:] = np.cumsum([p.size for p in parts])
    ox = orc.OracleIndex(b.bits, b.n_bits)
    want = _bits_of(ox.search_reads(letters, rows, k, 10))
    with sg.Index.from_bits(b.bits, b.n_bits, k=k, k_presearch=10, search_mode=mode) as ix:
        nk = sg.count_kmers(rows, k)
        d_mem = torch.full(((nk + 31) // 32,), -1, dtype=torch.int32, device=cuda)
        ix.search_reads(_t(letters, cuda), _t(rows, cuda), None, nk, d_member_bits=d_mem)
        torch.cuda.synchronize()
        got_dev = d_mem.cpu().numpy().view(np.uint32)
        got_host = ix.member_reads_host(letters, rows)
    assert np.array_equal(got_dev, want)
    assert np.array_equal(got_host[: want.size], want)


def test_host_pipelines_across_chunks(small, cuda):
    """More than one 64M-letter chunk: the answers pipeline and the membership pipeline (whose
    second chunk starts at a k-mer index that is not a multiple of 32) against one device search."""
    import torch
    b, k = small["built"], small["k"]
    rng = wl.rng_for(77)
    g = small["genome"]
    n_reads = 470_000
    reads = np.concatenate([wl.sampled_reads(rng, g, n_reads // 10, 150, 0.01),
                            wl.uniform_reads(rng, n_reads - n_reads // 10, 150)])
    letters = np.ascontiguousarray(reads).reshape(-1)
    rows = np.arange(n_reads + 1, dtype=np.uint64) * np.uint64(150)
    with sg.Index.from_bits(b.bits, b.n_bits, k=k, k_presearch=10) as ix:
        want = run_reads(ix, letters, rows, cuda)
        host = ix.search_reads_host(letters, rows)
        mem = ix.member_reads_host(letters, rows)
    assert letters.size > (64 << 20)
    assert np.array_equal(host, want)
    assert np.array_equal(mem, _bits_of(want))


@pytest.mark.parametrize("transfer", ["sparse", "dense", "hybrid", "threads2"])
@pytest.mark.parametrize("chunk", [4096, 50_000])
def test_host_answers_sparse_transfer_many_chunks(small, cuda, monkeypatch, chunk, transfer):
    """The host answers pipeline brings a chunk's answers back as its membership bitmap, group
    offsets and found node ids and expands them on the host (or, dense, as u64 answers).  Many
    chunks (every stage of the six-slot rotation and of the expander thread), chunks where every k-mer is found (genome
    reads only), reads without a found k-mer, ragged, empty and shorter-than-k rows, against the
    oracle."""
    import torch
    b, k = small["built"], small["k"]
    rng = wl.rng_for(91)
    g = small["genome"]
    parts = []
    for i in range(400):
        length = int(rng.integers(0, 400))
        if i % 4 == 0:  # genome substring: every k-mer found
            s0 = int(rng.integers(0, g.size - 400))
            parts.append(g[s0:s0 + length])
        elif i % 4 == 1:
            parts.append(wl.uniform_reads(rng, 1, length).reshape(-1))
        elif i % 4 == 2:
            parts.append(np.zeros(0, np.uint8))
        else:  # at most one k-mer
            s0 = int(rng.integers(0, g.size - 400))
            parts.append(g[s0:s0 + int(rng.integers(0, k + 1))])
    parts += [g[i * 3000:(i + 1) * 3000] for i in range(20)]  # whole chunks of found k-mers
    letters = np.ascontiguousarray(np.concatenate(parts).astype(np.uint8))
    rows = np.zeros(len(parts) + 1, dtype=np.uint64)
    rows[1:] = np.cumsum([p.size for p in parts])
    want = orc.OracleIndex(b.bits, b.n_bits).search_reads(letters, rows, k, 10)
    monkeypatch.setenv("SBWT_PIPELINE_CHUNK_LETTERS", str(chunk))
    if transfer == "threads2":  # two host threads: the split by sbwt_pipeline_dense_share (70 % of chunks dense)
        monkeypatch.delenv("SBWT_PIPELINE_TRANSFER", raising=False)
    else:
        monkeypatch.setenv("SBWT_PIPELINE_TRANSFER", transfer)
    with sg.Index.from_bits(b.bits, b.n_bits, k=k, k_presearch=10) as ix:
        if transfer == "threads2":
            ix.set_host_threads(2)
        host = ix.search_reads_host(letters, rows)
        moved = ix.pipeline_bytes()
        pa = torch.empty(want.size, dtype=torch.int64).pin_memory()  # hybrid copies into pinned buffers
        ix.search_reads_host(letters, rows, pa)
        moved_pinned = ix.pipeline_bytes()
        mem = ix.member_reads_host(letters, rows)
        junk = np.full(mem.size, 0xA5A5A5A5, dtype=np.uint32)  # every output word is written, none or-ed into stale bits
        ix.member_reads_host(letters, rows, junk)
    assert np.array_equal(junk, mem)
    assert letters.size > 2 * chunk
    assert moved["h2d"] > letters.size and 0 < moved["d2h"]
    assert (moved["d2h"] >= 8 * want.size) == (transfer == "dense")
    if transfer == "threads2":  # the pinned call sent most answers dense, some sparse
        assert 0.25 * 8 * want.size < moved_pinned["d2h"] < 8 * want.size
    assert np.array_equal(pa.numpy().view(np.uint64), want)
    assert (want != orc.NOT_FOUND).mean() > 0.3 and (want == orc.NOT_FOUND).any()
    assert np.array_equal(host, want)
    assert np.array_equal(mem, _bits_of(want))


@pytest.mark.parametrize("compact", ["1", "0"])
@pytest.mark.parametrize("p", [2, 6, 10, 13])
def test_run_walk_compact_presearch_entries(small, cuda, monkeypatch, p, compact):
    """The run walk reads 4-byte presearch entries (left end + width) and the 8-byte entry only
    for intervals too wide for the width field: p = 2 (every interval wide), 6 (both kinds),
    10 and 13 (narrow and empty ones), with and without the compact table."""
    monkeypatch.setenv("SBWT_PRESEARCH_COMPACT", compact)
    b, k = small["built"], small["k"]
    want = orc.OracleIndex(b.bits, b.n_bits).search_reads(small["letters"], small["rows"], k, p)
    with sg.Index.from_bits(b.bits, b.n_bits, k=k, k_presearch=p) as ix:
        for mode in (sg.SEARCH_SKIP_ABSENT, sg.SEARCH_STREAM):
            ix.set_search_mode(mode)
            assert np.array_equal(run_reads(ix, small["letters"], small["rows"], cuda), want), mode
    lefts, rights = orc.OracleIndex(b.bits, b.n_bits).presearch(p)
    width = np.where(lefts <= rights, rights.astype(np.int64) - lefts.astype(np.int64) + 1, 0)
    if p == 2:
        assert (width >= 31).all()
    if p == 6:
        assert (width >= 31).any() and ((width > 0) & (width < 31)).any()


def test_build_times_reported(small, cuda):
    b = small["built"]
    with sg.Index.from_bits(b.bits, b.n_bits, k=31, k_presearch=10) as ix:
        t = ix.build_times()
        assert t["lines_ms"] > 0 and t["presearch_ms"] > 0 and t["backward_ms"] > 0 and t["poppy_ms"] == 0
        ix.presearch(12)
        assert ix.build_times()["presearch_ms"] > 0


def test_search_packed_back_to_back_calls_without_a_wait(small, cuda):
    """The kernel contract chooses between the run walk and the per-k-mer search on the device: calls
    on runs, shuffled positions and runs again, issued back to back with no synchronisation between
    them, each answer as the oracle does."""
    import torch
    b, k = small["built"], small["k"]
    ox = orc.OracleIndex(b.bits, b.n_bits)
    words = orc.pack(small["letters"])
    runs = orc.positions(small["rows"], k).copy()
    shuffled = runs[np.random.default_rng(5).permutation(runs.size)]
    want_runs, want_shuf = ox.search_positions(words, runs, k, 10), ox.search_positions(words, shuffled, k, 10)
    with sg.Index.from_bits(b.bits, b.n_bits, k=k, k_presearch=10) as ix:
        d_words = _t(words, cuda)
        d = [_t(x, cuda) for x in (runs, shuffled, runs, shuffled[: shuffled.size // 2])]
        torch.cuda.synchronize()
        for x in d:
            ix.search_packed(d_words, x)
        torch.cuda.synchronize()
    assert np.array_equal(_u64(d[0]), want_runs) and np.array_equal(_u64(d[2]), want_runs)
    assert np.array_equal(_u64(d[1]), want_shuf)
    assert np.array_equal(_u64(d[3]), want_shuf[: shuffled.size // 2])


@pytest.mark.parametrize("mode", [0, 1, 2])
@pytest.mark.parametrize("order", ["reads", "shuffled", "mixed"])
def test_search_packed_runs_and_random_positions(small, cuda, mode, order):
    """The kernel contract with the reference's positions (runs of consecutive positions,
    walked as runs), shuffled positions (searched per k-mer) and a mix of both, in every mode."""
    import torch
    b, k = small["built"], small["k"]
    ox = orc.OracleIndex(b.bits, b.n_bits)
    words = orc.pack(small["letters"])
    pos = orc.positions(small["rows"], k).copy()
    rng = np.random.default_rng(17)
    if order == "shuffled":
        pos = pos[rng.permutation(pos.size)]
    elif order == "mixed":  # a shuffled tail after runs, and runs that touch at read ends
        cut = pos.size * 3 // 4
        pos[cut:] = pos[cut:][rng.permutation(pos.size - cut)]
    want = ox.search_positions(words, pos, k, 10)
    with sg.Index.from_bits(b.bits, b.n_bits, k=k, k_presearch=10, search_mode=mode) as ix:
        d_pos = _t(pos, cuda)
        ix.search_packed(_t(words, cuda), d_pos)
        torch.cuda.synchronize()
        assert np.array_equal(_u64(d_pos), want)
