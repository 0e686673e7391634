"""The C ABI without a GPU: the library loads, exports every declared symbol,
and the host-side entry points behave like the reference's host code."""
import os
import re
import shutil
import subprocess

import numpy as np
import pytest

import oracle as orc
import sbwt_gpu_b200 as sg
from sbwt_gpu_b200 import _lib, workloads as wl

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    text = open(os.path.join(ROOT, "include", "sbwt_gpu.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(sbwt_\w+)\s*\(", text)))


def test_every_declared_symbol_is_exported():
    names = declared_functions()
    assert len(names) >= 20
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (sbwt_\w+)", out))
    missing = [n for n in names if n not in exported]
    assert not missing, missing
    for n in names:
        assert n in _lib.SIGNATURES, f"{n} has no ctypes signature"


def test_params_default_is_the_reference_default():
    p = sg.default_params()
    assert (p.k, p.k_presearch, p.bits_in_superblock, p.rank_structure, p.with_shuffles) == (30, 12, 1024, 1, 0)


def test_no_cpu_fallback_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(sg.SbwtError, match="no CUDA device"):
        sg.Index.from_bits([np.zeros(1, np.uint64)] * 4, 1)


def test_parameter_errors():
    with pytest.raises(sg.SbwtError, match="k must be at least 3"):
        sg.Index.from_bits([np.zeros(1, np.uint64)] * 4, 1, k=2)
    with pytest.raises(sg.SbwtError, match="exceeds k"):
        sg.Index.from_bits([np.zeros(1, np.uint64)] * 4, 1, k=5, k_presearch=6)


def test_read_queries_matches_oracle(tmp_path):
    rng = wl.rng_for(3)
    letters, rows = wl.mixed_reads(rng, wl.random_bases(rng, 2000), 5, 5, 77, 0.01)
    fa = tmp_path / "q.fa"
    wl.write_fasta(str(fa), letters, rows)
    raw = fa.read_bytes() + b">empty\n\nACG\nAC\r\nNNNNNNNNNNNNNNNNNNNNNNNNNNNNNNNNNNN\n"
    fa.write_bytes(raw)
    for k in (3, 31):
        l1, r1, nk1 = sg.read_queries(str(fa), k)
        l2, r2, nk2 = orc.read_queries(raw, k)
        assert np.array_equal(l1, l2) and np.array_equal(r1, r2) and nk1 == nk2
        assert sg.count_kmers(r1, k) == nk1


def test_read_queries_keeps_last_letter_without_newline(tmp_path):
    fa = tmp_path / "q.fa"
    fa.write_bytes(b">x\nACGTAC")
    letters, rows, nk = sg.read_queries(str(fa), 5)
    assert letters.tobytes() == b"ACGTAC" and nk == 2   # the reference drops the final C here


def test_format_answers_matches_oracle():
    rows = np.array([0, 40, 45, 100], dtype=np.uint64)
    k = 31
    n = sg.count_kmers(rows, k)
    ans = np.array([orc.NOT_FOUND if i % 3 == 0 else i * 1234567 for i in range(n)], dtype=np.uint64)
    assert sg.format_answers(rows, k, ans) == orc.format_answers(rows, k, ans)
    assert sg.format_answers(rows, k, ans).split(b"\n")[1] == b""  # a read shorter than k: empty line


def test_cli_help_and_bad_flags():
    cli = _lib.CLI_PATH
    r = subprocess.run([cli], capture_output=True, text=True)
    assert r.returncode == 0 and "usage" in r.stderr
    r = subprocess.run([cli, "--rank-structure=flat-poppy", "--file-a=x"], capture_output=True, text=True)
    assert r.returncode != 0
    r = subprocess.run([cli, "--bits-in-superblock=4096", "--rank-structure=cum-poppy", "--file-a=a", "--file-c=c",
                        "--file-g=g", "--file-t=t", "--file-queries=q"], capture_output=True, text=True)
    assert r.returncode != 0 and "4096" in r.stderr


def test_read_queries_many_concatenates(tmp_path):
    rng = wl.rng_for(21)
    paths, parts = [], []
    for f in range(4):
        letters, rows = wl.mixed_reads(rng, wl.random_bases(rng, 3000), 3 + f, 2, 50 + 10 * f, 0.0)
        p = str(tmp_path / f"f{f}.fa")
        wl.write_fasta(p, letters, rows)
        paths.append(p)
        parts.append(sg.read_queries(p, 31))
    letters, rows, nk, file_rows = sg.read_queries_many(paths, 31)
    assert np.array_equal(letters, np.concatenate([p[0] for p in parts]))
    assert nk == sum(p[2] for p in parts)
    assert file_rows.tolist() == np.cumsum([0] + [p[1].size - 1 for p in parts]).tolist()
    off = 0
    for f, p in enumerate(parts):
        r0, r1 = int(file_rows[f]), int(file_rows[f + 1])
        assert np.array_equal(rows[r0:r1 + 1] - rows[r0], p[1])
    with pytest.raises(sg.SbwtError):
        sg.read_queries_many(paths + [str(tmp_path / "missing.fa")], 31)


def _reads(n=40, seed=5):
    rng = wl.rng_for(seed)
    g = wl.random_bases(rng, 5000)
    letters, rows = wl.mixed_reads(rng, g, n // 2, n - n // 2, 60, 0.01)
    lens = np.diff(rows.astype(np.int64))
    lens[::7] = np.minimum(lens[::7], 20)  # some reads shorter than k
    parts = [letters[int(rows[i]):int(rows[i]) + int(lens[i])] for i in range(lens.size)]
    letters = np.concatenate(parts)
    rows = np.zeros(lens.size + 1, dtype=np.uint64)
    rows[1:] = np.cumsum(lens)
    return letters, rows


@pytest.mark.parametrize("crlf", [False, True])
def test_fastq_reads_equal_the_fasta_reads(tmp_path, crlf):
    """A FASTQ file (first byte '@') is read as four-line records whose sequence lines are the reads:
    the same letters and rows as the FASTA file of the same reads (no reference counterpart; the
    reference reads FASTA only)."""
    letters, rows = _reads()
    fq, fa = str(tmp_path / "q.fq"), str(tmp_path / "q.fa")
    wl.write_fastq(fq, letters, rows)
    wl.write_fasta(fa, letters, rows)
    a = sg.read_queries(fq, 31)
    b = sg.read_queries(fa, 31)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]) and a[2] == b[2]
    if crlf:  # CR LF line ends: the CR stays a letter of the read, as in the FASTA reading
        wl.write_fastq(fq, letters, rows, crlf=True)
        lt, rw, _ = sg.read_queries(fq, 31)
        assert rw.size == rows.size and lt.size == letters.size + rows.size - 1
        assert lt[int(rw[1]) - 1] == ord("\r")


@pytest.mark.parametrize("fmt", ["fasta", "fastq"])
@pytest.mark.parametrize("max_letters", [1, 333, 1000, 10_000_000])
def test_streamed_batches_concatenate_to_the_whole_file(tmp_path, fmt, max_letters):
    """sbwt_reader_next hands out batches of whole reads of at most max_letters letters (one longer read
    alone); concatenated, they are exactly the whole-file reading."""
    letters, rows = _reads(200, seed=6)
    path = str(tmp_path / ("q.fq" if fmt == "fastq" else "q.fa"))
    (wl.write_fastq if fmt == "fastq" else wl.write_fasta)(path, letters, rows)
    whole = sg.read_queries(path, 31)
    got_l, got_lens, nk = [], [], 0
    for lt, rw, k in sg.read_query_batches(path, 31, max_letters):
        assert rw.size >= 2 and (lt.size <= max_letters or rw.size == 2)
        got_l.append(lt)
        got_lens.append(np.diff(rw.astype(np.int64)))
        nk += k
    assert np.array_equal(np.concatenate(got_l), whole[0])
    assert np.array_equal(np.concatenate(got_lens), np.diff(whole[1].astype(np.int64)))
    assert nk == whole[2]


def test_malformed_and_truncated_fastq(tmp_path):
    bad = tmp_path / "bad.fq"
    bad.write_bytes(b"@r0\nACGTACGT\nX\nIIIIIIII\n")  # the third line must start with '+'
    with pytest.raises(sg.SbwtError, match="not FASTQ"):
        sg.read_queries(str(bad), 5)
    cut = tmp_path / "cut.fq"
    cut.write_bytes(b"@r0\nACGTACGT\n+\nIIIIIIII\n@r1\nACGT\n")
    with pytest.raises(sg.SbwtError, match="ends inside a FASTQ record"):
        sg.read_queries(str(cut), 5)
    ok = tmp_path / "ok.fq"
    ok.write_bytes(b"@r0\nACGTACGT\n+\nIIIIIIII\n@r1\nACGT\n+\nIIII")  # no final newline
    lt, rw, nk = sg.read_queries(str(ok), 5)
    assert lt.tobytes() == b"ACGTACGTACGT" and rw.tolist() == [0, 8, 12] and nk == 4
