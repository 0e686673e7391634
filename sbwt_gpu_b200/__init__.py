"""sbwt_gpu_b200 -- B200 (sm_100a) k-mer membership engine over the Spectral
Burrows-Wheeler Transform, a drop-in for the search path of epicharri/sbwt_gpu.

The engine is C++/CUDA behind the C ABI of ``include/sbwt_gpu.h``
(``libsbwt_gpu.so``, plus the ``sbwt_search`` command-line tool).  This module
is a thin ctypes layer over that ABI for tests, benchmarks and Python callers;
it does no compute of its own.  Names follow the reference:

* ``Index.load``         <- epic::MatrixSBWT::create (include/matrix_sbwt.hpp:32-200)
* ``Index.presearch``    <- epic::PreSearch::call_presearch (include/presearch.hpp:32-130)
* ``Index.search_packed``<- epic::gpu::launch_search_kernel (include/gpu/search_and_presearch_launchers.hpp:21-60)
* ``read_queries``       <- epic::KmerSearch::read_file (include/epicseq/kmer_search.hpp:319-342)
* ``format_answers``     <- epic::ResultsPersister::save_results_to_file (include/epicseq/results_persister.hpp:82-95)
"""
import ctypes
import os
from ctypes import POINTER, byref, c_uint32, c_uint64, c_void_p

import numpy as np

from ._lib import (CLI_PATH, LIB_PATH, SBWT_CUM_POPPY, SBWT_LAYOUT_LINES, SBWT_LAYOUT_LINES512, SBWT_LAYOUT_LINES2048,
                   SBWT_LAYOUT_POPPY, SBWT_POPPY, Built,
                   MlpParams, Params, PrefilterStats, Profile, Queries, SbwtError, check, lib)

__all__ = [
    "Index", "Params", "SbwtError", "build_sbwt", "write_index_files", "read_queries", "format_answers",
    "count_kmers", "read_queries_many", "read_query_batches", "format_answers_device", "default_params", "SBWT_POPPY", "SBWT_CUM_POPPY", "SBWT_LAYOUT_LINES", "SBWT_LAYOUT_POPPY", "SBWT_LAYOUT_LINES512", "SBWT_LAYOUT_LINES2048",
    "pipeline_dense_share", "partition_rows", "search_reads_host_multi", "LIB_PATH", "CLI_PATH", "NOT_FOUND", "SEARCH_EVERY_KMER", "SEARCH_SKIP_ABSENT", "SEARCH_STREAM", "Prefilter", "mlp_params", "mlp_gradients", "mlp_logits", "MLP_PARAMS",
]

MLP_PARAMS = 256 * 128 + 256 + 256 * 256 + 256 + 256 + 1  # W1, b1, W2, b2, w3, b3

NOT_FOUND = 0xFFFFFFFFFFFFFFFF  # answer of an absent k-mer (printed as -1)
SBWT_KEEP = 0xFFFFFFFF  # sbwt_configure: leave the argument unchanged
SEARCH_EVERY_KMER, SEARCH_SKIP_ABSENT, SEARCH_STREAM = 0, 1, 2  # sbwt_params.search_mode


def default_params(**kw):
    """``sbwt_params`` with the reference's defaults (parameters.hpp:41-56), overridden by ``kw``."""
    p = Params()
    check(lib.sbwt_params_default(byref(p)))
    for key, val in kw.items():
        if not hasattr(p, key):
            raise TypeError(f"unknown parameter {key}")
        setattr(p, key, val)
    return p


def _ptr(a):
    """Data pointer of a numpy array or a torch tensor (host or device)."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return c_void_p(a.ctypes.data)
    return c_void_p(a.data_ptr())


def _stream_ptr(stream):
    if stream is None:
        return None
    return c_void_p(stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream))


class Index:
    """An SBWT index resident on one GPU (``sbwt_index*``)."""

    def __init__(self, handle):
        self._h = handle

    # -------------------------------------------------------------- creation
    @classmethod
    def load(cls, file_a, file_c, file_g, file_t, params=None, **kw):
        p = params if params is not None else default_params(**kw)
        h = c_void_p()
        check(lib.sbwt_index_load(os.fsencode(file_a), os.fsencode(file_c), os.fsencode(file_g),
                                  os.fsencode(file_t), byref(p), byref(h)))
        return cls(h)

    @classmethod
    def from_bits(cls, bits, n_bits, params=None, **kw):
        """bits: four uint64 arrays (reference in-memory layout: position p at bit 63-p%64 of word p/64)."""
        p = params if params is not None else default_params(**kw)
        arrs = [np.ascontiguousarray(b, dtype=np.uint64) for b in bits]
        need = (int(n_bits) + 63) // 64
        for a in arrs:
            if a.size < need:
                raise ValueError(f"a bit vector holds {a.size} words, {need} needed")
        ptrs = (c_void_p * 4)(*[a.ctypes.data for a in arrs])
        h = c_void_p()
        check(lib.sbwt_index_from_host(ptrs, int(n_bits), byref(p), byref(h)))
        return cls(h)

    def close(self):
        if self._h:
            lib.sbwt_index_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ------------------------------------------------------------ inspection
    def info(self):
        n = c_uint64()
        C = (c_uint64 * 5)()
        k = c_uint32()
        p = c_uint32()
        check(lib.sbwt_index_info(self._h, byref(n), C, byref(k), byref(p)))
        return {"n_bits": n.value, "C": [int(x) for x in C], "k": k.value, "k_presearch": p.value}

    def presearch(self, p):
        check(lib.sbwt_presearch(self._h, int(p)))

    def presearch_table(self):
        p = self.info()["k_presearch"]
        if p == 0:
            raise SbwtError("the index has no presearch table")
        count = 1 << (2 * p)
        lefts = np.empty(count, dtype=np.uint64)
        rights = np.empty(count, dtype=np.uint64)
        check(lib.sbwt_presearch_export(self._h, _ptr(lefts), _ptr(rights), count))
        return lefts, rights

    def rank_structures(self, bits_in_superblock, rank_structure, c):
        n = self.info()["n_bits"]
        log_h = 31 if bits_in_superblock == 4096 else 32
        l0w = 1 + (n >> log_h)
        l12w = 1 + ((n + bits_in_superblock - 1) // bits_in_superblock)
        L0 = np.empty(l0w, dtype=np.uint64)
        L12 = np.empty(l12w, dtype=np.uint64)
        check(lib.sbwt_rank_export(self._h, bits_in_superblock, rank_structure, c, _ptr(L0), l0w, _ptr(L12), l12w))
        return L0, L12

    def configure(self, layout=SBWT_LAYOUT_LINES, bits_in_superblock=1024, rank_structure=SBWT_POPPY,
                  with_shuffles=0, kmers_per_thread=SBWT_KEEP, threads_per_kmer=SBWT_KEEP,
                  threads_per_block=SBWT_KEEP):
        check(lib.sbwt_configure(self._h, layout, bits_in_superblock, rank_structure, int(with_shuffles),
                                 kmers_per_thread, threads_per_kmer, threads_per_block))

    def build_times(self):
        """Device ms of the last build phases: lines, poppy, presearch table, backward-step structures."""
        ms = (ctypes.c_float * 4)()
        check(lib.sbwt_build_times(self._h, ms))
        return {"lines_ms": ms[0], "poppy_ms": ms[1], "presearch_ms": ms[2], "backward_ms": ms[3]}

    def set_walk_options(self, window=None, blocks_per_sm=None, evict=None, l2_persist=None):
        """Knobs of the run walk (None: unchanged): window 64/128/256, resident blocks per SM (0: as many
        as fit), evict 0 (by table size) / 1 (never) / 2 (always), l2_persist 0/1."""
        keep = 0xFFFFFFFF
        check(lib.sbwt_set_walk_options(self._h, keep if window is None else int(window),
                                        keep if blocks_per_sm is None else int(blocks_per_sm),
                                        -1 if evict is None else int(evict),
                                        -1 if l2_persist is None else int(l2_persist)))

    def set_host_threads(self, threads):
        """Host threads of the host pipelines (0: the OpenMP default)."""
        check(lib.sbwt_set_host_threads(self._h, int(threads)))

    def pipeline_bytes(self):
        """Bytes the last host-buffer search (search_reads_host, member_reads_host) copied
        host->device and device->host."""
        h2d, d2h = ctypes.c_uint64(0), ctypes.c_uint64(0)
        check(lib.sbwt_pipeline_bytes(self._h, ctypes.byref(h2d), ctypes.byref(d2h)))
        return {"h2d": h2d.value, "d2h": d2h.value}

    def set_search_mode(self, mode):
        """SEARCH_EVERY_KMER, SEARCH_SKIP_ABSENT or SEARCH_STREAM (default) for searches of reads;
        the answers are the same in every mode."""
        check(lib.sbwt_set_search_mode(self._h, int(mode)))

    def node_bytes(self):
        """Per-column node bytes of the backward step: first letter (0 = $, 1..4 = ACGT) | 8 on group starts."""
        n = self.info()["n_bits"]
        out = np.empty(n, dtype=np.uint8)
        check(lib.sbwt_node_bytes_export(self._h, _ptr(out), n))
        return out

    def autotune(self, d_letters, d_row_starts, d_answers, n_kmers, tune_p=False, tune_poppy=False,
                 tune_shapes=False):
        """Times candidate layouts and run-walk knobs (and p, poppy layouts, per-k-mer kernel shapes on
        request) on a device sample, keeps the fastest; returns the JSON report."""
        n_rows = int(d_row_starts.numel()) - 1
        flags = (2 if tune_p else 0) | (4 if tune_poppy else 0) | (8 if tune_shapes else 0)
        buf = ctypes.create_string_buffer(1 << 16)
        check(lib.sbwt_autotune(self._h, _ptr(d_letters), int(d_letters.numel()), _ptr(d_row_starts), n_rows,
                                int(n_kmers), _ptr(d_answers), flags, buf, len(buf)))
        import json
        return json.loads(buf.value.decode())

    def set_l2_fetch_granularity(self, nbytes):
        """cudaLimitMaxL2FetchGranularity for this process (the reference's --device-set-limit-search)."""
        check(lib.sbwt_set_l2_fetch_granularity(self._h, int(nbytes)))

    def use_graphs(self, on=True):
        """CUDA-graph replay of repeated sbwt_search_reads calls (same buffers and sizes)."""
        check(lib.sbwt_use_graphs(self._h, int(on)))

    def profile(self, on=True):
        """Enables CUDA-event timing of each sbwt_search_reads phase."""
        check(lib.sbwt_profile_enable(self._h, int(on)))

    def last_profile(self):
        pr = Profile()
        check(lib.sbwt_profile_read(self._h, byref(pr)))
        return {"pack_ms": pr.pack_ms, "table_ms": pr.table_ms, "search_ms": pr.search_ms,
                "member_ms": pr.member_ms, "launches": pr.launches, "search_blocks": pr.search_blocks}

    # ---------------------------------------------------------------- search
    def search_packed(self, d_words, d_positions, n_kmers=None, stream=None):
        """Reference kernel contract: positions in, answers out, in place (device tensors, 64-bit)."""
        n = int(d_positions.numel()) if n_kmers is None else int(n_kmers)
        check(lib.sbwt_search_packed(self._h, _ptr(d_words), int(d_words.numel()), _ptr(d_positions), n,
                                     _stream_ptr(stream)))

    def search_reads(self, d_letters, d_row_starts, d_answers, n_kmers, d_member_bits=None, stream=None):
        """Device-resident reads (uint8 letters, int64 row starts) -> device answers."""
        n_rows = int(d_row_starts.numel()) - 1
        check(lib.sbwt_search_reads(self._h, _ptr(d_letters), int(d_letters.numel()), _ptr(d_row_starts), n_rows,
                                    _ptr(d_answers), _ptr(d_member_bits), int(n_kmers), _stream_ptr(stream)))

    def search_kmers(self, d_kmers, d_answers, n=None, stream=None):
        """Exact answers of k-mers given as MSB-first 64-bit words (device tensors)."""
        n = int(d_kmers.numel()) if n is None else int(n)
        check(lib.sbwt_search_kmers(self._h, _ptr(d_kmers), n, _ptr(d_answers), _stream_ptr(stream)))

    def search_kmers_filtered(self, prefilter, d_kmers, d_answers, n=None, stream=None):
        """The same behind the learned prefilter; returns the number of k-mers answered without a search."""
        n = int(d_kmers.numel()) if n is None else int(n)
        sk = c_uint64()
        check(lib.sbwt_search_kmers_filtered(self._h, prefilter._h, _ptr(d_kmers), n, _ptr(d_answers), byref(sk),
                                             _stream_ptr(stream)))
        return sk.value

    def search_reads_filtered(self, prefilter, d_letters, d_row_starts, d_answers, n_kmers, d_member_bits=None,
                              stream=None, count_skipped=True):
        """search_reads behind the learned prefilter; returns the number of k-mers answered without a search
        (None with count_skipped=False, which keeps the call asynchronous)."""
        n_rows = int(d_row_starts.numel()) - 1
        sk = c_uint64()
        check(lib.sbwt_search_reads_filtered(self._h, prefilter._h, _ptr(d_letters), int(d_letters.numel()),
                                             _ptr(d_row_starts), n_rows, _ptr(d_answers), _ptr(d_member_bits),
                                             int(n_kmers), byref(sk) if count_skipped else None, _stream_ptr(stream)))
        return sk.value if count_skipped else None

    def search_reads_host(self, letters, row_starts, answers=None):
        """Host reads -> host answers (numpy), streamed through the GPU."""
        letters = np.ascontiguousarray(letters, dtype=np.uint8) if isinstance(letters, np.ndarray) else letters
        rs = row_starts
        n_rows = (rs.size if isinstance(rs, np.ndarray) else rs.numel()) - 1
        if isinstance(rs, np.ndarray):
            rs = np.ascontiguousarray(rs, dtype=np.uint64)
            nk = int(lib.sbwt_count_kmers(_ptr(rs), n_rows, self.info()["k"]))
        else:
            nk = count_kmers(rs.numpy().view(np.uint64), self.info()["k"])
        if answers is None:
            answers = np.empty(max(nk, 1), dtype=np.uint64)
        n_letters = letters.size if isinstance(letters, np.ndarray) else letters.numel()
        check(lib.sbwt_search_reads_host(self._h, _ptr(letters), int(n_letters), _ptr(rs), n_rows, _ptr(answers), nk))
        return answers[:nk] if isinstance(answers, np.ndarray) else answers

    def member_reads_host(self, letters, row_starts, member_bits=None):
        """Host reads -> host membership bitmap (uint32 words, bit j%32 of word j/32), streamed
        through the GPU; only the bitmap crosses the bus."""
        letters = np.ascontiguousarray(letters, dtype=np.uint8) if isinstance(letters, np.ndarray) else letters
        rs = row_starts
        n_rows = (rs.size if isinstance(rs, np.ndarray) else rs.numel()) - 1
        if isinstance(rs, np.ndarray):
            rs = np.ascontiguousarray(rs, dtype=np.uint64)
            nk = int(lib.sbwt_count_kmers(_ptr(rs), n_rows, self.info()["k"]))
        else:
            nk = count_kmers(rs.numpy().view(np.uint64), self.info()["k"])
        if member_bits is None:
            member_bits = np.empty(max((nk + 31) // 32, 1), dtype=np.uint32)
        n_letters = letters.size if isinstance(letters, np.ndarray) else letters.numel()
        check(lib.sbwt_search_reads_host_member(self._h, _ptr(letters), int(n_letters), _ptr(rs), n_rows,
                                                _ptr(member_bits), nk))
        return member_bits


# ------------------------------------------------------- learned prefilter

def mlp_params(**kw):
    """``sbwt_mlp_params`` with the defaults of the prefilter configuration, overridden by ``kw``."""
    p = MlpParams()
    check(lib.sbwt_mlp_params_default(byref(p)))
    for key, val in kw.items():
        if not hasattr(p, key):
            raise TypeError(f"unknown parameter {key}")
        setattr(p, key, val)
    return p


class Prefilter:
    """A trained MLP + backup Bloom filter (``sbwt_prefilter*``)."""

    def __init__(self, handle):
        self._h = handle

    @classmethod
    def train(cls, index, params=None, **kw):
        p = params if params is not None else mlp_params(**kw)
        h = c_void_p()
        check(lib.sbwt_prefilter_train(index._h, byref(p), byref(h)))
        return cls(h)

    def stats(self):
        st = PrefilterStats()
        check(lib.sbwt_prefilter_stats_get(self._h, byref(st)))
        return {name: getattr(st, name) for name, _ in PrefilterStats._fields_}

    def params(self):
        th = np.empty(MLP_PARAMS, dtype=np.float32)
        check(lib.sbwt_prefilter_params(self._h, _ptr(th), MLP_PARAMS))
        return th

    def logits(self, d_kmers, d_logits, n=None, stream=None):
        n = int(d_kmers.numel()) if n is None else int(n)
        check(lib.sbwt_prefilter_logits(self._h, _ptr(d_kmers), n, _ptr(d_logits), _stream_ptr(stream)))

    def close(self):
        if self._h:
            lib.sbwt_prefilter_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def mlp_gradients(k, theta, kmers, labels):
    """Loss and gradient of one BCE step of the GPU training kernels (test hook)."""
    th = np.ascontiguousarray(theta, dtype=np.float32)
    km = np.ascontiguousarray(kmers, dtype=np.uint64)
    lb = np.ascontiguousarray(labels, dtype=np.uint8)
    grad = np.empty(MLP_PARAMS, dtype=np.float32)
    loss = ctypes.c_float()
    check(lib.sbwt_mlp_gradients(int(k), _ptr(th), _ptr(km), _ptr(lb), km.size, byref(loss), _ptr(grad)))
    return loss.value, grad


def mlp_logits(k, theta, kmers):
    """Logits of the fused tensor-core inference kernel (test hook)."""
    th = np.ascontiguousarray(theta, dtype=np.float32)
    km = np.ascontiguousarray(kmers, dtype=np.uint64)
    out = np.empty(max(km.size, 1), dtype=np.float32)
    check(lib.sbwt_mlp_logits(int(k), _ptr(th), _ptr(km), km.size, _ptr(out)))
    return out[: km.size]


# ------------------------------------------------------------------ builder

class BuiltIndex:
    """Bit vectors of an SBWT built on the host (reference in-memory word layout)."""

    def __init__(self, bits, n_bits, n_kmers, n_dummies):
        self.bits = bits
        self.n_bits = n_bits
        self.n_kmers = n_kmers
        self.n_dummies = n_dummies


def _as_letters_and_starts(seqs):
    if isinstance(seqs, tuple):
        letters, starts = seqs
        return np.ascontiguousarray(letters, dtype=np.uint8), np.ascontiguousarray(starts, dtype=np.uint64)
    parts = [np.frombuffer(s.encode() if isinstance(s, str) else bytes(s), dtype=np.uint8) for s in seqs]
    starts = np.zeros(len(parts) + 1, dtype=np.uint64)
    starts[1:] = np.cumsum([p.size for p in parts])
    letters = np.concatenate(parts) if parts else np.zeros(0, dtype=np.uint8)
    return letters, starts


def build_sbwt(seqs, k, device=None):
    """Builds the plain-matrix SBWT of all k-mers of ``seqs`` (list of str/bytes, or (letters, starts)):
    on the host, or on GPU ``device`` when given (same bits)."""
    letters, starts = _as_letters_and_starts(seqs)
    b = Built()
    if device is None:
        check(lib.sbwt_build(_ptr(letters), _ptr(starts), starts.size - 1, int(k), byref(b)))
    else:
        check(lib.sbwt_build_gpu(_ptr(letters), _ptr(starts), starts.size - 1, int(k), int(device), byref(b)))
    try:
        bits = [np.ctypeslib.as_array(b.bits[c], shape=(b.n_words,)).copy() for c in range(4)]
    finally:
        lib.sbwt_build_free(byref(b))
    return BuiltIndex(bits, int(b.n_bits), int(b.n_kmers), int(b.n_dummies))


def write_index_files(prefix, built):
    """Writes ``prefix``.A/.C/.G/.T in the reference's bit-vector file format."""
    paths = []
    for c, ch in enumerate("ACGT"):
        path = f"{prefix}.{ch}"
        check(lib.sbwt_write_bitvector(os.fsencode(path), _ptr(built.bits[c]), built.n_bits))
        paths.append(path)
    return paths


# ------------------------------------------------------------------ queries

def read_queries(path, k):
    """FASTA reads as the reference reads them: (letters uint8, row_starts uint64, n_kmers)."""
    q = Queries()
    check(lib.sbwt_queries_read(os.fsencode(path), int(k), byref(q)))
    try:
        letters = np.ctypeslib.as_array(q.letters, shape=(q.n_letters + 32,))[: q.n_letters].copy() \
            if q.n_letters else np.zeros(0, dtype=np.uint8)
        rows = np.ctypeslib.as_array(q.row_starts, shape=(q.n_rows + 1,)).copy()
        nk = int(q.n_kmers)
    finally:
        lib.sbwt_queries_free(byref(q))
    return letters, rows, nk


def read_query_batches(path, k, max_letters):
    """Streams a FASTA or FASTQ query file in batches of whole reads (sbwt_reader_next): yields
    (letters uint8, row_starts uint64, n_kmers) per batch."""
    h = c_void_p()
    check(lib.sbwt_reader_open(os.fsencode(path), int(k), byref(h)))
    try:
        while True:
            q = Queries()
            check(lib.sbwt_reader_next(h, int(max_letters), byref(q)))
            try:
                if q.n_rows == 0:
                    return
                letters = np.ctypeslib.as_array(q.letters, shape=(q.n_letters + 32,))[: q.n_letters].copy() \
                    if q.n_letters else np.zeros(0, dtype=np.uint8)
                rows = np.ctypeslib.as_array(q.row_starts, shape=(q.n_rows + 1,)).copy()
                nk = int(q.n_kmers)
            finally:
                lib.sbwt_queries_free(byref(q))
            yield letters, rows, nk
    finally:
        lib.sbwt_reader_close(h)


def read_queries_many(paths, k):
    """Several query files as one batch: (letters, row_starts, n_kmers, file_rows)."""
    arr = (ctypes.c_char_p * len(paths))(*[os.fsencode(p) for p in paths])
    file_rows = np.zeros(len(paths) + 1, dtype=np.uint64)
    q = Queries()
    check(lib.sbwt_queries_read_many(arr, len(paths), int(k), byref(q), _ptr(file_rows)))
    try:
        letters = np.ctypeslib.as_array(q.letters, shape=(q.n_letters + 32,))[: q.n_letters].copy() \
            if q.n_letters else np.zeros(0, dtype=np.uint8)
        rows = np.ctypeslib.as_array(q.row_starts, shape=(q.n_rows + 1,)).copy()
        nk = int(q.n_kmers)
    finally:
        lib.sbwt_queries_free(byref(q))
    return letters, rows, nk, file_rows


def pipeline_dense_share(n_columns, host_threads=0):
    """Share of the chunks of a host-pipeline search whose u64 answers cross PCIe as such, for an index of
    n_columns and host_threads threads (0: the OpenMP default); needs no GPU."""
    return float(lib.sbwt_pipeline_dense_share(int(n_columns), int(host_threads)))


def partition_rows(row_starts, k, n_parts):
    """Row bounds (n_parts + 1) of contiguous ranges with near-equal k-mer counts (sbwt_partition_rows)."""
    rs = np.ascontiguousarray(row_starts, dtype=np.uint64)
    bounds = np.zeros(n_parts + 1, dtype=np.uint64)
    check(lib.sbwt_partition_rows(_ptr(rs), rs.size - 1, int(k), int(n_parts), _ptr(bounds)))
    return bounds


def search_reads_host_multi(indexes, letters, row_starts, answers=None):
    """Host reads searched on several index replicas (one per GPU), each on its own contiguous range of
    rows; returns the host answers (sbwt_search_reads_host_multi)."""
    letters = np.ascontiguousarray(letters, dtype=np.uint8)
    rs = np.ascontiguousarray(row_starts, dtype=np.uint64)
    k = indexes[0].info()["k"]
    nk = int(lib.sbwt_count_kmers(_ptr(rs), rs.size - 1, k))
    if answers is None:
        answers = np.empty(max(nk, 1), dtype=np.uint64)
    handles = (c_void_p * len(indexes))(*[ix._h.value if isinstance(ix._h, c_void_p) else ix._h for ix in indexes])
    check(lib.sbwt_search_reads_host_multi(handles, len(indexes), _ptr(letters), letters.size, _ptr(rs), rs.size - 1,
                                           _ptr(answers), nk))
    return answers[:nk] if isinstance(answers, np.ndarray) else answers


def count_kmers(row_starts, k):
    rs = np.ascontiguousarray(row_starts, dtype=np.uint64)
    return int(lib.sbwt_count_kmers(_ptr(rs), rs.size - 1, int(k)))


def format_answers(row_starts, k, answers):
    """The reference's stdout text for the answers of the given rows (bytes)."""
    rs = np.ascontiguousarray(row_starts, dtype=np.uint64)
    ans = np.ascontiguousarray(answers, dtype=np.uint64)
    size = lib.sbwt_format_answers(_ptr(rs), rs.size - 1, int(k), _ptr(ans), None, 0)
    buf = ctypes.create_string_buffer(int(size) + 1)
    got = lib.sbwt_format_answers(_ptr(rs), rs.size - 1, int(k), _ptr(ans), buf, int(size) + 1)
    if got < 0:
        raise SbwtError("format buffer too small")
    return buf.raw[:got]


def format_answers_device(d_row_starts, k, d_answers, stream=None):
    """The same text formatted on the GPU from device tensors (int64 row starts and answers); bytes."""
    import torch
    n_rows = int(d_row_starts.numel()) - 1
    nk = int(d_answers.numel())
    nbytes = c_uint64(0)
    check(lib.sbwt_format_answers_device(_ptr(d_row_starts), n_rows, int(k), _ptr(d_answers), nk, None, 0,
                                         byref(nbytes), _stream_ptr(stream)))
    out = torch.empty(max(int(nbytes.value), 1), dtype=torch.uint8, device=d_answers.device)
    check(lib.sbwt_format_answers_device(_ptr(d_row_starts), n_rows, int(k), _ptr(d_answers), nk, _ptr(out),
                                         int(out.numel()), byref(nbytes), _stream_ptr(stream)))
    return bytes(out[: int(nbytes.value)].cpu().numpy())
