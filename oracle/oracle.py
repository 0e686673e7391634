"""CPU oracle of the SBWT search path -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
module, and only as the checker: the product (sbwt_gpu_b200) never imports it.

Two oracles live here:

* ``Oracle*`` / module functions: ctypes over ``liboracle.so``, the C
  restatement of the reference (oracle/sbwt_oracle.c, every function citing
  the reference file:line it follows).  Its rank build is pinned word for word
  against the reference's own RankDataStructures compiled from the reference
  sources (oracle/_ref/ref_rank); its end-to-end answers against fixtures the
  reference program itself produced (tests/golden/).
* ``independent_*``: the SBWT definition restated with numpy (sorted k-mer
  set, dummy nodes, colex order), used to check membership and colex ranks
  without any rank structure.
"""
import ctypes
import os
import subprocess
from ctypes import POINTER, c_char_p, c_int, c_int64, c_uint32, c_uint64, c_void_p

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_RANK = os.path.join(HERE, "_ref", "ref_rank")
REF_SEARCH = os.path.join(HERE, "_ref", "search")
NOT_FOUND = 0xFFFFFFFFFFFFFFFF
POPPY, CUM_POPPY = 1, 2
SB_KINDS = [(256, 1), (512, 1), (1024, 1), (2048, 1), (4096, 1), (256, 2), (512, 2), (1024, 2), (2048, 2)]


def build_oracle():
    subprocess.run(["make", "-s", "-C", HERE, "liboracle.so"], check=True)


def _load():
    if not os.path.exists(LIB_PATH):
        build_oracle()
    lib = ctypes.CDLL(LIB_PATH)
    P = c_void_p
    sig = {
        "orc_file_bits": (c_int64, [c_char_p]),
        "orc_padded_words": (c_uint64, [c_uint64]),
        "orc_read_words": (c_int, [c_char_p, P, c_uint64]),
        "orc_l0_words": (c_uint64, [c_uint64, c_uint32]),
        "orc_l12_words": (c_uint64, [c_uint64, c_uint32]),
        "orc_rank_build": (c_int, [P, c_uint64, c_uint32, c_int, P, P, P]),
        "orc_rank": (c_uint64, [P, P, P, c_uint32, c_int, c_uint64]),
        "orc_c_array": (None, [P, P]),
        "orc_presearch": (None, [P, P, P, P, c_uint32, c_int, c_uint32, P, P]),
        "orc_presearch_at": (None, [P, P, P, P, c_uint32, c_int, c_uint32, P, c_uint64, P, P]),
        "orc_read_queries": (c_int64, [P, c_uint64, c_uint32, P, P, P, P]),
        "orc_pack": (None, [P, c_uint64, P]),
        "orc_positions": (c_uint64, [P, c_uint64, c_uint32, P]),
        "orc_search": (None, [P, P, P, P, c_uint32, c_int, P, P, c_uint32, c_uint32, P, P, c_uint64, P, P]),
        "orc_format_answers": (c_int64, [P, c_uint64, c_uint32, P, P, c_uint64]),
        "orc_num_threads": (c_int, []),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


def _p(a):
    return c_void_p(a.ctypes.data) if a is not None else None


def _ptrs(arrs):
    return (c_void_p * 4)(*[a.ctypes.data for a in arrs])


# --------------------------------------------------------------- a1 .. a3

def file_bits(path):
    return int(lib.orc_file_bits(os.fsencode(path)))


def read_words(path):
    """Byte-swapped words of one bit-vector file (bit_vector.hpp:111-128)."""
    n = file_bits(path)
    if n < 0:
        raise ValueError(f"bad bit-vector file {path}: code {n}")
    nw = int(lib.orc_padded_words(n))
    words = np.zeros(nw, dtype=np.uint64)
    rc = lib.orc_read_words(os.fsencode(path), _p(words), nw)
    if rc != 0:
        raise ValueError(f"bad bit-vector file {path}: code {rc}")
    return words, n


def rank_build(words, n_bits, sb=1024, kind=POPPY):
    l0 = np.zeros(int(lib.orc_l0_words(n_bits, sb)), dtype=np.uint64)
    l12 = np.zeros(int(lib.orc_l12_words(n_bits, sb)), dtype=np.uint64)
    ones = np.zeros(1, dtype=np.uint64)
    if lib.orc_rank_build(_p(words), n_bits, sb, kind, _p(l0), _p(l12), _p(ones)) != 0:
        raise ValueError("unsupported (sb, kind)")
    return l0, l12, int(ones[0])


def c_array(ones):
    o = np.asarray(ones, dtype=np.uint64)
    C = np.zeros(5, dtype=np.uint64)
    lib.orc_c_array(_p(o), _p(C))
    return C


def padded_words(n_bits):
    return int(lib.orc_padded_words(n_bits))


class OracleIndex:
    """The reference's index state: 4 vectors, their L0/L12, the C array."""

    def __init__(self, words, n_bits, sb=1024, kind=POPPY):
        nw = padded_words(n_bits) + 64  # the reference reads up to one basic block past n
        self.words = []
        for w in words:
            a = np.zeros(nw, dtype=np.uint64)
            m = min(w.size, (n_bits + 63) // 64)
            a[:m] = w[:m]
            if n_bits % 64:
                a[(n_bits - 1) // 64] &= np.uint64((0xFFFFFFFFFFFFFFFF << (64 - n_bits % 64)) & 0xFFFFFFFFFFFFFFFF)
            self.words.append(a)
        self.n = int(n_bits)
        self.sb, self.kind = sb, kind
        built = [rank_build(w, self.n, sb, kind) for w in self.words]
        self.L0 = [b[0] for b in built]
        self.L12 = [b[1] for b in built]
        self.ones = [b[2] for b in built]
        self.C = c_array(self.ones)

    @classmethod
    def from_files(cls, paths, sb=1024, kind=POPPY):
        ws, ns = zip(*[read_words(p) for p in paths])
        if len(set(ns)) != 1:
            raise ValueError("bit vectors of different lengths")
        return cls(list(ws), ns[0], sb, kind)

    def rank(self, c, i):
        return int(lib.orc_rank(_p(self.words[c]), _p(self.L0[c]), _p(self.L12[c]), self.sb, self.kind, int(i)))

    def presearch(self, p):
        count = 1 << (2 * p)
        lefts = np.zeros(count, dtype=np.uint64)
        rights = np.zeros(count, dtype=np.uint64)
        lib.orc_presearch(_ptrs(self.words), _ptrs(self.L0), _ptrs(self.L12), _p(self.C), self.sb, self.kind, p,
                          _p(lefts), _p(rights))
        return lefts, rights

    def presearch_at(self, p, idx):
        """Entries of the p-mers idx (uint64 array) of the presearch table."""
        idx = np.ascontiguousarray(idx, dtype=np.uint64)
        lefts = np.zeros(max(idx.size, 1), dtype=np.uint64)
        rights = np.zeros(max(idx.size, 1), dtype=np.uint64)
        lib.orc_presearch_at(_ptrs(self.words), _ptrs(self.L0), _ptrs(self.L12), _p(self.C), self.sb, self.kind, p,
                             _p(idx), idx.size, _p(lefts), _p(rights))
        return lefts[: idx.size], rights[: idx.size]

    def search_positions(self, words, positions, k, p, table=None, want_steps=False):
        """search_kernel.hpp:61-104 over packed words + positions."""
        n = positions.size
        ans = np.zeros(max(n, 1), dtype=np.uint64)
        steps = np.zeros(max(n, 1), dtype=np.uint8) if want_steps else None
        if p:
            lefts, rights = table if table is not None else self.presearch(p)
        else:
            lefts = rights = None
        pos = np.ascontiguousarray(positions, dtype=np.uint64)
        lib.orc_search(_ptrs(self.words), _ptrs(self.L0), _ptrs(self.L12), _p(self.C), self.sb, self.kind,
                       _p(lefts), _p(rights), p, k, _p(words), _p(pos), n, _p(ans), _p(steps))
        return (ans[:n], steps[:n]) if want_steps else ans[:n]

    def search_reads(self, letters, row_starts, k, p, table=None, want_steps=False):
        words = pack(letters)
        pos = positions(row_starts, k)
        return self.search_positions(words, pos, k, p, table, want_steps)


# --------------------------------------------------------------- a7 .. a13

def read_queries(data, k):
    """KmerSearch::read_file on the bytes of a query file (reference quirks included)."""
    buf = np.frombuffer(bytes(data), dtype=np.uint8).copy()
    size = buf.size
    letters = np.zeros(max(size, 1), dtype=np.uint8)
    starts = np.zeros(size + 2, dtype=np.uint64)
    nl = np.zeros(1, dtype=np.uint64)
    nk = np.zeros(1, dtype=np.uint64)
    rows = lib.orc_read_queries(_p(buf), size, k, _p(letters), _p(starts), _p(nl), _p(nk))
    return letters[: int(nl[0])].copy(), starts[: rows + 1].copy(), int(nk[0])


def pack(letters):
    """create_kmer_string over letters padded as add_paddings (kmer_search.hpp:292-301)."""
    n = letters.size
    padded = ((n + 32 + 31) // 32) * 32
    buf = np.zeros(padded, dtype=np.uint8)
    buf[:n] = letters
    words = np.zeros(padded // 32, dtype=np.uint64)
    lib.orc_pack(_p(buf), padded, _p(words))
    return words


def positions(row_starts, k):
    rs = np.ascontiguousarray(row_starts, dtype=np.uint64)
    rows = rs.size - 1
    lens = np.diff(rs.astype(np.int64))
    total = int(np.maximum(lens - k + 1, 0).sum()) if rows else 0
    out = np.zeros(max(total, 1), dtype=np.uint64)
    got = lib.orc_positions(_p(rs), rows, k, _p(out))
    assert got == total
    return out[:total]


def format_answers(row_starts, k, answers):
    rs = np.ascontiguousarray(row_starts, dtype=np.uint64)
    ans = np.ascontiguousarray(answers, dtype=np.uint64)
    cap = 22 * max(ans.size, 1) + rs.size + 16
    out = ctypes.create_string_buffer(cap)
    n = lib.orc_format_answers(_p(rs), rs.size - 1, k, _p(ans), out, cap)
    if n < 0:
        raise RuntimeError("format buffer too small")
    return out.raw[:n]


def num_threads():
    return int(lib.orc_num_threads())


# ------------------------------------------------- reference's own programs

def ref_rank_available():
    return os.path.exists(REF_RANK)


def ref_rank(path, sb, kind, tmpdir):
    """L0, L12, ones and data words computed by the reference's own code."""
    out = os.path.join(str(tmpdir), f"refrank_{sb}_{kind}.bin")
    env = dict(os.environ, MALLOC_PERTURB_="255")
    subprocess.run([REF_RANK, path, str(sb), str(kind), out], check=True, env=env,
                   stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
    raw = np.fromfile(out, dtype=np.uint64)
    n, l0w, l12w, ones, pw = (int(x) for x in raw[:5])
    o = 5
    L0 = raw[o:o + l0w]; o += l0w
    L12 = raw[o:o + l12w]; o += l12w
    data = raw[o:o + pw]
    return {"n": n, "L0": L0, "L12": L12, "ones": ones, "words": data}


# ------------------------------------------------------ independent oracle

CODE = np.full(256, -1, dtype=np.int64)
for _ch, _v in zip(b"ACGTacgt", [0, 1, 2, 3, 0, 1, 2, 3]):
    CODE[_ch] = _v


def kmer_colex_keys(seq_bytes, k):
    """Colex keys (last letter in the top 2 bits) of the ACGT-only k-mers of one sequence."""
    codes = CODE[np.frombuffer(seq_bytes, dtype=np.uint8)]
    n = codes.size
    if n < k:
        return np.zeros(0, dtype=np.uint64)
    valid = codes >= 0
    c = np.where(valid, codes, 0).astype(np.uint64)
    keys = np.zeros(n - k + 1, dtype=np.uint64)
    for i in range(k):  # letter i of the window goes to bits 2i..2i+1
        keys |= c[i:n - k + 1 + i] << np.uint64(2 * i)
    bad = np.convolve(~valid, np.ones(k, dtype=np.int64), mode="valid") > 0
    return keys[~bad]


def independent_sbwt(seqs, k):
    """SBWT node set by the definition: sorted distinct k-mers and sorted dummies.

    Returns (kmer_keys, dummy_keys, dummy_lens) with dummies sorted colex and
    the node order = merge of dummies (len < k) into k-mers by (key, len).
    """
    keys = np.unique(np.concatenate([kmer_colex_keys(s if isinstance(s, bytes) else s.encode(), k)
                                     for s in seqs] or [np.zeros(0, np.uint64)]))
    mask_km1 = np.uint64((1 << (2 * (k - 1))) - 1)
    suffixes = np.unique(keys >> np.uint64(2))
    prefixes = keys & mask_km1
    sources = keys[~np.isin(prefixes, suffixes)]
    dk, dl = [0], [0]
    for x in sources.tolist():
        for i in range(1, k):
            dk.append((x & ((1 << (2 * i)) - 1)) << (2 * (k - i)))
            dl.append(i)
    d = sorted(set(zip(dk, dl)))
    return keys, np.array([a for a, _ in d], dtype=np.uint64), np.array([b for _, b in d], dtype=np.int64)


def query_colex_keys(kmer_words_msb_first, k):
    """Colex keys of k-mers given as MSB-first 2-bit words (first letter in bits 63..62)."""
    w = np.asarray(kmer_words_msb_first, dtype=np.uint64)
    keys = np.zeros_like(w)
    for i in range(k):
        c = (w >> np.uint64(62 - 2 * i)) & np.uint64(3)
        keys |= c << np.uint64(2 * i)
    return keys


def independent_answers(kmer_keys, dummy_keys, query_keys):
    """Colex rank of each query k-mer among all nodes, or NOT_FOUND."""
    pos = np.searchsorted(kmer_keys, query_keys)
    hit = pos < kmer_keys.size
    hit[hit] = kmer_keys[pos[hit]] == query_keys[hit]
    # dummies before a k-mer: dummy key <= k-mer key (equal key: the dummy's shorter length sorts first)
    rank = pos.astype(np.uint64) + np.searchsorted(dummy_keys, query_keys, side="right").astype(np.uint64)
    return np.where(hit, rank, np.uint64(NOT_FOUND))


def extract_kmers(letters, row_starts, k):
    """MSB-first 64-bit windows of every k-mer (search_kernel.hpp:66-68), via the oracle's packer."""
    words = pack(letters)
    pos = positions(row_starts, k)
    b = pos * np.uint64(2)
    wi = (b >> np.uint64(6)).astype(np.int64)
    sh = b & np.uint64(63)
    hi = words[wi] << sh
    lo = np.where(sh == 0, np.uint64(0), words[wi + 1] >> (np.uint64(64) - np.where(sh == 0, np.uint64(1), sh)))
    return hi | lo
