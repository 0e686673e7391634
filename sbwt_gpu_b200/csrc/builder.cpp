// builder.cpp -- host construction of the plain-matrix SBWT in the reference's
// matrix format.
//
// The reference loads four bit vectors written by an external SBWT tool
// (include/matrix_sbwt.hpp:44-55); it ships no construction code.  This file
// builds them from a k-mer spectrum so that the engine is self-contained.
//
// Definitions (Alanko, Puglisi, Vuohtoniemi, "Small searchable k-spectrums via
// subset rank queries on the spectral Burrows-Wheeler transform", 2023):
//   * nodes = the distinct k-mers K plus, for every source k-mer x (no k-mer of
//     K has x[0..k-2] as its (k-1)-suffix), the dummy nodes $^{k-i} x[0..i-1]
//     for i = 0..k-1 ($^k is the root);
//   * nodes are sorted colexicographically ($ < A < C < G < T, comparing from
//     the last character backwards);
//   * column v, row c is 1 iff node v is the colex-first node among those
//     sharing its (k-1)-suffix v[1..k-1] and v[1..k-1]c is a node.
// Each non-root node then has exactly one incoming 1, so vector c holds the
// number of nodes ending in c, and the reference's C array (C[0] = 1,
// matrix_sbwt.hpp:150-157) plus rank gives the search of
// include/gpu/search_kernel.hpp:84-96.
//
// Encoding: a node is (key, len).  key holds the node's reversed string
// 2 bits per character, last character in bits 2k-1..2k-2, $ encoded as 0;
// len = number of non-$ characters (k for k-mers).  Sorting by (key, len) is
// colex order: a run of trailing zero codes is told apart from $ padding by
// the shorter len, which is exactly where $ < A decides.
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "sbwt_gpu.h"
#include "common.h"

namespace sbwt {

namespace {

inline int code_of(uint8_t ch) {
    switch (ch) {
    case 'A': case 'a': return 0;
    case 'C': case 'c': return 1;
    case 'G': case 'g': return 2;
    case 'T': case 't': return 3;
    default: return -1;
    }
}

inline int nthreads() {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

// Parallel LSD radix sort of 64-bit keys on their low `bits` bits (8-bit
// digits), in place with one scratch buffer.
void radix_sort_u64(std::vector<uint64_t> &a, unsigned bits) {
    const size_t n = a.size();
    if (n < 2) return;
    std::vector<uint64_t> tmp(n);
    const int T = nthreads();
    std::vector<size_t> hist((size_t)T * 256);
    uint64_t *src = a.data(), *dst = tmp.data();
    const unsigned passes = (bits + 7) / 8;
    for (unsigned pass = 0; pass < passes; pass++) {
        const unsigned sh = 8 * pass;
        std::fill(hist.begin(), hist.end(), 0);
#pragma omp parallel num_threads(T)
        {
#ifdef _OPENMP
            const int t = omp_get_thread_num();
#else
            const int t = 0;
#endif
            const size_t b = n * (size_t)t / T, e = n * (size_t)(t + 1) / T;
            size_t *h = &hist[(size_t)t * 256];
            for (size_t i = b; i < e; i++) h[(src[i] >> sh) & 255]++;
#pragma omp barrier
#pragma omp single
            {
                size_t sum = 0;
                for (int d = 0; d < 256; d++)
                    for (int tt = 0; tt < T; tt++) {
                        size_t c = hist[(size_t)tt * 256 + d];
                        hist[(size_t)tt * 256 + d] = sum;
                        sum += c;
                    }
            }
            for (size_t i = b; i < e; i++) {
                const uint64_t v = src[i];
                dst[h[(v >> sh) & 255]++] = v;
            }
        }
        std::swap(src, dst);
    }
    if (src != a.data()) std::memcpy(a.data(), src, n * sizeof(uint64_t));
}

struct Node {
    uint64_t key;
    uint32_t len;
    bool operator<(const Node &o) const { return key < o.key || (key == o.key && len < o.len); }
    bool operator==(const Node &o) const { return key == o.key && len == o.len; }
};

}  // namespace

int build_sbwt(const uint8_t *seqs, const uint64_t *seq_starts, uint64_t n_seqs, uint32_t k, sbwt_built *out) {
    if (!out) return set_error("sbwt_build: out is NULL");
    std::memset(out, 0, sizeof(*out));
    if (k < 3 || k > 32) return set_error("sbwt_build: k must be in [3, 32], got %u", k);
    const uint64_t full = (k == 32) ? ~0ull : ((1ull << (2 * k)) - 1ull);
    const uint64_t mask_km1 = (1ull << (2 * (k - 1))) - 1ull;  // k-1 <= 31
    const unsigned top = 2 * (k - 1);

    // 1. every k-mer of every sequence as a colex key (rolling; ACGT only).
    std::vector<uint64_t> counts(n_seqs + 1, 0);
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t s = 0; s < (int64_t)n_seqs; s++) {
        const uint64_t b = seq_starts[s], e = seq_starts[s + 1];
        uint64_t run = 0, c = 0;
        for (uint64_t i = b; i < e; i++) {
            if (code_of(seqs[i]) < 0) { run = 0; continue; }
            if (++run >= k) c++;
        }
        counts[s + 1] = c;
    }
    for (uint64_t s = 0; s < n_seqs; s++) counts[s + 1] += counts[s];
    std::vector<uint64_t> keys;
    try { keys.resize(counts[n_seqs]); } catch (const std::bad_alloc &) {
        return set_error("sbwt_build: out of host memory for %llu k-mers", (unsigned long long)counts[n_seqs]);
    }
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t s = 0; s < (int64_t)n_seqs; s++) {
        const uint64_t b = seq_starts[s], e = seq_starts[s + 1];
        uint64_t run = 0, key = 0, o = counts[s];
        for (uint64_t i = b; i < e; i++) {
            const int cd = code_of(seqs[i]);
            if (cd < 0) { run = 0; key = 0; continue; }
            key = (key >> 2) | ((uint64_t)cd << top);
            if (++run >= k) keys[o++] = key & full;
        }
    }
    radix_sort_u64(keys, 2 * k);
    keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
    const uint64_t nk = keys.size();
    if (nk == 0) return set_error("sbwt_build: the input holds no k-mer of length %u", k);

    // 2. sources: x whose (k-1)-prefix is not the (k-1)-suffix of any k-mer.
    // Within the k-mers ending in c the prefixes (key & mask_km1) are sorted,
    // and so are the suffixes (key >> 2) over all k-mers: one merge per c.
    std::vector<uint64_t> cstart(5, nk);
    {
        uint64_t i = 0;
        for (int c = 0; c < 4; c++) {
            while (i < nk && (keys[i] >> top) < (uint64_t)c) i++;
            cstart[c] = i;
        }
        cstart[4] = nk;
    }
    std::vector<Node> dummies;
    std::vector<std::vector<uint64_t>> sources(4);
#pragma omp parallel for num_threads(4)
    for (int c = 0; c < 4; c++) {
        uint64_t y = 0;
        for (uint64_t x = cstart[c]; x < cstart[c + 1]; x++) {
            const uint64_t pre = keys[x] & mask_km1;
            while (y < nk && (keys[y] >> 2) < pre) y++;
            if (y >= nk || (keys[y] >> 2) != pre) sources[c].push_back(keys[x]);
        }
    }
    // 3. dummies $^{k-i} x[0..i-1], i = 0..k-1 (i = 0 is the root).
    for (int c = 0; c < 4; c++)
        for (uint64_t x : sources[c])
            for (uint32_t i = 0; i < k; i++) {
                const uint64_t pm = (i == 0) ? 0ull : (x & ((1ull << (2 * i)) - 1ull));
                dummies.push_back(Node{i == 0 ? 0ull : (pm << (2 * (k - i))), i});
            }
    if (dummies.empty()) dummies.push_back(Node{0ull, 0u});  // the root always exists
    std::sort(dummies.begin(), dummies.end());
    dummies.erase(std::unique(dummies.begin(), dummies.end()), dummies.end());
    const uint64_t nd = dummies.size();
    const uint64_t n = nk + nd;

    // 4. merged node order: positions of the dummies among the k-mers.
    std::vector<uint64_t> dpos(nd);
    {
        uint64_t x = 0;
        for (uint64_t d = 0; d < nd; d++) {
            const Node nd_ = dummies[d];
            while (x < nk && Node{keys[x], k} < nd_) x++;
            dpos[d] = x + d;
        }
    }
    // 5. bits.  Node v's group id is (key >> 2, min(len, k-1)); group-first
    // nodes get the out-label set.  For each c, the nodes w ending in c (in
    // order) need the group with id (key & mask_km1, len - 1): both sequences
    // are increasing, so one merge per c sets every 1.
    const uint64_t nwords = (n + 63) / 64;
    uint64_t *bits[4] = {nullptr, nullptr, nullptr, nullptr};
    for (int c = 0; c < 4; c++) {
        bits[c] = (uint64_t *)std::calloc(nwords ? nwords : 1, sizeof(uint64_t));
        if (!bits[c]) {
            for (int d = 0; d < c; d++) std::free(bits[d]);
            return set_error("sbwt_build: out of host memory for the bit vectors");
        }
    }
    // Random access to the merged node sequence: k-mer x sits at
    // x + (number of dummies before it); a small cursor structure serves the
    // monotone scans below.
    struct Cursor {
        const std::vector<uint64_t> *keys;
        const std::vector<Node> *dum;
        const std::vector<uint64_t> *dpos;
        uint32_t k;
        uint64_t v = 0, x = 0, d = 0;  // next node index, next k-mer, next dummy
        Node cur{0, 0};
        bool next() {  // advances to node v (returns false at the end)
            const uint64_t nk_ = keys->size(), nd_ = dum->size();
            if (x >= nk_ && d >= nd_) return false;
            if (d < nd_ && (*dpos)[d] == v) { cur = (*dum)[d]; d++; }
            else { cur = Node{(*keys)[x], k}; x++; }
            v++;
            return true;
        }
    };
    // Lazily enumerates the group-first nodes (id key, id len, node index).
    struct GroupCursor {
        Cursor cu;
        uint32_t k;
        bool have = false;
        uint64_t gk = 0, gv = 0;
        uint32_t gl = 0;
        bool next() {
            while (cu.next()) {
                const uint64_t nk_ = cu.cur.key >> 2;
                const uint32_t nl_ = std::min<uint32_t>(cu.cur.len, k - 1);
                if (!have || nk_ != gk || nl_ != gl) {
                    have = true; gk = nk_; gl = nl_; gv = cu.v - 1;
                    return true;
                }
            }
            return false;
        }
    };
    int err = 0;
#pragma omp parallel for num_threads(4) reduction(| : err)
    for (int c = 0; c < 4; c++) {
        Cursor cu{&keys, &dummies, &dpos, k};
        GroupCursor gc{Cursor{&keys, &dummies, &dpos, k}, k};
        bool gvalid = gc.next();
        while (cu.next()) {
            const Node w = cu.cur;
            if (w.len == 0) continue;  // root
            if ((w.key >> top) != (uint64_t)c) continue;
            const uint64_t sk = w.key & mask_km1;
            const uint32_t sl = w.len - 1;
            while (gvalid && (gc.gk < sk || (gc.gk == sk && gc.gl < sl))) gvalid = gc.next();
            if (!gvalid || gc.gk != sk || gc.gl != sl) { err = 1; break; }
            const uint64_t v = gc.gv;
            bits[c][v >> 6] |= 1ull << (63 - (v & 63));
        }
    }
    if (err) {
        for (int c = 0; c < 4; c++) std::free(bits[c]);
        return set_error("sbwt_build: internal error: a node has no predecessor group");
    }
    out->n_bits = n;
    out->n_kmers = nk;
    out->n_dummies = nd;
    out->n_words = nwords;
    for (int c = 0; c < 4; c++) out->bits[c] = bits[c];
    return 0;
}

}  // namespace sbwt

extern "C" int sbwt_build(const uint8_t *seqs, const uint64_t *seq_starts, uint64_t n_seqs, uint32_t k,
                          sbwt_built *out) {
    sbwt::clear_error();
    try {
        return sbwt::build_sbwt(seqs, seq_starts, n_seqs, k, out);
    } catch (const std::bad_alloc &) {
        return sbwt::set_error("sbwt_build: out of host memory");
    }
}

extern "C" void sbwt_build_free(sbwt_built *b) {
    if (!b) return;
    for (int c = 0; c < 4; c++) { std::free(b->bits[c]); b->bits[c] = nullptr; }
}

extern "C" int sbwt_write_bitvector(const char *path, const uint64_t *bits, uint64_t n_bits) {
    sbwt::clear_error();
    FILE *f = std::fopen(path, "wb");
    if (!f) return sbwt::set_error("cannot open %s for writing", path);
    unsigned char hdr[8];
    for (int i = 0; i < 8; i++) hdr[i] = (unsigned char)(n_bits >> (8 * i));
    int ok = std::fwrite(hdr, 1, 8, f) == 8;
    // position p at byte 8 + p/8, bit 7 - p%8 (MSB first): the big-endian
    // bytes of each in-memory word.  Bits past n are written as zero.
    const uint64_t nbytes = (n_bits + 7) / 8;
    std::vector<unsigned char> buf(1 << 20);
    uint64_t o = 0;
    while (ok && o < nbytes) {
        const uint64_t m = std::min<uint64_t>(buf.size(), nbytes - o);
        for (uint64_t b = 0; b < m; b++) {
            const uint64_t byte = o + b;
            const uint64_t w = bits[byte >> 3];
            unsigned char v = (unsigned char)(w >> (56 - 8 * (byte & 7)));
            const uint64_t first = byte * 8;
            if (first + 8 > n_bits) v &= (unsigned char)(0xFF << (first + 8 - n_bits));
            buf[b] = v;
        }
        ok = std::fwrite(buf.data(), 1, m, f) == m;
        o += m;
    }
    ok = (std::fclose(f) == 0) && ok;
    if (!ok) return sbwt::set_error("write to %s failed", path);
    return 0;
}
