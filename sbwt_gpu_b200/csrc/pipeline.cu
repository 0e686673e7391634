// pipeline.cu -- sbwt_search_reads_host: a batch of reads in host memory is
// streamed through the GPU in chunks of rows.  Six CUDA streams take turns;
// on each, a chunk's letters and row table go host->device, the chunk is
// packed and searched, and its answers come back device->host, so the
// copies of one chunk overlap the search of another while the host prepares
// the next.
//
// The u64 answers do not cross PCIe as such (8 bytes a k-mer would make the
// device->host copy the bound): while node ids fit in 32 bits, a chunk comes
// back as its membership bitmap, per-group offsets and the found node ids,
// and host threads expand them into the caller's answers.  Per chunk b the
// issuing thread issues b, starts the node-id copy of b-2 (its count is known
// once b-2's bitmap and offsets are in) and hands b-3 to an expander thread,
// which expands it with the other host threads while the issuing thread goes
// on; a slot's buffers are reused (by chunk b+6) only once its expansion is
// done.
// With few host threads, a share of the chunks comes back as u64 answers by
// DMA straight into the caller's pinned buffer instead (dense_share).
//
// This replaces the strictly sequential host<->device chain of the reference
// (KmerSearch::search, include/epicseq/kmer_search.hpp:97-160: one H2D of the
// whole query, pack, positions, search, then one D2H of all results in
// ResultsPersister::save_results_to_file, results_persister.hpp:58-65).
#include <algorithm>
#include <cstdlib>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <vector>
#if defined(__x86_64__)
#include <immintrin.h>
#endif

#include <cub/cub.cuh>
#include <omp.h>

#include "internal.h"

namespace sbwt {
namespace {

#if defined(__x86_64__)
inline void store_stream(u64 *p, u64 v) { _mm_stream_si64(reinterpret_cast<long long *>(p), (long long)v); }
inline void store_fence() { _mm_sfence(); }
#else
inline void store_stream(u64 *p, u64 v) { *p = v; }
inline void store_fence() {}
#endif

bool is_pinned(const void *p) {
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return at.type == cudaMemoryTypeHost;
}

struct Chunk {
    u64 r0, r1;  // rows [r0, r1)
    u64 l0, l1;  // letters [l0, l1)
    u64 k0, nk;  // answers [k0, k0 + nk)
};

// Letters per chunk: large enough to amortise the launches, small enough
// that two chunks in flight stay well inside device memory.  The
// environment variable SBWT_PIPELINE_CHUNK_LETTERS (at least 4096) sets
// another size.
constexpr u64 kChunkLetters = 64ull << 20;

u64 chunk_letters() {
    const char *e = std::getenv("SBWT_PIPELINE_CHUNK_LETTERS");
    if (!e || !*e) return kChunkLetters;
    const unsigned long long v = std::strtoull(e, nullptr, 10);
    return v >= 4096 ? (u64)v : kChunkLetters;
}

// Sparse answers.  A chunk's answers leave the device as its membership
// bitmap, the offset of every group of kGroupWords bitmap words (2048
// k-mers) into the list of found node ids, and that list (32 bits a node):
// 0.125 + 4 x (found fraction) bytes per k-mer instead of 8.  The host
// expands them into the u64 answers (~0 for an absent k-mer).
constexpr u32 kGroupWords = 64;
constexpr u32 kGroupWarps = 4;  // groups (warps) per block of group_nodes_kernel

// How a chunk's answers cross PCIe: u64 answers (dense), the sparse form, or
// both (split: some chunks dense, copied straight into the caller's pinned
// buffer by the copy engines while the expander thread expands the sparse
// ones).  Sparse needs 32-bit node ids.  The share of dense chunks per host
// thread count T is the measured optimum (large workload, 16-core host,
// sweep of T x share through sbwt_search_reads_host): the all-dense form
// runs at 6.1G k-mers/s whatever T (49 GB/s of copies), all-sparse at 3.0G /
// 5.7G / 8.2G / 12.5G for T = 2 / 3 / 4 / 6 (about 23 GB/s of expansion per
// expanding thread, T - 1 of them); the best split was 0.7 at T <= 2 (6.6G),
// 0.5 at T = 3 (8.3G), 0.3 at T = 4 (10.2G) and none from T = 6 (12.5G);
// T = 5 takes 0.15, between its neighbours.  The copy engines' writes into
// host memory slow the expansion down, so the optimum lies below the share
// that a plain rate model gives.  The environment variable
// SBWT_PIPELINE_TRANSFER = dense | sparse | hybrid (every fourth chunk
// dense) overrides the choice, and SBWT_PIPELINE_DENSE_SHARE = f in [0, 1]
// sets the share itself.
enum Transfer { kDense, kSparse, kSplit };
constexpr int kMinExpandThreads = 6;
constexpr double kDenseShare[kMinExpandThreads] = {0.7, 0.7, 0.7, 0.5, 0.3, 0.15};  // by T (T = 0 as 1)

int host_threads(const sbwt_index *ix) { return ix->host_threads > 0 ? ix->host_threads : omp_get_max_threads(); }

// Share of chunks whose u64 answers cross PCIe as such (the rest sparse),
// for an index of n columns searched with T host threads.
double dense_share(u64 n, int T, Transfer *mode) {
    Transfer t;
    double f;
    const char *e = std::getenv("SBWT_PIPELINE_TRANSFER");
    if (n > 0xffffffffull || (e && std::strcmp(e, "dense") == 0)) {
        t = kDense, f = 1.0;
    } else if (e && std::strcmp(e, "sparse") == 0) {
        t = kSparse, f = 0.0;
    } else if (e && std::strcmp(e, "hybrid") == 0) {
        t = kSplit, f = 0.25;
    } else if (const char *d = std::getenv("SBWT_PIPELINE_DENSE_SHARE")) {
        f = std::min(1.0, std::max(0.0, std::atof(d)));
        t = f >= 1.0 ? kDense : f <= 0.0 ? kSparse : kSplit;
    } else if (T >= kMinExpandThreads) {
        t = kSparse, f = 0.0;
    } else {
        t = kSplit, f = kDenseShare[T < 0 ? 0 : T];
    }
    if (mode) *mode = t;
    return f;
}

// gcnt[g] = found k-mers of group g; gcnt[ng] = 0 (the exclusive scan's total).
__global__ void group_count_kernel(const uint32_t *__restrict__ member, u64 nw, u64 ng, u64 *__restrict__ gcnt) {
    const u64 g = ((u64)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const u32 lane = threadIdx.x & 31u;
    if (g > ng) return;  // whole warps
    u32 c = 0;
    if (g < ng) {
        for (u32 h = 0; h < kGroupWords; h += 32u) {
            const u64 w = g * kGroupWords + h + lane;
            if (w < nw) c += (u32)__popc(member[w]);
        }
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if (lane == 0) gcnt[g] = c;
}

// nodes[goff[g] + i] = node id of the i-th found k-mer of group g.  One warp
// per group gathers them into shared memory, then stores them in order
// (coalesced).
__global__ void __launch_bounds__(32 * kGroupWarps) group_nodes_kernel(const uint32_t *__restrict__ member,
                                                                       const u64 *__restrict__ answers, u64 nw,
                                                                       u64 ng, const u64 *__restrict__ goff,
                                                                       uint32_t *__restrict__ nodes) {
    __shared__ uint32_t buf[kGroupWarps][kGroupWords * 32];
    const u32 lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const u64 g = (u64)blockIdx.x * kGroupWarps + warp;
    if (g >= ng) return;  // whole warps
    uint32_t *b = buf[warp];
    u32 o = 0;
    for (u32 h = 0; h < kGroupWords; h += 32u) {
        const u64 w = g * kGroupWords + h + lane;
        const u32 m = w < nw ? member[w] : 0u;
        const u32 c = (u32)__popc(m);
        u32 incl = c;
#pragma unroll
        for (u32 d = 1; d < 32u; d <<= 1) {
            const u32 x = __shfl_up_sync(0xffffffffu, incl, d);
            if (lane >= d) incl += x;
        }
        u32 q = o + incl - c;
        for (u32 r = m; r; r &= r - 1u) b[q++] = (uint32_t)answers[w * 32u + (u32)(__ffs(r) - 1)];
        o += __shfl_sync(0xffffffffu, incl, 31);
    }
    __syncwarp();
    uint32_t *dst = nodes + goff[g];
    for (u32 q = lane; q < o; q += 32u) dst[q] = b[q];
}

#if defined(__x86_64__)
// The expansion of the groups [g0, g1) with 32-byte streaming stores: the
// output is walked in 32-byte-aligned blocks of 4 answers (a block of 4
// absent k-mers is one constant store), with single 8-byte streaming stores
// for the unaligned head and the tail.  Host CPUs with AVX2 only.
__attribute__((target("avx2"))) void expand_groups_avx2(u64 *answers, u64 nk, const uint32_t *member,
                                                        const u64 *goff, const uint32_t *nodes, u64 g0, u64 g1) {
    const u64 j0 = g0 * kGroupWords * 32u, j1 = std::min<u64>(g1 * kGroupWords * 32u, nk);
    if (j0 >= j1) return;
    u64 o = goff[g0];
    auto bit = [&](u64 j) { return (member[j >> 5] >> (j & 31u)) & 1u; };
    u64 j = j0;
    // head: up to the first 32-byte boundary of the output
    while (j < j1 && (reinterpret_cast<uintptr_t>(answers + j) & 31u)) {
        const u32 b = bit(j);
        store_stream(answers + j, b ? (u64)nodes[o] : ~0ull);
        o += b;
        j++;
    }
    const __m256i none = _mm256_set1_epi64x(-1);
    for (; j + 4 <= j1; j += 4) {
        // the 4 bits of k-mers j .. j+3 (they may straddle two bitmap words)
        const u64 w = j >> 5;
        const u32 sh = (u32)(j & 31u);
        const u64 pair = (u64)member[w] | (sh > 28u ? (u64)member[w + 1] << 32 : 0ull);
        const u32 m4 = (u32)(pair >> sh) & 15u;
        __m256i v;
        if (m4 == 0) {
            v = none;
        } else {
            long long x[4];
            for (u32 i = 0; i < 4; i++) {
                const u32 b = (m4 >> i) & 1u;
                x[i] = b ? (long long)nodes[o] : -1ll;
                o += b;
            }
            v = _mm256_set_epi64x(x[3], x[2], x[1], x[0]);
        }
        _mm256_stream_si256(reinterpret_cast<__m256i *>(answers + j), v);
    }
    for (; j < j1; j++) {  // tail
        const u32 b = bit(j);
        store_stream(answers + j, b ? (u64)nodes[o] : ~0ull);
        o += b;
    }
}

bool host_has_avx2() {
    static const bool yes = __builtin_cpu_supports("avx2");
    return yes;
}

// The same with AVX-512: blocks of 8 answers, one 64-byte (whole cache line)
// streaming store each, built without branches: the found node ids of the
// block are expand-loaded into the lanes of its set membership bits, widened
// to 64 bits and blended with ~0 for the absent k-mers.
__attribute__((target("avx512f,avx512vl"))) void expand_groups_avx512(u64 *answers, u64 nk, const uint32_t *member,
                                                                      const u64 *goff, const uint32_t *nodes, u64 g0,
                                                                      u64 g1) {
    const u64 j0 = g0 * kGroupWords * 32u, j1 = std::min<u64>(g1 * kGroupWords * 32u, nk);
    if (j0 >= j1) return;
    u64 o = goff[g0];
    auto bit = [&](u64 j) { return (member[j >> 5] >> (j & 31u)) & 1u; };
    u64 j = j0;
    // head: up to the first 64-byte boundary of the output
    while (j < j1 && (reinterpret_cast<uintptr_t>(answers + j) & 63u)) {
        const u32 b = bit(j);
        store_stream(answers + j, b ? (u64)nodes[o] : ~0ull);
        o += b;
        j++;
    }
    const __m512i none = _mm512_set1_epi64(-1);
    for (; j + 8 <= j1; j += 8) {
        // the 8 bits of k-mers j .. j+7 (they may straddle two bitmap words, both below nk)
        const u64 w = j >> 5;
        const u32 sh = (u32)(j & 31u);
        const u64 pair = (u64)member[w] | (sh > 24u ? (u64)member[w + 1] << 32 : 0ull);
        const __mmask8 m8 = (__mmask8)((pair >> sh) & 0xffu);
        const __m256i n32 = _mm256_maskz_expandloadu_epi32(m8, nodes + o);  // reads popcount(m8) ids
        const __m512i v = _mm512_mask_blend_epi64(m8, none, _mm512_cvtepu32_epi64(n32));
        _mm512_stream_si512(reinterpret_cast<__m512i *>(answers + j), v);
        o += (u64)__builtin_popcount((unsigned)m8);
    }
    for (; j < j1; j++) {  // tail
        const u32 b = bit(j);
        store_stream(answers + j, b ? (u64)nodes[o] : ~0ull);
        o += b;
    }
}

bool host_has_avx512() {
    static const bool yes = __builtin_cpu_supports("avx512f") && __builtin_cpu_supports("avx512vl");
    if (const char *e = std::getenv("SBWT_EXPAND_AVX512")) return yes && e[0] != '0';
    return yes;
}
#endif

// answers[j] for the nk k-mers of one chunk from its sparse form (streaming
// stores: the answers are not read back by this thread).  nodes may be read
// one element past the chunk's found ids (a select instead of a branch), so
// its buffer has slack.
void expand_answers(u64 *answers, u64 nk, const uint32_t *member, const u64 *goff, const uint32_t *nodes, int threads) {
#if defined(__x86_64__)
    if (host_has_avx2() && (reinterpret_cast<uintptr_t>(answers) & 7u) == 0) {
        const u64 nw = (nk + 31) / 32, ng = (nw + kGroupWords - 1) / kGroupWords;
#pragma omp parallel num_threads(threads) if (nk > (1u << 16))
        {
            // contiguous runs of groups per thread: contiguous output, aligned blocks inside
            const u64 nt = (u64)omp_get_num_threads(), t = (u64)omp_get_thread_num();
            const u64 per = (ng + nt - 1) / nt;
            if (host_has_avx512())
                expand_groups_avx512(answers, nk, member, goff, nodes, std::min(ng, t * per), std::min(ng, (t + 1) * per));
            else
                expand_groups_avx2(answers, nk, member, goff, nodes, std::min(ng, t * per), std::min(ng, (t + 1) * per));
            store_fence();
        }
        return;
    }
#endif
    const u64 nw = (nk + 31) / 32, ng = (nw + kGroupWords - 1) / kGroupWords;
#pragma omp parallel num_threads(threads) if (nk > (1u << 16))
    {
#pragma omp for schedule(static)
        for (int64_t g = 0; g < (int64_t)ng; g++) {
            u64 o = goff[g];
            const u64 w1 = std::min<u64>((u64)(g + 1) * kGroupWords, nw);
            for (u64 w = (u64)g * kGroupWords; w < w1; w++) {
                const uint32_t m = member[w];
                u64 *dst = answers + w * 32u;
                const u32 lim = (u32)std::min<u64>(32u, nk - w * 32u);
                if (lim == 32u && m == 0u) {
                    for (u32 i = 0; i < 32u; i++) store_stream(dst + i, ~0ull);
                } else if (lim == 32u && m == ~0u) {
                    for (u32 i = 0; i < 32u; i++) store_stream(dst + i, (u64)nodes[o + i]);
                    o += 32u;
                } else {
                    for (u32 i = 0; i < lim; i++) {
                        const u32 bit = (m >> i) & 1u;
                        store_stream(dst + i, bit ? (u64)nodes[o] : ~0ull);
                        o += bit;
                    }
                }
            }
        }
        store_fence();
    }
}

}  // namespace
}  // namespace sbwt

using namespace sbwt;

namespace sbwt {
namespace {

struct ExpandJob {
    u64 *answers;
    u64 nk;
    const uint32_t *member;
    const u64 *goff;
    const uint32_t *nodes;
};

// One thread that expands the sparse answers of the chunks handed to it, in
// order, with `threads` OpenMP threads.  Destroying it (also on an error
// return of the pipeline) finishes the jobs already handed over.
struct Expander {
    std::thread th;
    std::mutex m;
    std::condition_variable cv;
    std::deque<std::pair<int, ExpandJob>> jobs;
    int busy[sbwt_index::kPipeSlots] = {};  // jobs queued or running per slot
    bool stop = false, running = false;
    int threads = 1;

    void start(int t) {
        threads = t;
        running = true;
        th = std::thread([this] {
            for (;;) {
                std::pair<int, ExpandJob> j;
                {
                    std::unique_lock<std::mutex> lk(m);
                    cv.wait(lk, [this] { return stop || !jobs.empty(); });
                    if (jobs.empty()) return;
                    j = jobs.front();
                    jobs.pop_front();
                }
                const ExpandJob &e = j.second;
                expand_answers(e.answers, e.nk, e.member, e.goff, e.nodes, threads);
                std::lock_guard<std::mutex> lk(m);
                busy[j.first]--;
                cv.notify_all();
            }
        });
    }
    void submit(int slot, const ExpandJob &e) {
        std::lock_guard<std::mutex> lk(m);
        jobs.emplace_back(slot, e);
        busy[slot]++;
        cv.notify_all();
    }
    void wait_slot(int slot) {
        if (!running) return;
        std::unique_lock<std::mutex> lk(m);
        cv.wait(lk, [&] { return busy[slot] == 0; });
    }
    void finish() {
        if (!running) return;
        {
            std::lock_guard<std::mutex> lk(m);
            stop = true;
            cv.notify_all();
        }
        th.join();
        running = false;
    }
    ~Expander() { finish(); }
};

// The pipeline behind both host entry points: exactly one of `answers`
// (u64 per k-mer) and `member` (bit j%32 of word j/32) is non-NULL.
int pipeline_chunks(sbwt_index *ix, const uint8_t *letters, uint64_t n_letters, const uint64_t *row_starts,
                    uint64_t n_rows, uint64_t *answers, uint32_t *member, uint64_t n_kmers) {
    if (!ix) return set_error("index is NULL");
    if (n_rows == 0) return 0;
    if (!letters || !row_starts || (n_kmers && !answers && !member)) return set_error("NULL host pointer");
    if (row_starts[n_rows] > n_letters) return set_error("row_starts[n_rows] exceeds n_letters");
    const u32 k = ix->k;
    // validation and the k-mer total, threaded (this host work precedes every copy)
    int64_t bad_row = -1;
    u64 kk = 0;
#pragma omp parallel for schedule(static) reduction(+ : kk) reduction(max : bad_row)
    for (int64_t r = 0; r < (int64_t)n_rows; r++) {
        const u64 a = row_starts[r], b = row_starts[r + 1];
        if (b < a) bad_row = std::max<int64_t>(bad_row, r);
        else kk += b - a >= k ? b - a - k + 1 : 0;
    }
    if (bad_row >= 0)
        return set_error("row_starts must be non-decreasing (row %lld)", (long long)bad_row);
    if (kk != n_kmers)
        return set_error("n_kmers = %llu but the rows hold %llu k-mers", (unsigned long long)n_kmers,
                         (unsigned long long)kk);
    // chunks of whole rows: the end of each is found by binary search in the sorted row starts
    std::vector<Chunk> chunks;
    {
        const u64 chunk_size = chunk_letters();
        u64 r0 = 0, k0 = 0;
        while (r0 < n_rows) {
            const u64 *first = row_starts + r0 + 1, *last = row_starts + n_rows + 1;
            // first row end at or past chunk_size letters; at least one row per chunk
            u64 r1 = (u64)(std::lower_bound(first, last, row_starts[r0] + chunk_size) - row_starts);
            r1 = std::min<u64>(std::max<u64>(r1, r0 + 1), n_rows);
            u64 nk = 0;
#pragma omp parallel for schedule(static) reduction(+ : nk) if (r1 - r0 > (1u << 16))
            for (int64_t r = (int64_t)r0; r < (int64_t)r1; r++) {
                const u64 len = row_starts[r + 1] - row_starts[r];
                nk += len >= k ? len - k + 1 : 0;
            }
            chunks.push_back(Chunk{r0, r1, row_starts[r0], row_starts[r1], k0, nk});
            k0 += nk;
            r0 = r1;
        }
    }
    SBWT_CHECK_CUDA(cudaSetDevice(ix->device));
    constexpr int kSlots = sbwt_index::kPipeSlots;
    for (int i = 0; i < kSlots; i++)
        if (!ix->pipe_stream[i]) SBWT_CHECK_CUDA(cudaStreamCreateWithFlags(&ix->pipe_stream[i], cudaStreamNonBlocking));
    const bool pin_in = is_pinned(letters);
    const int threads = host_threads(ix);
    const bool pin_out = answers && (n_kmers == 0 || is_pinned(answers));
    Transfer xfer = kDense;
    double share = answers ? dense_share(ix->n, threads, &xfer) : 1.0;
    if (xfer == kSplit && !pin_out) xfer = kSparse, share = 0.0;  // dense chunks go straight into a pinned buffer
    const bool sparse = answers && xfer != kDense;  // some chunks come back in sparse form
    // dense chunks: all of them, or (split) chunk b when floor((b+1) f) > floor(b f), f spread evenly
    auto dense_chunk = [&](size_t b) {
        if (xfer == kDense) return true;
        if (xfer == kSparse) return false;
        return (u64)((double)(b + 1) * share) > (u64)((double)b * share);
    };
    ix->pipe_h2d = ix->pipe_d2h = 0;
    u64 max_letters = 0, max_rows = 0, max_k = 0;
    for (const Chunk &c : chunks) {
        max_letters = std::max(max_letters, c.l1 - c.l0);
        max_rows = std::max(max_rows, c.r1 - c.r0);
        max_k = std::max(max_k, c.nk);
    }
    const u64 max_words = (max_k + 31) / 32;
    const u64 max_groups = (max_words + kGroupWords - 1) / kGroupWords;
    size_t scan_bytes = 0;  // scratch of the group-offset scan (w.goff after the offsets)
    if (sparse)
        SBWT_CHECK_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, (u64 *)nullptr, (u64 *)nullptr,
                                                      (int64_t)max_groups + 1));
    const u64 scan_words = scan_bytes / sizeof(u64) + 1;
    for (int i = 0; i < kSlots; i++) {
        Workspace &w = ix->ws[i];
        SBWT_TRY(grow(w.letters, w.letters_cap, max_letters + 16));
        SBWT_TRY(grow(w.rows, w.rows_cap, max_rows + 1));
        SBWT_TRY(grow_host(w.h_rows, w.h_rows_cap, max_rows + 1));
        if (!pin_in) SBWT_TRY(grow_host(w.h_letters, w.h_letters_cap, max_letters + 16));
        if (answers) SBWT_TRY(grow(w.answers, w.answers_cap, max_k));
        if (answers && !sparse) {
            if (!pin_out) SBWT_TRY(grow_host(w.h_answers, w.h_answers_cap, max_k));
        } else {
            SBWT_TRY(grow(w.member, w.member_cap, max_words + 1));
            SBWT_TRY(grow_host(w.h_member, w.h_member_cap, max_words + 1));
        }
        if (sparse) {
            SBWT_TRY(grow(w.goff, w.goff_cap, max_groups + 1 + scan_words));
            SBWT_TRY(grow(w.nodes, w.nodes_cap, max_k));
            SBWT_TRY(grow_host(w.h_goff, w.h_goff_cap, max_groups + 1));
            SBWT_TRY(grow_host(w.h_nodes, w.h_nodes_cap, max_k + 32));  // slack: expand_answers may read one past
        }
    }
    // member: each output word is assigned by the first chunk that reaches it and or-ed by the
    // next one where a chunk starts inside a word (chunks are drained in order), so the
    // output needs no clearing pass first
    // pending[i]: chunk whose results sit in slot i's pinned staging (or are
    // on their way there); stage[i]: 0 idle, 1 issued, 2 (sparse) node ids
    // requested
    long pending[kSlots];
    int stage[kSlots];
    for (int i = 0; i < kSlots; i++) pending[i] = -1, stage[i] = 0;
    // sparse: once the slot's bitmap and group offsets are in, the number of
    // node ids is known and their copy can start
    auto fetch_nodes = [&](int slot) -> int {
        if (!sparse || stage[slot] != 1) return 0;
        stage[slot] = 2;
        if (pending[slot] < 0) return 0;
        SBWT_CHECK_CUDA(cudaStreamSynchronize(ix->pipe_stream[slot]));
        const Chunk &c = chunks[(size_t)pending[slot]];
        Workspace &w = ix->ws[slot];
        const u64 ng = ((c.nk + 31) / 32 + kGroupWords - 1) / kGroupWords;
        const u64 found = w.h_goff[ng];
        if (found > c.nk)
            return set_error("sparse answers: %llu node ids for %llu k-mers", (unsigned long long)found,
                             (unsigned long long)c.nk);
        if (found)
            SBWT_CHECK_CUDA(cudaMemcpyAsync(w.h_nodes, w.nodes, found * sizeof(uint32_t), cudaMemcpyDeviceToHost,
                                            ix->pipe_stream[slot]));
        ix->pipe_d2h += found * sizeof(uint32_t);
        return 0;
    };
    // Sparse chunks are expanded by an expander thread of their own (with the
    // host threads but one), so that this thread keeps issuing chunks and
    // waiting on their copies meanwhile; a slot is reused only once the
    // expander is done with its host buffers.
    Expander ex;
    // Expander threads: the host threads but the issuing one; from 16 host threads on, three
    // quarters of them (measured on a 16-core host, large workload, three runs each: 12
    // expanding threads 14.2-14.9G k-mers/s, 15 threads 12.6-14.0G: the expansion is bound by
    // the host's memory writes, and fewer writers contend less).  SBWT_EXPAND_THREADS caps it.
    int expand_threads = threads >= 16 ? threads * 3 / 4 : threads > 1 ? threads - 1 : 1;
    if (const char *e = std::getenv("SBWT_EXPAND_THREADS")) {
        const int c = std::atoi(e);
        if (c > 0 && c < expand_threads) expand_threads = c;
    }
    if (sparse) ex.start(expand_threads);
    auto drain = [&](int slot) -> int {
        SBWT_TRY(fetch_nodes(slot));
        SBWT_CHECK_CUDA(cudaStreamSynchronize(ix->pipe_stream[slot]));
        stage[slot] = 0;
        if (pending[slot] >= 0) {
            const Chunk &c = chunks[(size_t)pending[slot]];
            Workspace &w = ix->ws[slot];
            if (sparse) {
                ex.submit(slot, ExpandJob{answers + c.k0, c.nk, w.h_member, w.h_goff, w.h_nodes});
            } else if (answers) {
                std::memcpy(answers + c.k0, w.h_answers, c.nk * sizeof(u64));
            } else {
                // the chunk's bitmap starts at bit k0 of the output: shift it into place
                const uint32_t *src = w.h_member;
                const u64 nw = (c.nk + 31) / 32, w0 = c.k0 >> 5;
                const u32 sh = (u32)(c.k0 & 31u);
                const u64 out_words = (n_kmers + 31) / 32;
                uint32_t *dst = member + w0;
                if (sh == 0) {
#pragma omp parallel for schedule(static) if (nw > (1u << 16))
                    for (int64_t i = 0; i < (int64_t)nw; i++) dst[i] = src[i];
                } else {
                    // word w0 already holds the previous chunk's low bits; word w0+i gets the high
                    // part of src[i-1] and the low part of src[i]; word w0+nw (if any) is the next
                    // chunk's first word, assigned here and or-ed by it
                    dst[0] |= src[0] << sh;
#pragma omp parallel for schedule(static) if (nw > (1u << 16))
                    for (int64_t i = 1; i < (int64_t)nw; i++) dst[i] = (src[i] << sh) | (src[i - 1] >> (32u - sh));
                    if (w0 + nw < out_words) dst[nw] = src[nw - 1] >> (32u - sh);
                }
            }
            pending[slot] = -1;
        }
        return 0;
    };
    for (size_t b = 0; b < chunks.size(); b++) {
        const int slot = (int)(b % kSlots);
        const Chunk &c = chunks[b];
        cudaStream_t s = ix->pipe_stream[slot];
        Workspace &w = ix->ws[slot];
        SBWT_TRY(drain(slot));  // slot's previous chunk has finished with its buffers
        ex.wait_slot(slot);     // and the expander with its host buffers
        const u64 nr = c.r1 - c.r0, nl = c.l1 - c.l0;
        uint64_t *hr = w.h_rows;
#pragma omp parallel for schedule(static) if (nr > (1u << 16))
        for (int64_t r = 0; r <= (int64_t)nr; r++) hr[r] = row_starts[c.r0 + r] - c.l0;
        SBWT_CHECK_CUDA(cudaMemcpyAsync(w.rows, w.h_rows, (nr + 1) * sizeof(u64), cudaMemcpyHostToDevice, s));
        ix->pipe_h2d += (nr + 1) * sizeof(u64) + nl;
        if (pin_in) {
            SBWT_CHECK_CUDA(cudaMemcpyAsync(w.letters, letters + c.l0, nl, cudaMemcpyHostToDevice, s));
        } else {
            std::memcpy(w.h_letters, letters + c.l0, nl);
            SBWT_CHECK_CUDA(cudaMemcpyAsync(w.letters, w.h_letters, nl, cudaMemcpyHostToDevice, s));
        }
        stage[slot] = 1;
        if (answers && !dense_chunk(b)) {
            // answers and bitmap in one search, then the found node ids gathered per group
            SBWT_TRY(search_rows_device(ix, w, w.letters, nl, w.rows, nr, w.answers, w.member, c.nk, s));
            if (c.nk) {
                const u64 nw = (c.nk + 31) / 32, ng = (nw + kGroupWords - 1) / kGroupWords;
                u64 *goff = w.goff;
                void *tmp = w.goff + max_groups + 1;
                size_t tb = 0;
                SBWT_CHECK_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, goff, goff, (int64_t)ng + 1, s));
                if (tb > scan_words * sizeof(u64)) return set_error("sparse answers: scan scratch too small");
                group_count_kernel<<<(unsigned)(((ng + 1) * 32 + 255) / 256), 256, 0, s>>>(w.member, nw, ng, goff);
                SBWT_CHECK_CUDA(cudaGetLastError());
                SBWT_CHECK_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tb, goff, goff, (int64_t)ng + 1, s));
                group_nodes_kernel<<<(unsigned)((ng + kGroupWarps - 1) / kGroupWarps), 32 * kGroupWarps, 0, s>>>(
                    w.member, w.answers, nw, ng, goff, w.nodes);
                SBWT_CHECK_CUDA(cudaGetLastError());
                SBWT_CHECK_CUDA(cudaMemcpyAsync(w.h_member, w.member, nw * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
                SBWT_CHECK_CUDA(cudaMemcpyAsync(w.h_goff, goff, (ng + 1) * sizeof(u64), cudaMemcpyDeviceToHost, s));
                ix->pipe_d2h += nw * sizeof(uint32_t) + (ng + 1) * sizeof(u64);
                pending[slot] = (long)b;
            }
        } else if (answers) {
            SBWT_TRY(search_rows_device(ix, w, w.letters, nl, w.rows, nr, w.answers, nullptr, c.nk, s));
            if (c.nk) {
                ix->pipe_d2h += c.nk * sizeof(u64);
                if (pin_out) {
                    SBWT_CHECK_CUDA(cudaMemcpyAsync(answers + c.k0, w.answers, c.nk * sizeof(u64),
                                                    cudaMemcpyDeviceToHost, s));
                } else {
                    SBWT_CHECK_CUDA(cudaMemcpyAsync(w.h_answers, w.answers, c.nk * sizeof(u64),
                                                    cudaMemcpyDeviceToHost, s));
                    pending[slot] = (long)b;
                }
            }
        } else if (c.nk) {
            SBWT_TRY(search_rows_device(ix, w, w.letters, nl, w.rows, nr, nullptr, w.member, c.nk, s));
            SBWT_CHECK_CUDA(cudaMemcpyAsync(w.h_member, w.member, (c.nk + 31) / 32 * sizeof(uint32_t),
                                            cudaMemcpyDeviceToHost, s));
            ix->pipe_d2h += (c.nk + 31) / 32 * sizeof(uint32_t);
            pending[slot] = (long)b;
        }
        if (sparse) {
            // node ids of chunk b-2 start on their way (its bitmap and offsets have had a whole
            // iteration to arrive); chunk b-3's are in, it is expanded while b-1 and b run
            if (b >= 2) SBWT_TRY(fetch_nodes((int)((b - 2) % kSlots)));
            if (b >= 3) SBWT_TRY(drain((int)((b - 3) % kSlots)));
        }
    }
    // the chunks still in flight, oldest first
    for (size_t i = 0; i < (size_t)kSlots; i++) SBWT_TRY(drain((int)((chunks.size() + i) % kSlots)));
    ex.finish();
    return 0;
}

// An error leaves no copy or kernel of the call in flight: the next call
// reuses the buffers they would write.
int run_pipeline(sbwt_index *ix, const uint8_t *letters, uint64_t n_letters, const uint64_t *row_starts,
                 uint64_t n_rows, uint64_t *answers, uint32_t *member, uint64_t n_kmers) {
    const int rc = pipeline_chunks(ix, letters, n_letters, row_starts, n_rows, answers, member, n_kmers);
    if (rc && ix)
        for (cudaStream_t st : ix->pipe_stream)
            if (st) cudaStreamSynchronize(st);
    return rc;
}

}  // namespace
}  // namespace sbwt

extern "C" int sbwt_search_reads_host(sbwt_index *ix, const uint8_t *letters, uint64_t n_letters,
                                      const uint64_t *row_starts, uint64_t n_rows, uint64_t *answers,
                                      uint64_t n_kmers) {
    clear_error();
    if (n_kmers && !answers) return set_error("NULL host pointer");
    return run_pipeline(ix, letters, n_letters, row_starts, n_rows, answers, nullptr, n_kmers);
}

extern "C" int sbwt_search_reads_host_member(sbwt_index *ix, const uint8_t *letters, uint64_t n_letters,
                                             const uint64_t *row_starts, uint64_t n_rows, uint32_t *member_bits,
                                             uint64_t n_kmers) {
    clear_error();
    if (n_kmers && !member_bits) return set_error("NULL host pointer");
    return run_pipeline(ix, letters, n_letters, row_starts, n_rows, nullptr, member_bits, n_kmers);
}

extern "C" int sbwt_set_host_threads(sbwt_index *ix, int threads) {
    clear_error();
    if (!ix) return set_error("index is NULL");
    if (threads < 0) return set_error("host threads must be >= 0 (0: the OpenMP default)");
    ix->host_threads = threads;
    return 0;
}

extern "C" double sbwt_pipeline_dense_share(uint64_t n_columns, int host_threads) {
    return dense_share(n_columns, host_threads > 0 ? host_threads : omp_get_max_threads(), nullptr);
}

// ------------------------------------------------------------ several GPUs
//
// A batch in host memory spread over several index replicas (one per GPU):
// the rows are cut into contiguous ranges of near-equal k-mer counts (a row
// is never split), each replica runs the host pipeline on its range from a
// host thread of its own, and writes its disjoint slice of the caller's
// answers.  No exchange between the GPUs: the index is read-only and every
// k-mer independent.  The reference pins device 0 (include/parameters.hpp:81).

extern "C" int sbwt_partition_rows(const uint64_t *row_starts, uint64_t n_rows, uint32_t k, int n_parts,
                                   uint64_t *bounds) {
    clear_error();
    if (!row_starts || !bounds || n_parts < 1) return set_error("sbwt_partition_rows: bad arguments");
    // k-mers before each row, then the first row at or past each part's share
    std::vector<u64> before(n_rows + 1);
    u64 t = 0;
    for (u64 r = 0; r < n_rows; r++) {
        before[r] = t;
        if (row_starts[r + 1] < row_starts[r]) return set_error("row_starts must be non-decreasing (row %llu)",
                                                                (unsigned long long)r);
        const u64 len = row_starts[r + 1] - row_starts[r];
        t += len >= k ? len - k + 1 : 0;
    }
    before[n_rows] = t;
    bounds[0] = 0;
    for (int i = 1; i < n_parts; i++) {
        const u64 target = (u64)((unsigned __int128)t * (unsigned)i / (unsigned)n_parts);
        // the row boundary whose k-mer count before it is nearest to the target
        u64 r = (u64)(std::lower_bound(before.begin(), before.end(), target) - before.begin());
        if (r > 0 && target - before[r - 1] < before[r] - target) r--;
        bounds[i] = std::max<u64>(r, bounds[i - 1]);
    }
    bounds[n_parts] = n_rows;
    return 0;
}

extern "C" int sbwt_search_reads_host_multi(sbwt_index *const *indexes, int n_indexes, const uint8_t *letters,
                                            uint64_t n_letters, const uint64_t *row_starts, uint64_t n_rows,
                                            uint64_t *answers, uint64_t n_kmers) {
    clear_error();
    if (!indexes || n_indexes < 1) return set_error("sbwt_search_reads_host_multi: no index");
    for (int i = 0; i < n_indexes; i++) {
        if (!indexes[i]) return set_error("index %d is NULL", i);
        if (indexes[i]->k != indexes[0]->k || indexes[i]->n != indexes[0]->n || indexes[i]->C[4] != indexes[0]->C[4])
            return set_error("index %d is not a replica of index 0", i);
        for (int j = 0; j < i; j++)
            if (indexes[j] == indexes[i]) return set_error("index %d is passed twice", i);
    }
    if (n_rows == 0) return 0;
    if (!letters || !row_starts || (n_kmers && !answers)) return set_error("NULL host pointer");
    const u32 k = indexes[0]->k;
    std::vector<u64> bounds((size_t)n_indexes + 1);
    SBWT_TRY(sbwt_partition_rows(row_starts, n_rows, k, n_indexes, bounds.data()));
    // answers of part i start at the k-mers before its first row
    std::vector<u64> k0((size_t)n_indexes + 1, 0);
    for (int i = 0; i < n_indexes; i++) {
        u64 nk = 0;
        for (u64 r = bounds[i]; r < bounds[i + 1]; r++) {
            const u64 len = row_starts[r + 1] - row_starts[r];
            nk += len >= k ? len - k + 1 : 0;
        }
        k0[i + 1] = k0[i] + nk;
    }
    if (k0[n_indexes] != n_kmers)
        return set_error("n_kmers = %llu but the rows hold %llu k-mers", (unsigned long long)n_kmers,
                         (unsigned long long)k0[n_indexes]);
    // host threads: the OpenMP threads of this call shared among the replicas (unless set per index)
    const int share = std::max(1, omp_get_max_threads() / n_indexes);
    std::vector<int> rc((size_t)n_indexes, 0);
    std::vector<std::string> err((size_t)n_indexes);
    std::vector<std::thread> th;
    for (int i = 0; i < n_indexes; i++) {
        th.emplace_back([&, i] {
            sbwt_index *ix = indexes[i];
            const int saved = ix->host_threads;
            if (saved == 0) ix->host_threads = share;
            rc[i] = run_pipeline(ix, letters, n_letters, row_starts + bounds[i], bounds[i + 1] - bounds[i],
                                 answers ? answers + k0[i] : nullptr, nullptr, k0[i + 1] - k0[i]);
            if (rc[i]) err[i] = last_error();
            ix->host_threads = saved;
        });
    }
    for (auto &t : th) t.join();
    for (int i = 0; i < n_indexes; i++)
        if (rc[i]) return set_error("replica %d (device %d): %s", i, indexes[i]->device, err[i].c_str());
    return 0;
}
