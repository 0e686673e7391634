// pipeline.cu -- sbwt_search_reads_host: a batch of reads in host memory is
// streamed through the GPU in chunks of rows.  Three CUDA streams take
// turns; on each, a chunk's letters and row table go host->device, the chunk
// is packed and searched, and its answers come back device->host, so the
// copies of one chunk overlap the search of another while the host prepares
// the next.
//
// This replaces the strictly sequential host<->device chain of the reference
// (KmerSearch::search, include/epicseq/kmer_search.hpp:97-160: one H2D of the
// whole query, pack, positions, search, then one D2H of all results in
// ResultsPersister::save_results_to_file, results_persister.hpp:58-65).
#include <algorithm>
#include <cstring>
#include <vector>

#include "internal.h"

namespace sbwt {
namespace {

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
// that two chunks in flight stay well inside device memory.
constexpr u64 kChunkLetters = 64ull << 20;

}  // namespace
}  // namespace sbwt

using namespace sbwt;

namespace sbwt {
namespace {

// The pipeline behind both host entry points: exactly one of `answers`
// (u64 per k-mer) and `member` (bit j%32 of word j/32) is non-NULL.
int run_pipeline(sbwt_index *ix, const uint8_t *letters, uint64_t n_letters, const uint64_t *row_starts,
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
        u64 r0 = 0, k0 = 0;
        while (r0 < n_rows) {
            const u64 *first = row_starts + r0 + 1, *last = row_starts + n_rows + 1;
            // first row end at or past kChunkLetters letters; at least one row per chunk
            u64 r1 = (u64)(std::lower_bound(first, last, row_starts[r0] + kChunkLetters) - row_starts);
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
    const bool pin_out = answers && (n_kmers == 0 || is_pinned(answers));
    u64 max_letters = 0, max_rows = 0, max_k = 0;
    for (const Chunk &c : chunks) {
        max_letters = std::max(max_letters, c.l1 - c.l0);
        max_rows = std::max(max_rows, c.r1 - c.r0);
        max_k = std::max(max_k, c.nk);
    }
    const u64 max_words = (max_k + 31) / 32;
    for (int i = 0; i < kSlots; i++) {
        Workspace &w = ix->ws[i];
        SBWT_TRY(grow(w.letters, w.letters_cap, max_letters + 16));
        SBWT_TRY(grow(w.rows, w.rows_cap, max_rows + 1));
        SBWT_TRY(grow_host(w.h_rows, w.h_rows_cap, max_rows + 1));
        if (!pin_in) SBWT_TRY(grow_host(w.h_letters, w.h_letters_cap, max_letters + 16));
        if (answers) {
            SBWT_TRY(grow(w.answers, w.answers_cap, max_k));
            if (!pin_out) SBWT_TRY(grow_host(w.h_answers, w.h_answers_cap, max_k));
        } else {
            SBWT_TRY(grow(w.member, w.member_cap, max_words + 1));
            SBWT_TRY(grow_host(w.h_member, w.h_member_cap, max_words + 1));
        }
    }
    if (member) std::memset(member, 0, (n_kmers + 31) / 32 * sizeof(uint32_t));
    // pending[i]: chunk whose results sit in slot i's pinned staging
    long pending[kSlots];
    for (long &x : pending) x = -1;
    auto drain = [&](int slot) -> int {
        SBWT_CHECK_CUDA(cudaStreamSynchronize(ix->pipe_stream[slot]));
        if (pending[slot] >= 0) {
            const Chunk &c = chunks[(size_t)pending[slot]];
            if (answers) {
                std::memcpy(answers + c.k0, ix->ws[slot].h_answers, c.nk * sizeof(u64));
            } else {
                // the chunk's bitmap starts at bit k0 of the output: shift it into place
                const uint32_t *src = ix->ws[slot].h_member;
                const u64 nw = (c.nk + 31) / 32, w0 = c.k0 >> 5;
                const u32 sh = (u32)(c.k0 & 31u);
                const u64 out_words = (n_kmers + 31) / 32;
                if (sh == 0) {
                    for (u64 i = 0; i < nw; i++) member[w0 + i] |= src[i];
                } else {
                    // word w0+i gets the high part of src[i-1] and the low part of src[i]
                    uint32_t *dst = member + w0;
                    dst[0] |= src[0] << sh;
#pragma omp parallel for schedule(static) if (nw > (1u << 16))
                    for (int64_t i = 1; i < (int64_t)nw; i++) dst[i] |= (src[i] << sh) | (src[i - 1] >> (32u - sh));
                    if (w0 + nw < out_words) dst[nw] |= src[nw - 1] >> (32u - sh);
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
        const u64 nr = c.r1 - c.r0, nl = c.l1 - c.l0;
        uint64_t *hr = w.h_rows;
#pragma omp parallel for schedule(static) if (nr > (1u << 16))
        for (int64_t r = 0; r <= (int64_t)nr; r++) hr[r] = row_starts[c.r0 + r] - c.l0;
        SBWT_CHECK_CUDA(cudaMemcpyAsync(w.rows, w.h_rows, (nr + 1) * sizeof(u64), cudaMemcpyHostToDevice, s));
        if (pin_in) {
            SBWT_CHECK_CUDA(cudaMemcpyAsync(w.letters, letters + c.l0, nl, cudaMemcpyHostToDevice, s));
        } else {
            std::memcpy(w.h_letters, letters + c.l0, nl);
            SBWT_CHECK_CUDA(cudaMemcpyAsync(w.letters, w.h_letters, nl, cudaMemcpyHostToDevice, s));
        }
        if (answers) {
            SBWT_TRY(search_rows_device(ix, w, w.letters, nl, w.rows, nr, w.answers, nullptr, c.nk, s));
            if (c.nk) {
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
            pending[slot] = (long)b;
        }
    }
    for (size_t i = 0; i < (size_t)kSlots; i++) SBWT_TRY(drain((int)((chunks.size() + i) % kSlots)));
    return 0;
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
