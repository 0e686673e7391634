// packed_runs.cu -- the reference's kernel contract (sbwt_search_packed:
// packed k-mer string + a positions array overwritten by the answers,
// include/gpu/search_kernel.hpp:61-104) on the run-walking kernel.
//
// K-mers whose positions follow each other (positions[j] = positions[j-1] + 1)
// are consecutive windows of the packed string, so they form a run the walk
// can take right to left with the absent-run skip and backward steps, whatever
// the reads were; the reference's own positions (one run per read,
// include/gpu/positions_kernel.hpp:18-36) are of that kind.  The run starts
// become a row table (first k-mer index and letter offset of each run), after
// which the search is the one of sbwt_search_reads, writing its answers over
// the positions.  When the runs are short (random positions) the per-k-mer
// search is used instead.  The choice is made on the device: the run count
// never comes back to the host, the run table is sized for the most runs the
// walk takes (a quarter of the k-mers), both searches are launched and each
// returns at once unless it is the one the count chose, so a call is
// stream-ordered with no host wait.
#include <cub/cub.cuh>

#include "internal.h"

namespace sbwt {
namespace {

// The positions are read once.  Pass 1 (kThreads x kPerThread consecutive
// k-mers per block) writes the run-start bitmap (bit j of word j/32 = k-mer j
// starts a run) and counts each block's starts; an exclusive scan of the
// counts gives each block its first run index; pass 2 reads only the bitmap
// (one word per thread, kWords words per block: the same k-mers as pass 1's
// block) and writes the run table and the chunk-row table.
constexpr u32 kThreads = 256;
constexpr u32 kPerThread = 16;
constexpr u32 kBlockItems = kThreads * kPerThread;
constexpr u32 kWords = kBlockItems / 32;  // pass 2 threads per block

__global__ void __launch_bounds__(kThreads) start_bits_kernel(const u64 *__restrict__ pos, u64 n,
                                                              uint32_t *__restrict__ bits,
                                                              u64 *__restrict__ block_count) {
    __shared__ u32 warp_sum[kThreads / 32];
    const u64 base = (u64)blockIdx.x * kBlockItems;
    const u32 lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    u64 v[kPerThread], before[kPerThread];
#pragma unroll
    for (u32 it = 0; it < kPerThread; it++) {
        const u64 j = base + it * kThreads + threadIdx.x;
        v[it] = j < n ? pos[j] : 0ull;
        before[it] = (lane == 0 && j > 0 && j - 1u < n) ? pos[j - 1u] : 0ull;  // the word's left neighbour
    }
    u32 c = 0;
#pragma unroll
    for (u32 it = 0; it < kPerThread; it++) {
        const u64 j = base + it * kThreads + threadIdx.x;
        u64 prev = __shfl_up_sync(0xffffffffu, v[it], 1);
        if (lane == 0) prev = before[it];
        const bool st = j < n && (j == 0 || v[it] != prev + 1u);
        const u32 m = __ballot_sync(0xffffffffu, st);
        if (lane == 0) bits[j >> 5] = m;  // every word of the block, zero past n
        c += (u32)__popc(m);
    }
    if (lane == 0) warp_sum[warp] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        u32 t = 0;
        for (u32 w = 0; w < kThreads / 32; w++) t += warp_sum[w];
        block_count[blockIdx.x] = t;
    }
}

// Run r (in order of its first k-mer j): kstart[r] = j, row_start[r] =
// pos[j]; kstart[n_rows] = n.  chunk_row[c] (chunks of chunk_words * 32
// k-mers) = the run holding k-mer c * chunk_words * 32 = (runs starting at or
// before it) - 1.
__global__ void __launch_bounds__(kWords) run_table_kernel(const u64 *__restrict__ pos, u64 n,
                                                           const uint32_t *__restrict__ bits,
                                                           const u64 *__restrict__ block_offset,
                                                           const u64 *__restrict__ runs_dev, u32 chunk_words,
                                                           u64 *__restrict__ kstart, u64 *__restrict__ row_start,
                                                           u32 *__restrict__ chunk_row) {
    const u64 n_rows = *runs_dev;
    if (!runs_usable(n_rows, n)) return;  // the per-k-mer search takes this call
    __shared__ u32 warp_tot[kWords / 32];
    const u32 lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const u64 w = (u64)blockIdx.x * kWords + threadIdx.x;
    const u32 m = bits[w];
    const u32 c = (u32)__popc(m);
    u32 incl = c;  // inclusive scan over the warp
#pragma unroll
    for (u32 o = 1; o < 32u; o <<= 1) {
        const u32 x = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += x;
    }
    if (lane == 31u) warp_tot[warp] = incl;
    __syncthreads();
    u64 out = block_offset[blockIdx.x] + (incl - c);
    for (u32 q = 0; q < warp; q++) out += warp_tot[q];
    const u64 j0 = w * 32u;
    if (j0 < n && w % chunk_words == 0) chunk_row[w / chunk_words] = (u32)(out + (m & 1u) - 1u);
    for (u32 b = m; b; b &= b - 1u) {
        const u64 j = j0 + (u32)(__ffs(b) - 1);
        kstart[out] = j;
        row_start[out] = pos[j];
        out++;
    }
    if (w == 0) kstart[n_rows] = n;
}

}  // namespace

// Builds the run table of `positions` into w.kstart (runs + 1 entries),
// w.rows (runs row starts) and w.chunk_row (the run of every chunk-th k-mer;
// chunk a multiple of 32), where runs = *runs_dev, the run count, left on the
// device; when runs_usable(runs, n_kmers) is false nothing is written and the
// per-k-mer search takes the call.  No host wait.
int packed_runs(Workspace &w, const u64 *positions, u64 n_kmers, u32 chunk, cudaStream_t s, const u64 **runs_dev) {
    *runs_dev = nullptr;
    if (chunk == 0 || chunk % 32u) return set_error("run chunks must be whole bitmap words");
    const u64 nb = (n_kmers + kBlockItems - 1) / kBlockItems;
    // w.scan: block counts (then their exclusive scan, in place; the total at counts[nb]), the
    // scan's scratch, the start bitmap
    size_t tmp_bytes = 0;
    SBWT_CHECK_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, w.scan, w.scan, (int64_t)nb + 1, s));
    const u64 tmp_words = tmp_bytes / sizeof(u64) + 1;
    SBWT_TRY(grow(w.scan, w.scan_cap, nb + 1 + tmp_words + nb * (kWords / 2)));
    const u64 max_runs = n_kmers / kMinRunKmers;
    SBWT_TRY(grow(w.kstart, w.kstart_cap, max_runs + 1));
    SBWT_TRY(grow(w.rows, w.rows_cap, max_runs + 1));
    SBWT_TRY(grow(w.chunk_row, w.chunk_cap, (n_kmers + chunk - 1) / chunk));
    u64 *counts = w.scan, *tmp = w.scan + nb + 1;
    uint32_t *bits = reinterpret_cast<uint32_t *>(tmp + tmp_words);
    SBWT_CHECK_CUDA(cudaMemsetAsync(counts + nb, 0, sizeof(u64), s));
    start_bits_kernel<<<(unsigned)nb, kThreads, 0, s>>>(positions, n_kmers, bits, counts);
    SBWT_CHECK_CUDA(cudaGetLastError());
    SBWT_CHECK_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, counts, counts, (int64_t)nb + 1, s));
    run_table_kernel<<<(unsigned)nb, kWords, 0, s>>>(positions, n_kmers, bits, counts, counts + nb, chunk / 32u,
                                                     w.kstart, w.rows, w.chunk_row);
    SBWT_CHECK_CUDA(cudaGetLastError());
    *runs_dev = counts + nb;
    return 0;
}

}  // namespace sbwt
