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
// search is used instead.
#include <cub/cub.cuh>

#include "internal.h"

namespace sbwt {
namespace {

// Run starts are found in two passes over the positions, each thread block
// taking kBlockItems consecutive k-mers: pass 1 counts the starts of each
// block, an exclusive scan of the counts gives each block its first output
// slot, and pass 2 writes the start indices in order (warp ballots, then the
// warps' counts in shared memory).
constexpr u32 kThreads = 256;
constexpr u32 kPerThread = 16;
constexpr u32 kBlockItems = kThreads * kPerThread;

__device__ __forceinline__ bool run_start(const u64 *__restrict__ pos, u64 j) {
    return j == 0 || pos[j] != pos[j - 1] + 1u;
}

__global__ void __launch_bounds__(kThreads) block_starts_kernel(const u64 *__restrict__ pos, u64 n,
                                                                u64 *__restrict__ block_count) {
    __shared__ u32 warp_sum[kThreads / 32];
    const u64 base = (u64)blockIdx.x * kBlockItems;
    u32 c = 0;
#pragma unroll 4
    for (u32 it = 0; it < kPerThread; it++) {
        const u64 j = base + it * kThreads + threadIdx.x;
        c += (j < n && run_start(pos, j)) ? 1u : 0u;
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31u) == 0) warp_sum[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        u32 t = 0;
        for (u32 w = 0; w < kThreads / 32; w++) t += warp_sum[w];
        block_count[blockIdx.x] = t;
    }
}

// kstart[block_offset[b] + i] = index of the i-th run start of block b.
__global__ void __launch_bounds__(kThreads) write_starts_kernel(const u64 *__restrict__ pos, u64 n,
                                                                const u64 *__restrict__ block_offset,
                                                                u64 *__restrict__ kstart) {
    __shared__ u32 warp_cnt[kThreads / 32];
    const u64 base = (u64)blockIdx.x * kBlockItems;
    const u32 lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    u64 out = block_offset[blockIdx.x];
    for (u32 it = 0; it < kPerThread; it++) {
        const u64 j = base + it * kThreads + threadIdx.x;
        const bool st = j < n && run_start(pos, j);
        const u32 m = __ballot_sync(0xffffffffu, st);
        if (lane == 0) warp_cnt[warp] = __popc(m);
        __syncthreads();
        u32 before = 0, total = 0;
        for (u32 w = 0; w < kThreads / 32; w++) {
            const u32 cw = warp_cnt[w];
            before += w < warp ? cw : 0u;
            total += cw;
        }
        if (st) kstart[out + before + __popc(m & ((1u << lane) - 1u))] = j;
        out += total;
        __syncthreads();
    }
}

// row_start[r] = letter offset of run r's first k-mer; kstart[n_rows] = n.
__global__ void run_rows_kernel(const u64 *__restrict__ pos, u64 *__restrict__ kstart, u64 n_rows, u64 n,
                                u64 *__restrict__ row_start) {
    const u64 r = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (r < n_rows) row_start[r] = pos[kstart[r]];
    if (r == 0) kstart[n_rows] = n;
}

}  // namespace

// Builds the run table of `positions` into w.kstart (n_rows + 1 entries) and
// w.rows (n_rows row starts); *n_rows = 0 when the runs average fewer than
// four k-mers (the caller then searches every k-mer).  Synchronises s once
// (the run count comes back to the host to size the tables).
int packed_runs(Workspace &w, const u64 *positions, u64 n_kmers, cudaStream_t s, u64 *n_rows) {
    *n_rows = 0;
    const u64 nb = (n_kmers + kBlockItems - 1) / kBlockItems;
    // w.scan: block counts, then their exclusive scan in place, then the scan's scratch
    size_t tmp_bytes = 0;
    SBWT_CHECK_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, w.scan, w.scan, (int64_t)nb + 1, s));
    SBWT_TRY(grow(w.scan, w.scan_cap, nb + 1 + tmp_bytes / sizeof(u64) + 1));
    u64 *counts = w.scan, *tmp = w.scan + nb + 1;
    SBWT_CHECK_CUDA(cudaMemsetAsync(counts + nb, 0, sizeof(u64), s));
    block_starts_kernel<<<(unsigned)nb, kThreads, 0, s>>>(positions, n_kmers, counts);
    SBWT_CHECK_CUDA(cudaGetLastError());
    SBWT_CHECK_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, counts, counts, (int64_t)nb + 1, s));
    u64 runs = 0;
    SBWT_CHECK_CUDA(cudaMemcpyAsync(&runs, counts + nb, sizeof runs, cudaMemcpyDeviceToHost, s));
    SBWT_CHECK_CUDA(cudaStreamSynchronize(s));
    if (runs == 0 || runs * 4 > n_kmers) return 0;
    SBWT_TRY(grow(w.kstart, w.kstart_cap, runs + 1));
    SBWT_TRY(grow(w.rows, w.rows_cap, runs + 1));
    write_starts_kernel<<<(unsigned)nb, kThreads, 0, s>>>(positions, n_kmers, counts, w.kstart);
    run_rows_kernel<<<(unsigned)((runs + 255) / 256), 256, 0, s>>>(positions, w.kstart, runs, n_kmers, w.rows);
    SBWT_CHECK_CUDA(cudaGetLastError());
    *n_rows = runs;
    return 0;
}

}  // namespace sbwt
