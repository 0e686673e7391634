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

struct RunStart {
    const u64 *pos;
    __device__ __forceinline__ bool operator()(const u64 j) const { return j == 0 || pos[j] != pos[j - 1] + 1u; }
};

__global__ void count_runs_kernel(const u64 *__restrict__ pos, u64 n, unsigned long long *__restrict__ count) {
    const u64 j = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    const bool start = j < n && (j == 0 || pos[j] != pos[j - 1] + 1u);
    const u32 m = __ballot_sync(0xffffffffu, start);
    if ((threadIdx.x & 31u) == 0 && m) atomicAdd(count, (unsigned long long)__popc(m));
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
    SBWT_TRY(grow(w.counter, w.counter_cap, 1));
    SBWT_CHECK_CUDA(cudaMemsetAsync(w.counter, 0, sizeof(unsigned long long), s));
    const unsigned blocks = (unsigned)((n_kmers + 255) / 256);
    count_runs_kernel<<<blocks, 256, 0, s>>>(positions, n_kmers, w.counter);
    SBWT_CHECK_CUDA(cudaGetLastError());
    unsigned long long runs = 0;
    SBWT_CHECK_CUDA(cudaMemcpyAsync(&runs, w.counter, sizeof runs, cudaMemcpyDeviceToHost, s));
    SBWT_CHECK_CUDA(cudaStreamSynchronize(s));
    if (runs == 0 || runs * 4 > n_kmers) return 0;
    SBWT_TRY(grow(w.kstart, w.kstart_cap, runs + 1));
    SBWT_TRY(grow(w.rows, w.rows_cap, runs + 1));
    size_t tmp_bytes = 0;
    cub::CountingInputIterator<u64> idx(0);
    SBWT_CHECK_CUDA(cub::DeviceSelect::If(nullptr, tmp_bytes, idx, w.kstart, w.counter, (int64_t)n_kmers,
                                          RunStart{positions}, s));
    SBWT_TRY(grow(w.scan, w.scan_cap, tmp_bytes / sizeof(u64) + 1));
    SBWT_CHECK_CUDA(cub::DeviceSelect::If(w.scan, tmp_bytes, idx, w.kstart, w.counter, (int64_t)n_kmers,
                                          RunStart{positions}, s));
    run_rows_kernel<<<(unsigned)((runs + 255) / 256), 256, 0, s>>>(positions, w.kstart, runs, n_kmers, w.rows);
    SBWT_CHECK_CUDA(cudaGetLastError());
    *n_rows = runs;
    return 0;
}

}  // namespace sbwt
