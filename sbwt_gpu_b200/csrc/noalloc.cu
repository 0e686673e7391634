// noalloc.cu -- sbwt_search_reads_noalloc: the device-buffer search of a
// batch of reads (the same kernels as sbwt_search_reads) without any device
// allocation.  No counterpart in the reference, which allocates its buffers
// per search (include/gpu/kmer_data.hpp:28-54).
//
// Who needs it: callers that cannot call cudaMalloc while they search.  A
// process whose device memory is already handed out by another allocator
// (a framework's caching allocator that reserved the GPU up front) would
// see a cudaMalloc inside the library fail; an application that accounts
// for every device allocation itself cannot let a library grow buffers
// behind its back.  sbwt_search_reads grows its scratch buffers with
// cudaMalloc on first use; this entry point instead places all of its
// scratch (the packed letters, the per-row k-mer table, the scan block sums,
// the chunk table, the work-stealing counter and, for the per-k-mer kernels
// of a membership-only search, the answers) in one file-scope __device__
// array of kNoAllocBytes (32 MiB).  Every GPU that loads the library holds
// that array until the process exits.  The space a batch needs grows with
// its letters (2 bits each), its rows (16 bytes each) and its k-mers, so a
// batch of many short rows reaches the limit with fewer letters than one of
// long rows; a batch beyond it is rejected with an error that gives the
// bytes it needs.
//
// The first call on a device looks up the array's device address
// (cudaGetSymbolAddress, with that device current) and caches it; make that
// first call before any stream capture.  All calls share the array and it
// keeps the last call's contents: the counter is cleared on every call and
// everything else is overwritten before it is read.  Calls whose executions
// overlap on the GPU (two streams, or two host threads) race on the array.
#include <cstring>
#include <mutex>

#include "internal.h"

namespace sbwt {
namespace {

constexpr size_t kNoAllocBytes = 32ull << 20;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

std::mutex g_noalloc_mutex;
void *g_noalloc_ptr[kMaxDevices] = {nullptr};

// Device address of the scratch array on `device` (the current device).
int noalloc_scratch(int device, unsigned char **out) {
    if (device < 0 || device >= kMaxDevices) return set_error("device %d out of range", device);
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_ptr[device]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            return set_error("cudaGetSymbolAddress of the search scratch failed: %s", cudaGetErrorString(e));
        g_noalloc_ptr[device] = p;
    }
    *out = (unsigned char *)g_noalloc_ptr[device];
    return 0;
}

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

}  // namespace
}  // namespace sbwt

using namespace sbwt;

extern "C" int sbwt_search_reads_noalloc(sbwt_index *ix, const uint8_t *d_letters, uint64_t n_letters,
                                         const uint64_t *d_row_starts, uint64_t n_rows, uint64_t *d_answers,
                                         uint32_t *d_member_bits, uint64_t n_kmers, void *stream) {
    clear_error();
    if (!ix) return set_error("index is NULL");
    if (n_rows == 0 || n_kmers == 0) return 0;
    if (!d_letters || !d_row_starts) return set_error("NULL device pointer");
    if (!d_answers && !d_member_bits) return set_error("NULL answers and membership pointers");
    SBWT_CHECK_CUDA(cudaSetDevice(ix->device));
    const cudaStream_t s = (cudaStream_t)stream;
    SearchArgs a = base_args(ix, true);
    // membership only: the run-walking kernel writes the bitmap itself; the
    // per-k-mer kernels derive it from answers, which then go to the scratch
    const bool scratch_answers = !d_answers && !a.runs;
    // scratch layout: counter | kstart | scan block sums | chunk table | packed words | answers
    const u64 n_words = (n_letters + 32 + 31) / 32;
    const size_t off_kstart = 256;
    const size_t off_scan = align256(off_kstart + (n_rows + 1) * sizeof(u64));
    const size_t off_chunks = align256(off_scan + scan_scratch_words(n_rows) * sizeof(u64));
    const size_t off_words = align256(off_chunks + ((n_kmers + a.chunk - 1) / a.chunk) * sizeof(u32));
    const size_t off_answers = align256(off_words + n_words * sizeof(u64));
    const size_t need = scratch_answers ? off_answers + n_kmers * sizeof(u64) : off_words + n_words * sizeof(u64);
    if (need > kNoAllocBytes)
        return set_error("sbwt_search_reads_noalloc: this batch (%llu letters, %llu rows, %llu k-mers) needs %zu "
                         "bytes of scratch, more than the fixed %zu; split the batch or use sbwt_search_reads",
                         (unsigned long long)n_letters, (unsigned long long)n_rows, (unsigned long long)n_kmers,
                         need, kNoAllocBytes);
    unsigned char *base = nullptr;
    SBWT_TRY(noalloc_scratch(ix->device, &base));
    u64 *const words = (u64 *)(base + off_words);
    if (scratch_answers) d_answers = (u64 *)(base + off_answers);

    SBWT_TRY(launch_pack(d_letters, n_letters, words, s));
    a.counter = (unsigned long long *)base;  // launch_search clears it on the stream before the kernel
    a.kstart = (u64 *)(base + off_kstart);
    a.chunk_row = (u32 *)(base + off_chunks);
    SBWT_TRY(launch_kstart(d_row_starts, n_rows, ix->k, (u64 *)(base + off_kstart), (u64 *)(base + off_scan), s));
    SBWT_TRY(launch_chunk_rows(a.kstart, n_rows, n_kmers, a.chunk, (u32 *)(base + off_chunks), s));
    a.member = a.runs ? d_member_bits : nullptr;
    a.words = words;
    a.row_starts = d_row_starts;
    a.n_rows = n_rows;
    a.max_pos = (n_words - 1) * 32 - 1;
    a.answers = d_answers;  // NULL (run-walking kernel only): membership bitmap only
    a.n_kmers = n_kmers;
    SBWT_TRY(launch_search(ix, a, s, nullptr));
    if (d_member_bits && !a.runs) SBWT_TRY(launch_member_bits(d_answers, n_kmers, d_member_bits, s));
    return 0;
}
