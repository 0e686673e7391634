// noalloc.cu -- sbwt_search_reads_noalloc: the device-buffer search of a
// batch of reads (the same kernels as sbwt_search_reads) without any device
// allocation.
//
// Who needs it: callers that must not allocate device memory at search
// time -- a caller capturing the search into its own CUDA graph (cudaMalloc
// is not capturable and would break the capture), or a process whose device
// memory is already handed out by another allocator (a framework's caching
// allocator that reserved the whole GPU), where a cudaMalloc inside the
// library would fail.  sbwt_search_reads grows its scratch buffers with
// cudaMalloc on first use; this entry point instead places all of its
// scratch (the packed letters, the per-row k-mer table, the scan block sums,
// the chunk table and the work-stealing counter) in one file-scope
// __device__ array of kNoAllocBytes (32 MiB).  Every GPU that loads the
// library holds that array until the process exits.
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
    if (!d_letters || !d_row_starts || !d_answers) return set_error("NULL device pointer");
    SBWT_CHECK_CUDA(cudaSetDevice(ix->device));
    const cudaStream_t s = (cudaStream_t)stream;
    const u32 chunk = search_chunk(ix, true);
    // scratch layout: counter | kstart | scan block sums | chunk table | packed words
    const u64 n_words = (n_letters + 32 + 31) / 32;
    const size_t off_kstart = 256;
    const size_t off_scan = align256(off_kstart + (n_rows + 1) * sizeof(u64));
    const size_t off_chunks = align256(off_scan + scan_scratch_words(n_rows) * sizeof(u64));
    const size_t off_words = align256(off_chunks + ((n_kmers + chunk - 1) / chunk) * sizeof(u32));
    const size_t need = off_words + n_words * sizeof(u64);
    if (need > kNoAllocBytes)
        return set_error("sbwt_search_reads_noalloc: this batch needs %zu bytes of scratch, more than its fixed "
                         "%zu (about %llu letters per call at most); split the batch or use sbwt_search_reads",
                         need, kNoAllocBytes, (unsigned long long)((kNoAllocBytes / 2) * 4));
    unsigned char *base = nullptr;
    SBWT_TRY(noalloc_scratch(ix->device, &base));
    unsigned long long *counter = (unsigned long long *)base;
    u64 *kstart = (u64 *)(base + off_kstart);
    u64 *scan = (u64 *)(base + off_scan);
    u32 *chunk_row = (u32 *)(base + off_chunks);
    u64 *words = (u64 *)(base + off_words);

    SBWT_TRY(launch_pack(d_letters, n_letters, words, s));
    SBWT_TRY(launch_kstart(d_row_starts, n_rows, ix->k, kstart, scan, s));
    SBWT_TRY(launch_chunk_rows(kstart, n_rows, n_kmers, chunk, chunk_row, s));
    SearchArgs a;
    std::memset(&a, 0, sizeof(a));
    a.lines = ix->d_lines;
    a.lpc = ix->lpc;
    a.bits = ix->d_bits;
    a.L0 = ix->d_L0;
    a.L12 = ix->d_L12;
    a.wpv = ix->wpv;
    a.l0w = ix->l0w;
    a.l12w = ix->l12w;
    std::memcpy(a.C, ix->C, sizeof(a.C));
    a.pre = ix->d_pre;
    a.p = ix->p;
    a.k = ix->k;
    a.chunk = chunk;
    a.runs = runs_form(ix);
    a.stream = a.runs && stream_form(ix);
    if (a.stream) a.sv = stream_view(ix);
    set_gather_policies(ix, a);
    a.member = a.runs ? d_member_bits : nullptr;
    a.words = words;
    a.row_starts = d_row_starts;
    a.kstart = kstart;
    a.chunk_row = chunk_row;
    a.n_rows = n_rows;
    a.max_pos = (n_words - 1) * 32 - 1;
    a.answers = d_answers;
    a.n_kmers = n_kmers;
    a.counter = counter;  // launch_search clears it on the stream before the kernel
    SBWT_TRY(launch_search(ix, a, s, nullptr));
    if (d_member_bits && !a.runs) SBWT_TRY(launch_member_bits(d_answers, n_kmers, d_member_bits, s));
    return 0;
}
