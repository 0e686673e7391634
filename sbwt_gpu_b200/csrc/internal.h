// internal.h -- the index handle and the host-side launchers shared by the
// CUDA translation units.  Not part of the C ABI.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "sbwt_gpu.h"
#include "common.h"
#include "stream.cuh"

namespace sbwt {

using u64 = uint64_t;
using u32 = uint32_t;

// Device-side parameters of one search launch (passed by value).
struct SearchArgs {
    // LINES layout
    const ulonglong4 *lines;
    u32 lpc;  // lines per vector
    // POPPY layout
    const u64 *bits;  // 4 vectors of wpv words
    const u64 *L0;    // 4 x l0w words
    const u64 *L12;   // 4 x l12w words
    u64 wpv, l0w, l12w;
    // common
    u64 C[5];
    const void *pre;  // presearch table: uint2 (n < 2^32) or ulonglong2 entries; NULL if p == 0
    // with `runs`: the compact presearch table (one u32 an entry, below) or NULL
    const uint32_t *pre32;
    u32 p;
    u32 k;
    const u64 *words;       // packed letters
    const u64 *positions;   // reference contract: letter offset of k-mer j (NULL: read mode)
    const u64 *row_starts;  // read mode: letter offset of each row (n_rows + 1)
    const u64 *kstart;      // read mode: first k-mer index of each row (n_rows + 1)
    const u32 *chunk_row;   // read mode: row of the first k-mer of each chunk
    u64 n_rows;             // read mode: rows (kstart[n_rows] = k-mers in the batch)
    const u64 *runs_dev;    // kernel contract: the run count on the device, or NULL.  The run walk
                            // takes it as n_rows and searches only when the runs are usable
                            // (runs_usable); the per-k-mer kernels search only when they are not
    u64 max_pos;            // largest letter offset whose 64-bit window lies inside `words`
    u64 *answers;
    u64 n_kmers;
    unsigned long long *counter;  // work-stealing cursor (zeroed before launch)
    u32 chunk;                    // k-mers per grab; with `runs`, k-mers per window of chunk_row
    u32 runs;                     // read mode: walk runs right to left with the absent-run skip
    u32 stream;                   // with `runs`: backward steps from a found k-mer (needs sv)
    u32 index64;                  // with `runs`: the walk's 64-bit index form whatever the batch size
    u32 ef_pre, ef_back;          // with `runs`: evict-first gathers from the presearch / backward
                                  // table (each set when that table cannot stay in L2; device.cuh)
    dev::StreamView sv;           // backward table, node nibbles, select samples (stream.cuh)
    uint32_t *member;             // with `runs`: membership bitmap written by the search kernel, or NULL
    // k-mer list mode: k-mer j is kmer_list[j] (MSB-first word)
    const u64 *kmer_list;
    // learned prefilter: skip k-mer j if logits[j] < tau and the Bloom filter rejects it
    const float *logits;
    float tau;
    const uint32_t *bloom_bits;
    u64 bloom_mask;
    u32 bloom_hashes;
    unsigned long long *skipped;
    // run walk of a batch of reads behind the learned prefilter: bit j%32 of
    // word j/32 = k-mer j rejected by the model and the backup Bloom filter
    const uint32_t *reject;
};

struct KernelShape {
    int layout = SBWT_LAYOUT_LINES;
    u32 kpt = 0;   // k-mer slots per thread (0: the queue-fed single-slot kernel)
    u32 tpk = 1;   // lanes per k-mer
    u32 tpb = 128; // threads per block
    u32 sb = 1024;
    int kind = SBWT_POPPY;
    int shuffles = 0;
    int mode = SBWT_SEARCH_STREAM;  // batches of reads with the queue-fed form (sbwt_params.search_mode)
    // knobs of the run walk (batches of reads), set by the autotuner:
    u32 window = 128;        // k-mers per window (line layout: 64, 128 or 256)
    u32 blocks_per_sm = 0;   // resident blocks per SM of the persistent grid (0: as many as fit)
    int evict = 0;           // evict-first gathers: 0 = when a table exceeds half of L2, 1 = never, 2 = always
    int l2_persist = 0;      // the rank lines of the search layout held in the L2 set-aside (l2_window)
    int index64 = 0;         // 64-bit k-mer and letter indices even for batches that fit 32 bits
};

// Device buffers of one in-flight search (grow-only).
struct Workspace {
    uint64_t *words = nullptr;  size_t words_cap = 0;
    uint64_t *kstart = nullptr; size_t kstart_cap = 0;
    uint32_t *chunk_row = nullptr; size_t chunk_cap = 0;
    uint64_t *scan = nullptr;   size_t scan_cap = 0;
    unsigned long long *counter = nullptr; size_t counter_cap = 0;
    // host pipeline only
    uint8_t *letters = nullptr; size_t letters_cap = 0;
    uint64_t *rows = nullptr;   size_t rows_cap = 0;
    uint64_t *answers = nullptr; size_t answers_cap = 0;
    uint64_t *h_rows = nullptr; size_t h_rows_cap = 0;  // pinned host staging
    uint8_t *h_letters = nullptr; size_t h_letters_cap = 0;
    uint64_t *h_answers = nullptr; size_t h_answers_cap = 0;
    uint32_t *member = nullptr; size_t member_cap = 0;    // membership bitmap (both host pipelines)
    uint32_t *h_member = nullptr; size_t h_member_cap = 0;
    // sparse answers of the host pipeline: per group of k-mers the offset of
    // its first found node id, and the found node ids (32 bits) in order
    uint64_t *goff = nullptr;   size_t goff_cap = 0;     // group offsets, then the scan's scratch
    uint32_t *nodes = nullptr;  size_t nodes_cap = 0;
    uint64_t *h_goff = nullptr; size_t h_goff_cap = 0;
    uint32_t *h_nodes = nullptr; size_t h_nodes_cap = 0;
    // CUDA graph of the last pack -> table -> search -> bitmap chain, replayed
    // while every launch parameter (the key) stays the same
    cudaGraphExec_t graph = nullptr;
    uint64_t graph_key[12] = {0};
    void release();
};

}  // namespace sbwt

struct sbwt_index {
    int device = 0;
    int num_sms = 0;
    uint64_t l2_bytes = 0;
    uint64_t n = 0;
    uint32_t k = 30;
    uint64_t C[5] = {0, 0, 0, 0, 0};
    // raw vectors (reference word layout), 4 x wpv words, zero past n
    uint64_t *d_bits = nullptr;
    uint64_t wpv = 0;
    // LINES layout
    ulonglong4 *d_lines = nullptr;
    uint32_t lpc = 0;
    bool lines_ok = false;
    // wide lines (SBWT_LAYOUT_LINES512 / LINES2048): wide_s sectors per line, 0 = not built
    ulonglong4 *d_wide = nullptr;
    uint32_t wide_s = 0, wide_lpc = 0;
    // POPPY layout
    uint64_t *d_L0 = nullptr, *d_L12 = nullptr;
    uint64_t l0w = 0, l12w = 0;
    uint32_t sb = 0;
    int kind = 0;
    bool poppy_ok = false;
    // presearch table
    uint32_t p = 0;
    void *d_pre = nullptr;
    // compact presearch table for the run walk (indexes below 2^27 columns):
    // entry = L | w << 27, w = R - L + 1 (0: empty interval, kPreEscape: look
    // the entry up in d_pre, the interval is wider than the field holds)
    uint32_t *d_pre32 = nullptr;
    bool pre64 = false;
    int compact_pre = -1;  // the compact table: -1 = from SBWT_PRESEARCH_COMPACT, 0 = off, 1 = on
    // backward-step structures (stream.cu): node nibbles, select samples, backward table
    uint8_t *d_node = nullptr;
    uint32_t *d_sel = nullptr;
    uint64_t *d_back = nullptr;  // backward table (stream.cuh, SBWT_BACK_TABLE)
    uint32_t sel_off[4] = {0, 0, 0, 0}, sel_n[4] = {0, 0, 0, 0};
    bool stream_ok = false;
    // device ms of the last build of: lines, poppy, presearch table, backward-step structures
    float build_ms[4] = {0, 0, 0, 0};
    // launch shape
    sbwt::KernelShape shape;
    // scan block sums of the rank builds
    uint64_t *d_scan = nullptr;
    size_t scan_cap = 0;
    // per-call work buffers: ws[0] serves the device-pointer entry points,
    // ws[0 .. kPipeSlots) the streams of the host pipeline
    static constexpr int kPipeSlots = 6;
    sbwt::Workspace ws[kPipeSlots];
    cudaStream_t pipe_stream[kPipeSlots] = {};
    // bytes the last host-pipeline call copied host->device and device->host
    uint64_t pipe_h2d = 0, pipe_d2h = 0;
    // host threads of the host pipelines (0: the OpenMP default)
    int host_threads = 0;
    // bumped whenever a device structure a search reads is rebuilt (graph keys)
    uint64_t gen = 1;
    bool use_graph = false;
    // L2 set-aside for the rank lines (l2_window): bytes this index asked for
    // (0: none), and the device's limits
    size_t l2_setaside = 0;
    size_t l2_max_persist = 0, l2_max_window = 0;
    // per-call profiling (sbwt_profile_enable)
    bool prof_on = false;
    cudaEvent_t prof_ev[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    uint32_t prof_launches = 0, prof_blocks = 0;
    bool prof_member = false;
};

namespace sbwt {

// rank_build.cu
int build_lines(sbwt_index *ix, cudaStream_t s, uint64_t ones[4]);
int build_poppy(sbwt_index *ix, uint32_t sb, int kind, cudaStream_t s);
// The wide-line layout of `sectors` (2 or 8) 32-byte sectors per line.
int build_wide(sbwt_index *ix, uint32_t sectors, cudaStream_t s);
inline uint32_t wide_sectors(int layout) {
    return layout == SBWT_LAYOUT_LINES512 ? 2u : layout == SBWT_LAYOUT_LINES2048 ? 8u : 0u;
}
int ensure_scan_scratch(sbwt_index *ix, uint64_t n_items);

// presearch.cu
int run_presearch(sbwt_index *ix, uint32_t p, cudaStream_t s);
int export_presearch(const sbwt_index *ix, uint64_t *lefts, uint64_t *rights, uint64_t count);

// ingest.cu
int launch_pack(const uint8_t *d_letters, uint64_t n_letters, uint64_t *d_words, cudaStream_t s);
int launch_kstart(const uint64_t *d_row_starts, uint64_t n_rows, uint32_t k, uint64_t *d_kstart, uint64_t *d_scan,
                  cudaStream_t s);
uint64_t scan_scratch_words(uint64_t n_items);
int launch_chunk_rows(const uint64_t *d_kstart, uint64_t n_rows, uint64_t n_kmers, uint32_t chunk,
                      uint32_t *d_chunk_row, cudaStream_t s);
int launch_member_bits(const uint64_t *d_answers, uint64_t n, uint32_t *d_bits, cudaStream_t s);
// The k-mers j0 .. j0+count-1 of the batch of reads described by a (words,
// row_starts, kstart, chunk_row, chunk, max_pos) as a list of 64-bit windows.
int launch_kmer_list(const SearchArgs &a, uint64_t j0, uint64_t count, uint64_t *d_out, cudaStream_t s);

// stream.cu
int build_stream(sbwt_index *ix, cudaStream_t s);
dev::StreamView stream_view(const sbwt_index *ix);

// packed_runs.cu
// The kernel contract's runs are walked when they average at least
// kMinRunKmers k-mers (fewer: random positions, searched one by one).
constexpr u64 kMinRunKmers = 4;
__host__ __device__ inline bool runs_usable(u64 runs, u64 n_kmers) { return runs != 0 && runs * kMinRunKmers <= n_kmers; }
int packed_runs(Workspace &w, const u64 *positions, u64 n_kmers, u32 chunk, cudaStream_t s, const u64 **runs_dev);

// api.cu
// Launch arguments of a search with the index's current shape and mode (the
// batch pointers left NULL); `rows`: a batch of reads.
SearchArgs base_args(const sbwt_index *ix, bool rows);
// Grows w for a batch of reads and enqueues pack -> per-row k-mer table ->
// chunk table on s; fills the batch fields of a (a.chunk set by base_args).
int prepare_rows(sbwt_index *ix, Workspace &w, SearchArgs &a, const uint8_t *d_letters, uint64_t n_letters,
                 const uint64_t *d_rows, uint64_t n_rows, uint64_t n_kmers, cudaStream_t s);
int search_rows_device(sbwt_index *ix, Workspace &w, const uint8_t *d_letters, u64 n_letters, const u64 *d_rows,
                       u64 n_rows, u64 *d_answers, uint32_t *d_member, u64 n_kmers, cudaStream_t s);
template <class T> int grow(T *&p, size_t &cap, size_t need);
template <class T> int grow_host(T *&p, size_t &cap, size_t need);

// api.cu: the L2 access-policy window of a search launch over the index's
// current layout (false: none applies); l2_setaside_acquire/release size the
// device's persisting set-aside for the indexes that use it.
bool l2_window(const sbwt_index *ix, cudaAccessPolicyWindow *w);
int l2_setaside_acquire(sbwt_index *ix);
void l2_setaside_release(sbwt_index *ix);

// search.cu
int launch_search(const sbwt_index *ix, SearchArgs &a, cudaStream_t s, uint32_t *launched_blocks);
// Evict-first policies for the run walk's gathers: a table gets one when it
// is larger than half of the device's L2 (it cannot stay there next to the
// lines).
void set_gather_policies(const sbwt_index *ix, SearchArgs &a);
// Whether a batch of reads searched with the index's current shape and mode
// runs the run-walking kernel (absent-run skip), and whether it also takes
// backward steps.
bool runs_form(const sbwt_index *ix);
bool stream_form(const sbwt_index *ix);
// Work granularity of a launch: k-mers per grab, or for the run-walking form
// k-mers per window of the row table.  `rows`: a batch of reads.
u32 search_chunk(const sbwt_index *ix, bool rows);
bool search_shape_supported(const KernelShape &sh, bool wide);

}  // namespace sbwt
