/*
 * sbwt_gpu.h -- C ABI of the B200 (sm_100a) SBWT k-mer search engine.
 *
 * The engine is a drop-in for the search path of epicharri/sbwt_gpu
 * (plain-matrix SBWT index -> poppy rank structures -> presearch table ->
 * query ingest -> per-k-mer search -> answers).  Each entry point below names
 * the reference interface it replaces (paths relative to the reference root).
 *
 * Conventions, as in the reference (include/gpu/cuda.hpp:7-13):
 *   - every `int` entry point returns 0 on success and non-zero on error;
 *     sbwt_last_error() gives the message of the last failure on this thread;
 *   - answers are u64: the colex rank of the k-mer's SBWT node, or
 *     0xFFFFFFFFFFFFFFFF (printed as -1) when the k-mer is absent
 *     (include/gpu/search_kernel.hpp:98-103);
 *   - the caller owns the buffers it passes; an sbwt_index owns the index,
 *     its rank layouts and its presearch table;
 *   - calls that take a `stream` are ordered on that cudaStream_t (passed as
 *     void*, NULL = the legacy default stream); one index may be used by one
 *     host thread at a time.
 * There is no CPU fallback: without a usable CUDA device every compute entry
 * point fails with an error.
 */
#ifndef SBWT_GPU_H
#define SBWT_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SBWT_GPU_ABI_VERSION 2

/* Rank-structure kinds of the reference (include/enums.hpp:9-11). */
#define SBWT_POPPY 1
#define SBWT_CUM_POPPY 2

/* Search layouts of this engine. */
#define SBWT_LAYOUT_LINES 0 /* 32-byte lines: 32-bit rank word + 224 bits (default) */
#define SBWT_LAYOUT_POPPY 1 /* the reference's L0/L12 poppy layout (bits_in_superblock, rank_structure) */
/* Wider interleave blocks: 512-bit (64-byte) and 2048-bit (256-byte) lines, each a
 * 32-bit rank word plus 16-bit counts per 32-byte sector and the block's bits, so a
 * rank reads the line's first sector and the one holding its bit (batches of reads
 * with the queue-fed kernels: kmers_per_thread 0, threads_per_kmer 1).  The
 * reference's block-size axis is its superblock size (include/parameters.hpp:13-37,
 * include/epicseq/search_caller.hpp:81-209). */
#define SBWT_LAYOUT_LINES512 2
#define SBWT_LAYOUT_LINES2048 3

typedef struct sbwt_index sbwt_index;

/* Run parameters.  Replaces epic::Parameters (include/parameters.hpp:39-63);
 * field names follow its members, defaults follow its initialisers. */
typedef struct {
    uint32_t k;                  /* k-mer length, 3..32 (parameters.hpp:49, default 30) */
    uint32_t k_presearch;        /* presearch depth p, 0 = without presearch (parameters.hpp:50) */
    uint32_t bits_in_superblock; /* 256|512|1024|2048|4096 (parameters.hpp:42) */
    int32_t rank_structure;      /* SBWT_POPPY | SBWT_CUM_POPPY (parameters.hpp:47) */
    int32_t with_shuffles;       /* cooperative rank for the poppy layout (parameters.hpp:45) */
    uint32_t threads_per_block;  /* 0 = engine default (parameters.hpp:51) */
    int32_t device;              /* CUDA device ordinal (the reference uses 0, parameters.hpp:81) */
    int32_t layout;              /* SBWT_LAYOUT_LINES | _POPPY | _LINES512 | _LINES2048 */
    uint32_t kmers_per_thread;   /* search kernel: 0 = one k-mer per lane fed from a per-warp queue
                                    (default); 1,2,3,4,6,8 = k-mer slots held in registers */
    uint32_t threads_per_kmer;   /* search kernel: lanes sharing one k-mer, 1|2|4 (0 = default) */
    int32_t search_mode;         /* searches of reads with the queue-fed kernel (SBWT_SEARCH_*, default
                                    SBWT_SEARCH_STREAM).  The answers are the same in every mode.
                                    No reference counterpart. */
} sbwt_params;

/* Search modes for batches of reads (sbwt_params.search_mode, sbwt_set_search_mode).
 * EVERY_KMER: every k-mer is searched from scratch, as the reference does.
 * SKIP_ABSENT: each read is walked from right to left; when a k-mer's search
 *   fails after m letters, those m letters are in no indexed k-mer, so the
 *   k-m+1 k-mers containing them are answered absent without a search.
 * STREAM: SKIP_ABSENT, and after a k-mer is found the k-mer one letter to its
 *   left is reached by one backward step (one load from a per-column table
 *   of predecessor groups) instead of a new search.  Needs the line layout's
 *   index size limit and about 8.6 bytes per column, built on the GPU when
 *   the mode is selected. */
#define SBWT_SEARCH_EVERY_KMER 0
#define SBWT_SEARCH_SKIP_ABSENT 1
#define SBWT_SEARCH_STREAM 2

/* Fills the defaults (k=30, p=12, SB=1024, poppy, no shuffles, device 0,
 * line layout).  No reference counterpart (the reference uses member
 * initialisers, parameters.hpp:41-56). */
int sbwt_params_default(sbwt_params *params);

/* Message of the last failed call on this thread ("" if none). */
const char *sbwt_last_error(void);

/* ------------------------------------------------------------------ index */

/* Loads the four A/C/G/T bit-vector files (u64 little-endian bit count, then
 * ceil(n/8) bytes, position p at byte 8+p/8, bit 7-p%8), builds the rank
 * structures on the GPU, the C array, and the presearch table for
 * params->k_presearch.  Replaces epic::MatrixSBWT::create
 * (include/matrix_sbwt.hpp:32-200) with BitVector::create/read
 * (include/bit_vector.hpp:65-138) and RankDataStructures
 * (include/rank_data_structures.hpp:59-198). */
int sbwt_index_load(const char *file_a, const char *file_c, const char *file_g, const char *file_t,
                    const sbwt_params *params, sbwt_index **out);

/* Same from host memory: bits[c] holds n_bits bits of vector c in the
 * reference's in-memory word layout (position p at bit 63-p%64 of word p/64,
 * i.e. after the byte swap of rank_data_structures.hpp:98).  Used by the
 * builder and the tests.  No file-level counterpart in the reference. */
int sbwt_index_from_host(const uint64_t *const bits[4], uint64_t n_bits, const sbwt_params *params,
                         sbwt_index **out);

void sbwt_index_free(sbwt_index *index);

/* Number of SBWT columns n and the C array (counts_before,
 * matrix_sbwt.hpp:150-157). */
int sbwt_index_info(const sbwt_index *index, uint64_t *n_bits, uint64_t C[5], uint32_t *k, uint32_t *k_presearch);

/* (Re)builds the presearch table for depth p (0 frees it: search without
 * presearch).  Replaces epic::PreSearch::call_presearch
 * (include/presearch.hpp:32-130) and the presearch kernel
 * (include/gpu/presearch_kernel.hpp:19-37). */
int sbwt_presearch(sbwt_index *index, uint32_t p);

/* Device time in ms of the index's last build phases: ms[0] the line layout
 * (rank words), ms[1] the poppy L0/L12 structures (0 if not built), ms[2]
 * the presearch table (its last build), ms[3] the backward-step structures.
 * The reference prints its presearch time (include/matrix_sbwt.hpp:188) and
 * builds its rank structures on the CPU (rank_data_structures.hpp:142-198). */
int sbwt_build_times(const sbwt_index *index, float ms[4]);

/* Copies the presearch table to the host in the reference's format: two
 * arrays node_lefts[4^p], node_rights[4^p] (include/gpu/device_memory.hpp:
 * 136-138). */
int sbwt_presearch_export(const sbwt_index *index, uint64_t *node_lefts, uint64_t *node_rights, uint64_t count);

/* Rebuilds the poppy rank structures on the GPU for (bits_in_superblock,
 * rank_structure) and copies L0 and L12 of vector c (0..3) to the host:
 * sizes are 1 + (n >> (SB==4096 ? 31 : 32)) and 1 + ceil(n/SB) words.
 * Replaces RankDataStructures::construct (rank_data_structures.hpp:142-198). */
int sbwt_rank_export(sbwt_index *index, uint32_t bits_in_superblock, int32_t rank_structure, int c,
                     uint64_t *L0, uint64_t l0_words, uint64_t *L12, uint64_t l12_words);

/* Pass for an unsigned sbwt_configure argument to leave it unchanged. */
#define SBWT_KEEP 0xFFFFFFFFu

/* Selects the search layout / kernel shape for later searches (building the
 * poppy structures if needed); kmers_per_thread, threads_per_kmer and
 * threads_per_block take SBWT_KEEP or 0 ... as sbwt_params documents.  No reference counterpart: the reference
 * picks these by template switch (include/epicseq/search_caller.hpp:81-209). */
int sbwt_configure(sbwt_index *index, int32_t layout, uint32_t bits_in_superblock, int32_t rank_structure,
                   int32_t with_shuffles, uint32_t kmers_per_thread, uint32_t threads_per_kmer,
                   uint32_t threads_per_block);

/* Knobs of the run walk (searches of reads), each SBWT_KEEP to leave it:
 * window = k-mers per window of the work split (64, 128, 256; line layout),
 * blocks_per_sm = resident blocks per SM of the persistent grid (0: as many
 * as fit), evict = the L2 policy of the presearch and backward-table gathers
 * (0: evict-first when the table exceeds half of L2, 1: never, 2: always),
 * l2_persist = hold the rank lines in the persisting L2 set-aside (1) or not
 * (0).  The autotuner sets them; the answers do not depend on them.  No
 * reference counterpart. */
int sbwt_set_walk_options(sbwt_index *index, uint32_t window, uint32_t blocks_per_sm, int32_t evict,
                          int32_t l2_persist);

/* Selects the search mode (SBWT_SEARCH_*) for later searches of reads on this
 * index, building the backward-step structures on first use of
 * SBWT_SEARCH_STREAM.  No reference counterpart: the reference searches every
 * k-mer (include/gpu/search_kernel.hpp:61-104). */
int sbwt_set_search_mode(sbwt_index *index, int32_t mode);

/* Copies the per-column node bytes of the backward step to the host (count =
 * number of columns): bits 0-2 the first letter of the node's label (0 = $,
 * 1..4 = A, C, G, T), bit 3 set on the first node of each group of nodes
 * sharing their last k-1 letters.  For tests; no reference counterpart. */
int sbwt_node_bytes_export(sbwt_index *index, uint8_t *out, uint64_t count);

/* Sets the L2 fetch granularity (32, 64 or 128 bytes; cudaLimitMaxL2FetchGranularity)
 * of the index's device for this process, as the reference does before its
 * presearch and search kernels (include/presearch.hpp:34-37,
 * include/epicseq/search_caller.hpp:91-96, flags --device-set-limit-presearch
 * and --device-set-limit-search). */
int sbwt_set_l2_fetch_granularity(sbwt_index *index, uint32_t bytes);

/* Turns CUDA-graph replay of sbwt_search_reads on or off (default off).
 * When on, a call on a non-default stream captures its whole kernel chain
 * (pack -> per-row table -> search -> bitmap) into a CUDA graph, and a later
 * call with the same buffers, sizes and launch shape replays that graph with
 * one launch.  No reference counterpart (the reference launches each kernel
 * separately, include/epicseq/kmer_search.hpp:97-160). */
int sbwt_use_graphs(sbwt_index *index, int on);

/* ----------------------------------------------------------------- search */

/* The reference kernel contract: d_kmer_string holds the packed letters
 * (n_words u64, 32 letters per word, letter j of a word at bits 63-2j..62-2j,
 * with at least one word of padding after the last letter);
 * d_positions_in_results_out[j] holds the letter offset of k-mer j on entry
 * and its answer on return (in place).  All pointers are device pointers.
 * Replaces epic::gpu::launch_search_kernel / search
 * (include/gpu/search_and_presearch_launchers.hpp:21-60,
 *  include/gpu/search_kernel.hpp:61-104).  Unlike the reference, no thread
 * runs past n_kmers.  In the run-walking search modes, k-mers at consecutive
 * positions (each position one more than the one before, as the reference's
 * positions of one read are) are walked as runs, as sbwt_search_reads does;
 * positions with runs shorter than four k-mers on average are searched one
 * k-mer at a time.  The choice is made on the device, so the call is
 * stream-ordered with no host wait; the handle's run table is sized for a
 * quarter of the k-mers (4 bytes per k-mer of device memory). */
int sbwt_search_packed(sbwt_index *index, const uint64_t *d_kmer_string, uint64_t n_words,
                       uint64_t *d_positions_in_results_out, uint64_t n_kmers, void *stream);

/* 2-bit packs n_letters ASCII letters (device) into d_words (device,
 * ceil((n_letters+32)/32) words; letters past n_letters are packed as A).
 * Mapping A/a->0 C/c->1 G/g->2 T/t->3, every other byte -> 0.  Replaces
 * create_kmer_string (include/gpu/create_kmer_string.hpp:22-42). */
int sbwt_pack(const uint8_t *d_letters, uint64_t n_letters, uint64_t *d_words, void *stream);

/* Searches every k-mer of a batch of reads held on the device:
 * d_letters = concatenated reads (n_letters bytes), d_row_starts[r] = offset
 * of read r (n_rows + 1 entries, last = n_letters).  K-mers never cross a
 * read boundary; a read shorter than k has no k-mers.  Writes one answer per
 * k-mer, reads in order, to d_answers (device, n_kmers entries, n_kmers =
 * sum of max(0, len-k+1)).  d_member_bits (optional, device, ceil(n_kmers/
 * 32) u32 words) receives bit j%32 of word j/32 = (answer j != -1).
 * d_answers may be NULL when d_member_bits is given (membership only).
 * Replaces the chain KmerSearch::parse_kmer_string_in_gpu ->
 * create_positions_in_gpu -> call_search (include/epicseq/kmer_search.hpp:
 * 97-185) with one pack kernel and one persistent work-stealing search
 * kernel; no per-k-mer positions array is materialised. */
int sbwt_search_reads(sbwt_index *index, const uint8_t *d_letters, uint64_t n_letters, const uint64_t *d_row_starts,
                      uint64_t n_rows, uint64_t *d_answers, uint32_t *d_member_bits, uint64_t n_kmers, void *stream);

/* sbwt_search_reads for callers that cannot call cudaMalloc while they
 * search: a process whose device memory another allocator already holds (a
 * framework's caching allocator that reserved the GPU), or an application
 * that accounts for every device allocation itself.  No counterpart in the
 * reference.  Same arguments and answers as sbwt_search_reads (d_answers may
 * be NULL when d_member_bits is given), but all scratch (packed letters,
 * per-row k-mer table, chunk table, scan sums, work counter, and the answers
 * of a membership-only search with the per-k-mer kernels) lives in one fixed
 * 32 MiB device array of the library (held by every GPU that loads it until
 * exit), so no cudaMalloc/cudaFree is made.  A batch needing more is rejected
 * with an error giving the bytes it needs: about 100M letters of 150-letter
 * reads fit, fewer when the rows are shorter.  The first call on a device looks
 * the array up (cudaGetSymbolAddress): make it before any stream capture.
 * Calls share the array: calls that overlap on the GPU race. */
int sbwt_search_reads_noalloc(sbwt_index *index, const uint8_t *d_letters, uint64_t n_letters,
                              const uint64_t *d_row_starts, uint64_t n_rows, uint64_t *d_answers,
                              uint32_t *d_member_bits, uint64_t n_kmers, void *stream);

/* Host-memory form of sbwt_search_reads: letters, row starts and answers
 * are host buffers (pinned or pageable).  The batch is streamed through the
 * GPU in chunks with copies overlapped with compute.  While the index has
 * fewer than 2^32 columns and six or more OpenMP threads are available, the
 * answers cross PCIe as a membership bitmap plus the 32-bit node ids of the
 * found k-mers, and the host threads write the u64 answers; with fewer
 * threads a share of the chunks (sbwt_pipeline_dense_share) comes back as
 * u64 answers by DMA into a pinned answer buffer instead; environment:
 * SBWT_PIPELINE_TRANSFER=dense|sparse|hybrid forces one form,
 * SBWT_PIPELINE_DENSE_SHARE=f sets the share of dense chunks,
 * SBWT_PIPELINE_CHUNK_LETTERS sets the chunk size (default 64M letters).
 * Replaces the
 * parse/position/search/copy-back chain of KmerSearch::search
 * (kmer_search.hpp:97-160) and ResultsPersister's device-to-host copy
 * (results_persister.hpp:58-65). */
int sbwt_search_reads_host(sbwt_index *index, const uint8_t *letters, uint64_t n_letters, const uint64_t *row_starts,
                           uint64_t n_rows, uint64_t *answers, uint64_t n_kmers);

/* A batch in host memory searched on several index replicas, one per GPU
 * (each loaded with its own sbwt_params.device; replicas may also share a
 * device): the rows are cut into contiguous ranges of near-equal k-mer
 * counts (sbwt_partition_rows; a row is never split), each replica runs
 * sbwt_search_reads_host on its range from a host thread of its own and
 * writes its disjoint slice of `answers`.  No data moves between the GPUs.
 * The OpenMP threads of the call are shared among the replicas unless
 * sbwt_set_host_threads set them.  The reference pins device 0
 * (include/parameters.hpp:81). */
int sbwt_search_reads_host_multi(sbwt_index *const *indexes, int n_indexes, const uint8_t *letters,
                                 uint64_t n_letters, const uint64_t *row_starts, uint64_t n_rows, uint64_t *answers,
                                 uint64_t n_kmers);
/* bounds[0..n_parts]: row ranges [bounds[i], bounds[i+1]) of near-equal
 * k-mer counts (each boundary the row boundary nearest to i/n_parts of the
 * k-mers); needs no GPU. */
int sbwt_partition_rows(const uint64_t *row_starts, uint64_t n_rows, uint32_t k, int n_parts, uint64_t *bounds);

/* Host threads the host pipelines use (expansion of the sparse answers,
 * row tables); 0 = the OpenMP default (OMP_NUM_THREADS).  No reference
 * counterpart (its host side is one thread). */
int sbwt_set_host_threads(sbwt_index *index, int threads);
/* Share of the chunks of a sbwt_search_reads_host call whose u64 answers
 * cross PCIe as such (the rest come back as bitmap + found node ids and are
 * expanded by the host threads), for an index of n_columns searched with
 * host_threads threads (0: the OpenMP default): 0 with six or more threads,
 * below that the measured best share (0.7 for 1-2 threads, 0.5 for 3, 0.3
 * for 4, 0.15 for 5), 1 for indexes of 2^32 columns or more; the
 * SBWT_PIPELINE_TRANSFER and SBWT_PIPELINE_DENSE_SHARE overrides included.
 * Needs no GPU.  No reference counterpart. */
double sbwt_pipeline_dense_share(uint64_t n_columns, int host_threads);

/* Bytes the last sbwt_search_reads_host or sbwt_search_reads_host_member
 * call on this index copied host->device (letters, row tables) and
 * device->host (answers in the form that crossed PCIe).  No reference
 * counterpart. */
int sbwt_pipeline_bytes(const sbwt_index *index, uint64_t *h2d, uint64_t *d2h);

/* Membership only: as sbwt_search_reads_host, but the result is the bitmap
 * member_bits (host, ceil(n_kmers/32) u32 words; bit j%32 of word j/32 =
 * k-mer j is indexed) and no answer array crosses the bus (1 bit instead of
 * 8 bytes per k-mer).  With the run-walking search modes the kernel writes
 * only the bitmap.  No reference counterpart (the reference always returns
 * the colex ranks, results_persister.hpp:58-65). */
int sbwt_search_reads_host_member(sbwt_index *index, const uint8_t *letters, uint64_t n_letters,
                                  const uint64_t *row_starts, uint64_t n_rows, uint32_t *member_bits,
                                  uint64_t n_kmers);

/* Kernel timing of the last sbwt_search_reads call on this index, from CUDA
 * events recorded on that call's stream around each phase (enabled with
 * sbwt_profile_enable; reading synchronizes on the last event).  The
 * reference times its kernels the same way (include/gpu/device_stream.hpp:
 * 52-86, search_and_presearch_launchers.hpp:41,53-54). */
typedef struct {
    float pack_ms;      /* 2-bit packing */
    float table_ms;     /* per-row k-mer table (scan) and chunk table */
    float search_ms;    /* the search kernel */
    float member_ms;    /* membership bitmap (0 if not requested) */
    uint32_t launches;  /* kernels launched by the call */
    uint32_t search_blocks; /* grid of the persistent search kernel */
} sbwt_profile;

int sbwt_profile_enable(sbwt_index *index, int on);
int sbwt_profile_read(sbwt_index *index, sbwt_profile *out);

/* Number of k-mers in a batch of rows (sum of max(0, len-k+1)). */
uint64_t sbwt_count_kmers(const uint64_t *row_starts, uint64_t n_rows, uint32_t k);

/* Autotuner (no reference counterpart; the reference takes its kernel
 * variant from flags, include/parameters.hpp:79-297).  Times
 * sbwt_search_reads on the given device sample: (1) the search layout --
 * 32-byte lines and the 512/2048-bit wide lines, with SBWT_TUNE_POPPY also
 * the poppy layouts SB 512/1024/2048, with SBWT_TUNE_SHAPES also the
 * per-k-mer kernel's shapes (k-mers per thread {1,2,3,4,6,8} x threads per
 * k-mer {1,2,4} x threads per block {128,256}); (2) the run walk's knobs on
 * the best layout (window 64/128/256 k-mers, resident blocks per SM, the
 * evict-first policy of the table gathers, compact presearch entries); (3)
 * with SBWT_TUNE_P the presearch depth {8,10,12,14,15} <= k.  Checks that
 * every candidate's answers have the same checksum, and leaves the fastest
 * configured on the index.  d_answers: device scratch of n_kmers u64.
 * report (optional): JSON of the choice, the time of the configuration
 * before tuning and every candidate (fails if report_cap is too small). */
#define SBWT_TUNE_P 2u
#define SBWT_TUNE_POPPY 4u
#define SBWT_TUNE_SHAPES 8u
int sbwt_autotune(sbwt_index *index, const uint8_t *d_letters, uint64_t n_letters, const uint64_t *d_row_starts,
                  uint64_t n_rows, uint64_t n_kmers, uint64_t *d_answers, uint32_t flags, char *report,
                  uint64_t report_cap);

/* ------------------------------------------------------ learned prefilter */

/* A small BF16 MLP (one-hot k-mer, 4k <= 128 inputs -> 256 ReLU -> 256 ReLU
 * -> 1 logit, FP32 accumulation on the tensor cores) in a learned-Bloom
 * sandwich in front of the exact search.  No reference counterpart.  A
 * k-mer whose logit is below tau is checked against a Bloom filter over
 * every indexed k-mer the model rejects; only a k-mer that both reject is
 * answered "absent" without a search.  No indexed k-mer is ever reported
 * absent, so answers equal the plain search's bit for bit. */
typedef struct sbwt_prefilter sbwt_prefilter;

typedef struct {
    uint32_t steps;       /* Adam steps (20000) */
    uint32_t batch;       /* batch size, a multiple of 256 (8192) */
    float lr;             /* Adam learning rate (1e-3) */
    uint64_t n_positive;  /* expected positives: k-mers of random index nodes, with replacement (5e7) */
    uint64_t n_negative;  /* expected negatives: half uniform random, half positives with 1-3 substitutions (5e7) */
    uint64_t seed;
    float tau;            /* logit threshold (0) */
    float bloom_fpr;      /* false-positive rate of the backup filter (0.01) */
    uint32_t bloom_hashes; /* (3) */
} sbwt_mlp_params;

typedef struct {
    float first_loss, final_loss;   /* mean BCE of the first and the last step */
    float train_ms, total_ms;       /* training loop; whole call */
    uint64_t n_train;               /* labelled candidates (labels from the exact search) */
    double label_positive_fraction; /* share of candidates the index holds */
    double train_accuracy;          /* on the first 4M candidates at tau */
    uint64_t n_indexed_kmers;       /* k-mers of the index (its non-dummy nodes) */
    uint64_t n_rejected_indexed;    /* of those, logit < tau: all inserted into the Bloom filter */
    uint64_t bloom_bits;
} sbwt_prefilter_stats;

int sbwt_mlp_params_default(sbwt_mlp_params *params);
/* Samples and labels the training set on the GPU, trains the MLP, builds the
 * Bloom filter (k must be the index's; the index needs the line layout). */
int sbwt_prefilter_train(sbwt_index *index, const sbwt_mlp_params *params, sbwt_prefilter **out);
int sbwt_prefilter_stats_get(const sbwt_prefilter *pf, sbwt_prefilter_stats *out);
/* The 99073 FP32 parameters: W1[256][128], b1[256], W2[256][256], b2[256], w3[256], b3. */
int sbwt_prefilter_params(const sbwt_prefilter *pf, float *theta, uint64_t count);
void sbwt_prefilter_free(sbwt_prefilter *pf);
/* Logits of n k-mers (device u64 words, first letter in bits 63..62). */
int sbwt_prefilter_logits(sbwt_prefilter *pf, const uint64_t *d_kmers, uint64_t n, float *d_logits, void *stream);

/* Exact answers of a list of k-mers given as MSB-first u64 words (device). */
int sbwt_search_kmers(sbwt_index *index, const uint64_t *d_kmers, uint64_t n, uint64_t *d_answers, void *stream);
/* The same behind the prefilter; *n_skipped (optional, synchronizes) = k-mers
 * answered without a search. */
int sbwt_search_kmers_filtered(sbwt_index *index, sbwt_prefilter *pf, const uint64_t *d_kmers, uint64_t n,
                               uint64_t *d_answers, uint64_t *n_skipped, void *stream);

/* sbwt_search_reads behind the learned prefilter (the learned-Bloom
 * sandwich): the model classifies every k-mer of the batch (its logit
 * against tau) and the backup Bloom filter, built over every indexed k-mer
 * the model rejects, is probed for the rejected ones; a k-mer rejected by
 * both is answered absent (~0) without a search, every other k-mer is
 * searched exactly, so no indexed k-mer is ever reported absent and the
 * answers equal sbwt_search_reads'.  Same arguments as sbwt_search_reads
 * plus the prefilter (trained on this index, same k); *n_skipped (optional,
 * synchronizes) = k-mers answered from the prefilter alone.  Needs the run
 * walk on the line layout (search mode stream or skip).  Scratch: 8 bytes per
 * k-mer of a 64M-k-mer inference chunk and one bit per k-mer, grown on the
 * prefilter handle.  In front of the reference's search kernel
 * (include/gpu/search_kernel.hpp:61-104, fed by include/epicseq/
 * kmer_search.hpp:97-153), which has no prefilter. */
int sbwt_search_reads_filtered(sbwt_index *index, sbwt_prefilter *pf, const uint8_t *d_letters, uint64_t n_letters,
                               const uint64_t *d_row_starts, uint64_t n_rows, uint64_t *d_answers,
                               uint32_t *d_member_bits, uint64_t n_kmers, uint64_t *n_skipped, void *stream);

/* Test hooks of the training kernels: loss and gradient of one BCE step for
 * the given parameters and batch (n a multiple of 256), and the logits of
 * the fused inference kernel, all on device 0. */
int sbwt_mlp_gradients(uint32_t k, const float *theta, const uint64_t *kmers, const uint8_t *labels, uint32_t n,
                       float *loss, float *grad);
int sbwt_mlp_logits(uint32_t k, const float *theta, const uint64_t *kmers, uint64_t n, float *logits);

/* ------------------------------------------------------------ query files */

/* Reads a FASTA query file the way KmerSearch::read_file does
 * (include/epicseq/kmer_search.hpp:319-342): every line that does not start
 * with '>' is one read; letters are concatenated.  Divergence: a last line
 * without '\n' keeps its last letter.  A file whose first byte is '@' is read
 * as FASTQ (four-line records; the sequence line is the read; no reference
 * counterpart).  The returned buffers are owned by the library (free with
 * sbwt_queries_free). */
typedef struct {
    uint8_t *letters;     /* n_letters bytes (+32 zero bytes of padding) */
    uint64_t n_letters;
    uint64_t *row_starts; /* n_rows + 1 entries */
    uint64_t n_rows;
    uint64_t n_kmers;     /* for the k given to sbwt_queries_read */
} sbwt_queries;

int sbwt_queries_read(const char *path, uint32_t k, sbwt_queries *out);

/* Reads n_files query files (in parallel) into one batch: rows of file f are
 * rows [file_rows[f], file_rows[f+1]) of *out (file_rows: n_files + 1
 * entries).  One batch means one persistent search launch over all files.
 * No reference counterpart (the reference takes one query file,
 * include/parameters.hpp:29). */
int sbwt_queries_read_many(const char *const *paths, int n_files, uint32_t k, sbwt_queries *out, uint64_t *file_rows);
void sbwt_queries_free(sbwt_queries *q);

/* Streaming reader of one query file (FASTA as sbwt_queries_read, or FASTQ):
 * sbwt_reader_next returns the next batch of whole reads, at most max_letters
 * letters unless a single read is longer (0: the rest of the file); a batch
 * with n_rows = 0 marks the end.  The file is read in 16 MiB blocks, so a
 * caller can search one batch while the next is read.  Replaces the
 * whole-file getline loop of KmerSearch::read_file (include/epicseq/
 * kmer_search.hpp:319-342).  Batches are freed with sbwt_queries_free. */
typedef struct sbwt_reader sbwt_reader;
int sbwt_reader_open(const char *path, uint32_t k, sbwt_reader **out);
int sbwt_reader_next(sbwt_reader *reader, uint64_t max_letters, sbwt_queries *out);
void sbwt_reader_close(sbwt_reader *reader);

/* Formats answers as the reference prints them (results_persister.hpp:82-95):
 * per read, each answer as a signed int64 followed by one space, then '\n'
 * (a read shorter than k gives an empty line).  Writes to `out` (size cap);
 * returns the number of bytes, or -1 if cap is too small (call with
 * out == NULL for the exact size). */
int64_t sbwt_format_answers(const uint64_t *row_starts, uint64_t n_rows, uint32_t k, const uint64_t *answers,
                            char *out, uint64_t cap);

/* The same text formatted on the GPU from device buffers: row_starts (n_rows
 * + 1 letter offsets, as sbwt_search_reads takes them) and n_kmers answers.
 * *bytes receives the text's length; with d_out == NULL nothing is written
 * (size query), otherwise cap must be at least *bytes.  Synchronises
 * `stream`.  Replaces the host loop of results_persister.hpp:82-95. */
int sbwt_format_answers_device(const uint64_t *d_row_starts, uint64_t n_rows, uint32_t k, const uint64_t *d_answers,
                               uint64_t n_kmers, char *d_out, uint64_t cap, uint64_t *bytes, void *stream);

/* -------------------------------------------------------------- builder */

/* Builds the plain-matrix SBWT of every k-mer of the given sequences
 * (forward strand; k-mers holding a byte other than ACGTacgt are skipped),
 * with dummy nodes for source k-mers, in the reference's matrix format.
 * seqs = concatenated sequences, seq_starts = n_seqs + 1 offsets.
 * Outputs: *n_bits = number of columns (nodes), bits[c] (library-owned,
 * ceil(n/64) words each, reference in-memory layout), free with
 * sbwt_build_free.  The reference relies on an external tool for this step;
 * this builder is this project's own. */
typedef struct {
    uint64_t n_bits;
    uint64_t n_kmers;   /* distinct k-mers */
    uint64_t n_dummies; /* dummy nodes including the root */
    uint64_t *bits[4];
    uint64_t n_words;
} sbwt_built;

int sbwt_build(const uint8_t *seqs, const uint64_t *seq_starts, uint64_t n_seqs, uint32_t k, sbwt_built *out);
void sbwt_build_free(sbwt_built *b);

/* The same construction on GPU `device` (k-mer enumeration, radix sort, dummy
 * nodes, bit-vector emit as kernels); its output equals sbwt_build's bit for
 * bit and is released with sbwt_build_free.  No reference counterpart (the
 * reference relies on an external construction tool, include/matrix_sbwt.hpp:
 * 44-55). */
int sbwt_build_gpu(const uint8_t *seqs, const uint64_t *seq_starts, uint64_t n_seqs, uint32_t k, int32_t device,
                   sbwt_built *out);

/* Writes vector c of a built index to `path` in the reference file format
 * (include/bit_vector.hpp:65-128). */
int sbwt_write_bitvector(const char *path, const uint64_t *bits, uint64_t n_bits);

#ifdef __cplusplus
}
#endif

#endif /* SBWT_GPU_H */
