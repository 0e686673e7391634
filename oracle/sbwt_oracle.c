/*
 * sbwt_oracle.c -- CPU restatement of the epicharri/sbwt_gpu search path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product (sbwt_gpu_b200/) links,
 * loads or calls this file.  It is the checker that the tests, smoke() and the
 * CPU-baseline leg of bench.py compare the CUDA path against.
 *
 * Every function restates one piece of the reference and cites the reference
 * file:line it follows (paths relative to the reference project root).  The
 * reference has no CPU search; the device functions (rank, presearch, search)
 * are restated here with PTX semantics made explicit: `x >> s` for s >= 64
 * yields 0 (PTX shr clamps the shift amount), which x86 does not do.
 *
 * Pinning: the rank build (orc_rank_build) is compared word for word with the
 * reference's own RankDataStructures compiled from its sources (oracle/_ref,
 * see oracle/Makefile); the full search output is compared with fixtures
 * produced by running the reference program itself (tests/golden/).
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef uint64_t u64;
typedef uint32_t u32;
typedef uint8_t u8;

/* PTX-style shift: shift amounts >= 64 give 0 (rank_kernel.hpp:184,218,226-229
 * rely on this; see the PTX ISA description of shr). */
static inline u64 shr64(u64 x, u32 s) { return s >= 64u ? 0ull : (x >> s); }
static inline u32 shr32(u32 x, u32 s) { return s >= 32u ? 0u : (x >> s); }
static inline u32 popc64(u64 x) { return (u32)__builtin_popcountll(x); }

/* bit_vector.hpp:156 / rank_data_structures.hpp:272-282 */
static inline u64 swap_bytes(u64 x) { return __builtin_bswap64(x); }

/* ------------------------------------------------------------------------ */
/* a1: index file format.  bit_vector.hpp:65-109 (header + checks) and      */
/* bit_vector.hpp:111-128 (raw read), byte swap rank_data_structures.hpp:98 */
/* ------------------------------------------------------------------------ */

/* Returns the bit count stored in the file header, or a negative error code:
 * -1 cannot open, -2 file shorter than 8 bytes, -3 zero bits, -4 file holds
 * fewer than ceil(n/8) data bytes.  bit_vector.hpp:65-101. */
int64_t orc_file_bits(const char *path)
{
    FILE *f = fopen(path, "rb");
    if (!f) return -1;
    if (fseek(f, 0, SEEK_END) != 0) { fclose(f); return -1; }
    long size = ftell(f);
    if (size < 8) { fclose(f); return -2; }
    fseek(f, 0, SEEK_SET);
    unsigned char hdr[8];
    if (fread(hdr, 1, 8, f) != 8) { fclose(f); return -2; }
    fclose(f);
    u64 n = 0;
    for (int i = 0; i < 8; i++) n |= ((u64)hdr[i]) << (8 * i); /* bit_vector.hpp:85-88 */
    if (n == 0) return -3;                                         /* bit_vector.hpp:90-94 */
    u64 nbytes = (n + 7ull) / 8ull;                                /* bit_vector.hpp:96 */
    if ((u64)size - 8ull < nbytes) return -4;                      /* bit_vector.hpp:97-101 */
    return (int64_t)n;
}

/* Words in memory, padded to a multiple of 4096 bits.  bit_vector.hpp:104 */
u64 orc_padded_words(u64 n_bits) { return ((n_bits + 4095ull) / 4096ull) * 4096ull / 64ull; }

/* Reads ceil(n/8) data bytes into `words` (caller zero-fills all
 * orc_padded_words(n) words first) and byte-swaps every word, giving the
 * layout the reference's device code reads: position p at bit (63 - p%64) of
 * word p/64.  bit_vector.hpp:111-128, rank_data_structures.hpp:98,103-113.
 * Divergence: the reference leaves the bytes of the last partial word past
 * ceil(n/8) uninitialised (bit_vector.hpp:119-124); here they are zero. */
int orc_read_words(const char *path, u64 *words, u64 n_words_padded)
{
    int64_t n = orc_file_bits(path);
    if (n < 0) return (int)n;
    if (orc_padded_words((u64)n) > n_words_padded) return -5;
    FILE *f = fopen(path, "rb");
    if (!f) return -1;
    fseek(f, 8, SEEK_SET);
    u64 nbytes = ((u64)n + 7ull) / 8ull;
    if (fread(words, 1, nbytes, f) != nbytes) { fclose(f); return -4; }
    fclose(f);
    for (u64 i = 0; i < n_words_padded; i++) words[i] = swap_bytes(words[i]);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* a2: poppy / cum_poppy rank structures.  rank_data_structures.hpp:59-198  */
/* ------------------------------------------------------------------------ */

enum { ORC_POPPY = 1, ORC_CUM_POPPY = 2 }; /* enums.hpp:9-10 */

static u32 log2_hyper(u32 sb) { return sb == 4096u ? 31u : 32u; } /* rank_data_structures.hpp:64-66 */

/* rank_data_structures.hpp:67 */
u64 orc_l0_words(u64 n_bits, u32 sb) { return 1ull + (n_bits >> log2_hyper(sb)); }
/* rank_data_structures.hpp:68 (includes the sentinel entry) */
u64 orc_l12_words(u64 n_bits, u32 sb) { return 1ull + ((n_bits + sb - 1ull) / sb * sb) / sb; }

/* Fills L0 and L12 exactly as RankDataStructures::precount_the_structures_
 * based_on_words_in_basicblock does (rank_data_structures.hpp:142-198),
 * including the sentinel entry (:158-161).  `words` are already byte-swapped
 * (popcount does not depend on byte order; the reference swaps while
 * counting, :98).  Returns the absolute number of ones (:150,193) through
 * *abs_ones.  Returns 0, or -1 for an unsupported (sb, kind). */
int orc_rank_build(const u64 *words, u64 n_bits, u32 sb, int kind, u64 *L0, u64 *L12, u64 *abs_ones)
{
    if (!(sb == 256 || sb == 512 || sb == 1024 || sb == 2048 || sb == 4096)) return -1;
    if (kind != ORC_POPPY && kind != ORC_CUM_POPPY) return -1;
    if (sb == 4096 && kind != ORC_POPPY) return -1; /* parameters.hpp:273-277 */
    const u32 wbb = sb / 256u;                       /* words per basic block */
    const u64 n_l0 = orc_l0_words(n_bits, sb);
    const u64 n_l12 = orc_l12_words(n_bits, sb);
    const u64 bits_in_hyper = 1ull << log2_hyper(sb);
    const u64 sb_per_hyper = bits_in_hyper / sb;
    const u32 one_if_4096 = (sb == 4096u);
    u64 i_data = 0, i12 = 0, absolute = 0;
    for (u64 i0 = 0; i0 < n_l0; i0++) {
        L0[i0] = absolute;
        u32 rel = 0;
        for (u64 r = 0; r < sb_per_hyper; r++) {
            if (i12 >= n_l12 - 1ull) { /* sentinel, :158-161 */
                L12[i12] = ((u64)rel) << (32 + one_if_4096);
                *abs_ones = absolute;
                return 0;
            }
            u32 bb[4];
            for (u32 b = 0; b < 4; b++) {
                u32 pc = 0;
                for (u32 j = 0; j < wbb; j++) pc += popc64(words[i_data + b * wbb + j]);
                bb[b] = pc;
            }
            i_data += 4ull * wbb;
            if (kind == ORC_POPPY) { /* :170-173 */
                L12[i12] = (((u64)rel) << (32 + one_if_4096)) |
                           (((u64)bb[0]) << (20 + 2 * one_if_4096)) |
                           (((u64)bb[1]) << (10 + one_if_4096)) | ((u64)bb[2]);
            } else if (sb < 2048u) { /* :174-182 */
                L12[i12] = (((u64)rel) << 32) | (((u64)bb[0]) << 20) |
                           (((u64)(bb[0] + bb[1])) << 10) | ((u64)(bb[0] + bb[1] + bb[2]));
            } else { /* sb == 2048, :183-189 */
                L12[i12] = (((u64)rel) << 32) | (((u64)bb[0]) << 22) |
                           (((u64)(bb[0] + bb[1])) << 11) | ((u64)(bb[0] + bb[1] + bb[2]));
            }
            i12++;
            u32 cnt = bb[0] + bb[1] + bb[2] + bb[3];
            absolute += cnt;
            rel += cnt;
        }
    }
    *abs_ones = absolute;
    return 0;
}

/* ------------------------------------------------------------------------ */
/* a4: device rank.  rank_kernel.hpp:212-296 (+ dispatch :398-415).         */
/* ------------------------------------------------------------------------ */

static u32 log2u(u32 x) { u32 l = 0; while ((1u << l) < x) l++; return l; }

/* popcount_inside_basic_block_normal, rank_kernel.hpp:212-251: ones in the
 * basic block of i that precede i. */
static u64 pop_inside_bb(const u64 *data, u32 sb, u64 i)
{
    if (sb == 256u) return popc64(shr64(data[i >> 6], 64u - (u32)(i & 63u))); /* :216-219 */
    const u32 wbb = sb / 256u;
    const u32 logbb = log2u(sb / 4u);
    const u64 *blk = data + (i >> logbb) * wbb; /* load_2_uint64_words, :103-122 */
    const u32 iW = (u32)((i >> 6) & (wbb - 1u));
    const u32 target = 64u - (u32)(i & 63u);
    u64 pc = 0;
    for (u32 j = 0; j < wbb; j++) {
        u32 s = (j == iW) * target + ((j > iW) << 6); /* :228-247 */
        pc += popc64(shr64(blk[j], s));
    }
    return pc;
}

/* popcount_before_basic_block, rank_kernel.hpp:253-296 */
static u64 pop_before_bb(const u64 *L0, const u64 *L12, u32 sb, int kind, u64 i)
{
    const u32 logsb = log2u(sb);
    const u32 logbb = logsb - 2u;
    const u64 e = L12[i >> logsb];
    const u32 b = (u32)((i & (sb - 1u)) >> logbb);
    if (kind == ORC_POPPY) {
        if (sb == 4096u) { /* :260-266 */
            u64 bc = shr64(e & 0x1ffffffffull, (3u - b) * 11u);
            return L0[i >> 31] + (e >> 33) + ((bc & 0x7ffu) + ((bc >> 11) & 0x7ffu) + (bc >> 22));
        }
        u32 bc = shr32((u32)(e & 0x3fffffffu), (3u - b) * 10u); /* :268-275 */
        return L0[i >> 32] + (e >> 32) + ((bc & 0x3ffu) + ((bc >> 10) & 0x3ffu) + ((bc >> 20) & 0x3ffu));
    }
    if (sb == 2048u) { /* :282-287; a u32 shifted by 33 is 0 under PTX */
        u32 bc = shr32((u32)(e & 0xffffffffu), (3u - b) * 11u);
        return L0[i >> 32] + (e >> 32) + (bc & 0x7ffu);
    }
    u32 bc = shr32((u32)(e & 0x3fffffffu), (3u - b) * 10u); /* :288-293 */
    return L0[i >> 32] + (e >> 32) + (bc & 0x3ffu);
}

/* rank, rank_kernel.hpp:409-415: number of ones in [0, i). */
u64 orc_rank(const u64 *data, const u64 *L0, const u64 *L12, u32 sb, int kind, u64 i)
{
    return pop_inside_bb(data, sb, i) + pop_before_bb(L0, L12, sb, kind, i);
}

/* ------------------------------------------------------------------------ */
/* Index bundle used by presearch and search.                               */
/* ------------------------------------------------------------------------ */

typedef struct {
    const u64 *data[4];
    const u64 *L0[4];
    const u64 *L12[4];
    u64 C[5];
    u32 sb;
    int kind;
} orc_index;

/* a3: C array, matrix_sbwt.hpp:150-157 */
void orc_c_array(const u64 ones[4], u64 C[5])
{
    C[0] = 1ull;
    for (int c = 0; c < 4; c++) C[c + 1] = C[c] + ones[c];
}

static inline u64 rank_c(const orc_index *ix, u32 c, u64 i)
{
    return orc_rank(ix->data[c], ix->L0[c], ix->L12[c], ix->sb, ix->kind, i);
}

/* a6: presearch kernel, presearch_kernel.hpp:19-37 (no early exit; an empty
 * interval stays empty): the entry of p-mer idx (first letter in its top two
 * bits). */
static void presearch_entry(const orc_index *ix, u32 p, u64 idx, u64 *left, u64 *right)
{
    u32 c = (u32)((idx >> ((p - 1u) * 2u)) & 3u);
    u64 l = ix->C[c], r = ix->C[c + 1] - 1ull;
    for (int s = (int)((p - 2u) * 2u); s >= 0; s -= 2) {
        c = (u32)((idx >> s) & 3u);
        l = ix->C[c] + rank_c(ix, c, l);
        r = ix->C[c] + rank_c(ix, c, r + 1ull) - 1ull;
    }
    *left = l;
    *right = r;
}

static void presearch_index(orc_index *ix, const u64 *const data[4], const u64 *const L0[4],
                            const u64 *const L12[4], const u64 C[5], u32 sb, int kind)
{
    for (int c = 0; c < 4; c++) { ix->data[c] = data[c]; ix->L0[c] = L0[c]; ix->L12[c] = L12[c]; }
    memcpy(ix->C, C, sizeof(ix->C));
    ix->sb = sb; ix->kind = kind;
}

/* Writes all 4^p entries. */
void orc_presearch(const u64 *const data[4], const u64 *const L0[4], const u64 *const L12[4], const u64 C[5],
                   u32 sb, int kind, u32 p, u64 *lefts, u64 *rights)
{
    orc_index ix;
    presearch_index(&ix, data, L0, L12, C, sb, kind);
    const u64 count = 1ull << (2 * p);
#pragma omp parallel for schedule(static)
    for (u64 idx = 0; idx < count; idx++) presearch_entry(&ix, p, idx, lefts + idx, rights + idx);
}

/* The entries of the p-mers idx[0 .. count) only (tables too large to
 * restate whole in a test). */
void orc_presearch_at(const u64 *const data[4], const u64 *const L0[4], const u64 *const L12[4], const u64 C[5],
                      u32 sb, int kind, u32 p, const u64 *idx, u64 count, u64 *lefts, u64 *rights)
{
    orc_index ix;
    presearch_index(&ix, data, L0, L12, C, sb, kind);
#pragma omp parallel for schedule(static)
    for (u64 t = 0; t < count; t++) presearch_entry(&ix, p, idx[t], lefts + t, rights + t);
}

/* ------------------------------------------------------------------------ */
/* a7: query file reading, kmer_search.hpp:292-342 (read_file, add_paddings)*/
/* ------------------------------------------------------------------------ */

/* Restates KmerSearch::read_file on an in-memory copy of the file:
 * std::istream::getline(buf, size_of_file - number_of_letters) per line;
 * letters_in_row = gcount - 1 (so a final line without '\n' loses its last
 * letter, and a line that fills the buffer loses one more), lines starting
 * with '>' give no letters, every other non-empty line is one read.
 * Output: letters (concatenated, caller buffer of >= size bytes), row starts
 * (rows + 1 entries, caller buffer of >= size + 1 entries), returns the number
 * of rows; *n_letters and *n_kmers (sum over rows of max(0, len-k+1)) out.
 * kmer_search.hpp:319-342. */
int64_t orc_read_queries(const u8 *file, u64 size, u32 k, u8 *letters, u64 *starts, u64 *n_letters, u64 *n_kmers)
{
    u64 pos = 0, nl = 0, rows = 0, nk = 0;
    int good = 1;
    while (good) {
        /* one getline(letters + nl, size - nl) */
        u64 cap = size - nl; /* count argument; at most cap-1 chars stored */
        u64 stored = 0, gcount = 0;
        int first_char_is_gt = 0;
        if (cap == 0) { good = 0; break; } /* getline with count 0 sets failbit */
        for (;;) {
            if (pos >= size) { good = 0; break; } /* eofbit */
            u8 ch = file[pos];
            if (ch == '\n') { pos++; gcount++; break; } /* delimiter extracted */
            if (stored == cap - 1u) { good = 0; break; } /* failbit */
            if (stored == 0) first_char_is_gt = (ch == '>');
            letters[nl + stored] = ch;
            stored++; gcount++; pos++;
        }
        if (stored == 0 && gcount == 0 && !good) { /* nothing extracted */ }
        u64 row = gcount > 0 ? gcount - 1u : 0u; /* kmer_search.hpp:328 */
        if (stored == 0) first_char_is_gt = 0;
        if (first_char_is_gt) row = 0;            /* :329 */
        if (row) { starts[rows++] = nl; }
        if (row >= k) nk += row + 1u - k;         /* :335 */
        nl += row;
    }
    starts[rows] = nl; /* :338 */
    *n_letters = nl;
    *n_kmers = nk;
    return (int64_t)rows;
}

/* ------------------------------------------------------------------------ */
/* a8: 2-bit packing, create_kmer_string.hpp:18-42 (LUT :18-20).            */
/* ------------------------------------------------------------------------ */

static inline u64 letter_code(u8 ch)
{
    switch (ch) {
    case 'C': case 'c': return 1;
    case 'G': case 'g': return 2;
    case 'T': case 't': return 3;
    default: return 0; /* A/a and every other byte */
    }
}

/* Letter j of a 32-letter group goes to bits (63-2j, 62-2j).  The caller
 * passes n_letters already padded as add_paddings does (multiple of 32 with
 * at least 32 letters of zero padding, kmer_search.hpp:292-301). */
void orc_pack(const u8 *letters, u64 n_letters, u64 *words)
{
    u64 nw = n_letters / 32u;
#pragma omp parallel for schedule(static)
    for (u64 w = 0; w < nw; w++) {
        u64 x = 0;
        for (u32 j = 0; j < 32u; j++) x |= letter_code(letters[w * 32u + j]) << (62u - 2u * j);
        words[w] = x;
    }
}

/* a9: positions, positions_kernel.hpp:18-36.  Row r with letters in
 * [starts[r], starts[r+1]) contributes positions starts[r] + i for
 * i in [0, len-k].  Rows shorter than k contribute nothing (the reference's
 * kernel underflows there, positions_kernel.hpp:28-29). */
u64 orc_positions(const u64 *starts, u64 rows, u32 k, u64 *positions)
{
    u64 j = 0;
    for (u64 r = 0; r < rows; r++) {
        u64 len = starts[r + 1] - starts[r];
        if (len < k) continue;
        for (u64 i = 0; i + k <= len; i++) positions[j++] = starts[r] + i;
    }
    return j;
}

/* a10: k-mer extraction, search_kernel.hpp:66-68 */
static inline u64 extract_kmer(const u64 *words, u64 pos)
{
    u64 b = pos << 1;
    return (words[b >> 6] << (b & 63u)) | (shr64(words[(b >> 6) + 1u], 63u - (u32)(b & 63u)) >> 1);
}

/* a11: search kernel, search_kernel.hpp:61-104.  p == 0 means "without
 * presearch" (:79-81).  Writes the colex rank of each k-mer's node or
 * 0xFFFF_FFFF_FFFF_FFFF, and (if steps != NULL) the number of executed
 * loop iterations (one iteration = one rank pair), counted as the
 * reference executes them: stopping after the step that empties the
 * interval (:89-95). */
void orc_search(const u64 *const data[4], const u64 *const L0[4], const u64 *const L12[4], const u64 C[5],
                u32 sb, int kind, const u64 *lefts, const u64 *rights, u32 p, u32 k,
                const u64 *words, const u64 *positions, u64 n, u64 *answers, u8 *steps)
{
    orc_index ix;
    for (int c = 0; c < 4; c++) { ix.data[c] = data[c]; ix.L0[c] = L0[c]; ix.L12[c] = L12[c]; }
    memcpy(ix.C, C, sizeof(ix.C));
    ix.sb = sb; ix.kind = kind;
#pragma omp parallel for schedule(dynamic, 4096)
    for (u64 j = 0; j < n; j++) {
        u64 kmer = extract_kmer(words, positions[j]);
        u64 l, r;
        u32 i0;
        if (p) {
            u64 m = kmer >> (64u - 2u * p); /* :73 */
            l = lefts[m]; r = rights[m]; i0 = p;
        } else {
            l = 0; r = C[4] - 1ull; i0 = 0; /* :79-81 */
        }
        u32 s = 0;
        for (u32 i = i0; i < k; i++) {
            u32 c = (u32)((kmer >> (62u - 2u * i)) & 3u);
            l = C[c] + rank_c(&ix, c, l);
            r = C[c] + rank_c(&ix, c, r + 1ull) - 1ull;
            s++;
            if (l > r) break;
        }
        answers[j] = (l > r) ? ~0ull : l; /* :98-103 */
        if (steps) steps[j] = (u8)s;
    }
}

/* ------------------------------------------------------------------------ */
/* a13: text output, results_persister.hpp:82-95.  Each k-mer of a row as a */
/* signed int64 followed by one space; '\n' after each row.  Rows shorter   */
/* than k print an empty line (the reference underflows, :85).             */
/* Returns bytes written, or -1 if `cap` is too small.                      */
/* ------------------------------------------------------------------------ */
int64_t orc_format_answers(const u64 *starts, u64 rows, u32 k, const u64 *answers, char *out, u64 cap)
{
    u64 o = 0, j = 0;
    char tmp[32];
    for (u64 r = 0; r < rows; r++) {
        u64 len = starts[r + 1] - starts[r];
        u64 cnt = len >= k ? len - k + 1u : 0u;
        for (u64 i = 0; i < cnt; i++) {
            int m = snprintf(tmp, sizeof tmp, "%lld ", (long long)(int64_t)answers[j++]);
            if (o + (u64)m > cap) return -1;
            memcpy(out + o, tmp, (size_t)m);
            o += (u64)m;
        }
        if (o + 1u > cap) return -1;
        out[o++] = '\n';
    }
    return (int64_t)o;
}

int orc_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
