// device.cuh -- device-side layouts and rank functions (sm_100a).
//
// Two rank layouts are served:
//
//  * LINES (this engine's search layout).  Each of the four vectors is cut
//    into 224-bit blocks; block b is stored as one 32-byte line (= one L2
//    sector) holding a 32-bit count of the ones before the block followed by
//    the block's 224 bits.  Line bits are MSB-first across the four u64
//    words: word0 = count << 32 | bits 0..31, word1 = bits 32..95,
//    word2 = bits 96..159, word3 = bits 160..223 (bit q of the block at line
//    bit 32+q, line bit b at bit 63-b%64 of word b/64).  rank_c(i) is one
//    256-bit load plus a masked popcount: one sector per rank, where the
//    reference's poppy needs an L12 word and a basic block in different
//    sectors (include/gpu/rank_kernel.hpp:212-296).  Counts are 32-bit, so
//    the layout serves indexes of fewer than 224 * 2^24 - 1 columns.
//
//  * POPPY (the reference layout).  L0 / L12 words exactly as
//    RankDataStructures builds them (include/rank_data_structures.hpp:
//    142-198) over the raw vectors; rank as include/gpu/rank_kernel.hpp:
//    212-296 + 409-415 defines it.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace sbwt {
namespace dev {

using u64 = uint64_t;
using u32 = uint32_t;

constexpr u32 kLineBits = 224;      // data bits per 32-byte line
constexpr u32 kLineBytes = 32;
constexpr u32 kMaxLinesPerChar = 1u << 24;  // 32-bit counts: 224 * 2^24 < 2^32

// Build option SBWT_LINES_EVICT_LAST=1: lines are read with an L2
// evict-last policy (kept in L2 ahead of other data).
#ifndef SBWT_LINES_EVICT_LAST
#define SBWT_LINES_EVICT_LAST 0
#endif

// Cache operator of the random gathers: SBWT_GATHER_CG = 1 reads the
// presearch and backward-table entries with ld.global.cg (cached in L2
// only), 2 also the rank lines; 0 reads them through the read-only L1 path
// (ld.global.nc).
#ifndef SBWT_GATHER_CG
#define SBWT_GATHER_CG 0
#endif
#if SBWT_GATHER_CG >= 2
#define SBWT_LINE_LD "ld.global.cg"
#else
#define SBWT_LINE_LD "ld.global.nc"
#endif
#if SBWT_GATHER_CG >= 1
#define SBWT_GATHER_LD "ld.global.cg"
#else
#define SBWT_GATHER_LD "ld.global.nc"
#endif

// 256-bit read-only load of one line (sm_100 supports .v4.u64 global loads).
__device__ __forceinline__ ulonglong4 ld_line(const ulonglong4 *p) {
    ulonglong4 v;
#if SBWT_LINES_EVICT_LAST
    u64 pol;
    asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
    asm(SBWT_LINE_LD ".L2::cache_hint.v4.u64 {%0, %1, %2, %3}, [%4], %5;"
        : "=l"(v.x), "=l"(v.y), "=l"(v.z), "=l"(v.w)
        : "l"(p), "l"(pol));
#else
    asm(SBWT_LINE_LD ".v4.u64 {%0, %1, %2, %3}, [%4];"
        : "=l"(v.x), "=l"(v.y), "=l"(v.z), "=l"(v.w)
        : "l"(p));
#endif
    return v;
}

__device__ __forceinline__ ulonglong2 ld_nc2(const ulonglong2 *p) {
    ulonglong2 v;
    asm("ld.global.nc.v2.u64 {%0, %1}, [%2];" : "=l"(v.x), "=l"(v.y) : "l"(p));
    return v;
}

__device__ __forceinline__ u64 ld_nc(const u64 *p) {
    u64 v;
    asm("ld.global.nc.u64 %0, [%1];" : "=l"(v) : "l"(p));
    return v;
}

// Gathers with little reuse (a presearch entry, a backward-table entry) from
// a table too large to stay in L2 are read with an L2 evict-first policy, so
// that they do not push the lines of the rank steps out of L2; gathers from a
// table that fits use evict-normal (evict-first there makes them miss:
// measured 28 % slower on an L2-resident index).  createpolicy and
// .L2::cache_hint: PTX ISA 7.4+, sm_80+.  Build option
// SBWT_GATHER_EVICT_FIRST=0 reads them plainly.
#ifndef SBWT_GATHER_EVICT_FIRST
#define SBWT_GATHER_EVICT_FIRST 1
#endif

__device__ __forceinline__ u64 l2_evict_first_policy() {
    u64 p;
    asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}

// Compact presearch entry (one u32): left end L in the low kPreLBits bits,
// width w = R - L + 1 above it; w = 0 is an empty interval and w =
// kPreEscape means the interval is too wide for the field (the 8-byte entry
// holds it).  Halves the table, so that at p = 12 (64 MiB) it can stay in L2.
constexpr u32 kPreLBits = 27;
constexpr u32 kPreEscape = 31;
constexpr u64 kPreMaxColumns = 1ull << kPreLBits;

__host__ __device__ __forceinline__ u32 pre_compact(u32 l, u32 r) {
    if (l > r) return 0u;
    const u32 w = r - l + 1u;
    return l | ((w < kPreEscape ? w : kPreEscape) << kPreLBits);
}

// A gather: with the evict-first policy pol when ef is set, plainly otherwise.
__device__ __forceinline__ uint2 ld_gather_u32x2(const uint2 *p, bool ef, u64 pol) {
#if SBWT_GATHER_EVICT_FIRST
    if (ef) {
        uint2 v;
        asm(SBWT_GATHER_LD ".L2::cache_hint.v2.u32 {%0, %1}, [%2], %3;" : "=r"(v.x), "=r"(v.y) : "l"(p), "l"(pol));
        return v;
    }
#endif
    (void)ef;
    (void)pol;
    return __ldg(p);
}

__device__ __forceinline__ u64 ld_gather_u64(const u64 *p, bool ef, u64 pol) {
#if SBWT_GATHER_EVICT_FIRST
    if (ef) {
        u64 v;
        asm(SBWT_GATHER_LD ".L2::cache_hint.u64 %0, [%1], %2;" : "=l"(v) : "l"(p), "l"(pol));
        return v;
    }
#endif
    (void)ef;
    (void)pol;
    return __ldg(reinterpret_cast<const unsigned long long *>(p));
}

// x >> s with the PTX rule that s >= 64 gives 0 (the reference relies on it,
// include/gpu/rank_kernel.hpp:218,226-229).
__device__ __forceinline__ u64 shr_clamp(u64 x, u32 s) {
    u64 r;
    asm("shr.b64 %0, %1, %2;" : "=l"(r) : "l"(x), "r"(s));
    return r;
}

__device__ __forceinline__ u32 shr_clamp32(u32 x, u32 s) {
    u32 r;
    asm("shr.b32 %0, %1, %2;" : "=r"(r) : "r"(x), "r"(s));
    return r;
}

// Ones among the top `b` bits of w, b in [0, 64].
__device__ __forceinline__ u32 popc_top(u64 w, u32 b) { return __popcll(shr_clamp(w, 64u - b)); }

__device__ __forceinline__ u32 clamp64(int v) { return (u32)min(max(v, 0), 64); }

// Ones among the first q data bits of a line (q in [0, 224]).
__device__ __forceinline__ u32 line_prefix(const ulonglong4 &w, u32 q) {
    const int t = (int)q + 32;  // line bits [32, t)
    return popc_top(w.x & 0xffffffffull, clamp64(t)) + popc_top(w.y, clamp64(t - 64)) +
           popc_top(w.z, clamp64(t - 128)) + popc_top(w.w, clamp64(t - 192));
}

// Partial form used when TPK lanes share a line: lane `part` of `parts`
// (parts = 2: two u64 words each; parts = 4: one word each) counts its words.
__device__ __forceinline__ u32 word_prefix(u64 w, u32 word_index, u32 q) {
    const int t = (int)q + 32 - 64 * (int)word_index;
    if (word_index == 0) w &= 0xffffffffull;
    return popc_top(w, clamp64(t));
}

// rank of line layout: count stored in the line + prefix popcount.
__device__ __forceinline__ u32 line_rank_from(const ulonglong4 &w, u32 q) {
    return (u32)(w.x >> 32) + line_prefix(w, q);
}

// Per-line running popcounts, shared by every rank taken in that line:
// count = ones before the line, p1..p3 = ones in line words 0 (data half),
// 0..1 and 0..2.
struct LineSums {
    u32 count, p1, p2, p3;
    u64 w0, w1, w2, w3;
};

__device__ __forceinline__ LineSums line_sums(const ulonglong4 &w) {
    LineSums s;
    s.count = (u32)(w.x >> 32);
    s.w0 = w.x & 0xffffffffull;
    s.w1 = w.y;
    s.w2 = w.z;
    s.w3 = w.w;
    s.p1 = __popcll(s.w0);
    s.p2 = s.p1 + __popcll(s.w1);
    s.p3 = s.p2 + __popcll(s.w2);
    return s;
}

// rank at data position q (< 224) of the line: the full words before the one
// holding q come from the running sums, that word is masked by one clamped
// shift.  *bit = the bit at q itself.
__device__ __forceinline__ u32 sums_rank(const LineSums &s, u32 q, u32 &bit) {
    const u32 t = q + 32u;  // line bit of q
    const u32 wi = t >> 6, b = t & 63u;
    const u32 full = wi == 0 ? 0u : wi == 1 ? s.p1 : wi == 2 ? s.p2 : s.p3;
    const u64 w = wi == 0 ? s.w0 : wi == 1 ? s.w1 : wi == 2 ? s.w2 : s.w3;
    bit = (u32)(w >> (63u - b)) & 1u;
    return s.count + full + __popcll(shr_clamp(w, 64u - b));
}

__device__ __forceinline__ void line_split(u32 x, u32 &line, u32 &q) {
    line = x / kLineBits;
    q = x - line * kLineBits;
}

// ------------------------------------------------------------- wide lines
//
// WIDE lines: the interleave block widened to S sectors (S = 2: 512-bit
// lines, S = 8: 2048-bit lines), with a two-level count so that a rank still
// reads at most two sectors of its line.  Line bits (MSB-first across the
// line's u64 words, as in LINES): [0, 32) the ones before the line (32-bit),
// then S-1 16-bit fields sub[1..S-1] (sub[s] = ones of the line's data bits
// that lie in sectors 0..s-1), then the data bits: data bit q at line bit
// H + q, H = 32 + 16 (S-1).  rank_c(i) = count + sub[s] + the ones of sector
// s before i's bit, s = the sector holding i's bit; the header sector and
// that sector are independent loads.  Fewer count bits per data bit than
// LINES (1.6 % at S = 8 against 14 %), one more sector per rank where the
// bit lies past the first sector.
template <int S> struct WideShape {
    static constexpr u32 kSectors = S;
    static constexpr u32 kHeaderBits = 32u + 16u * (S - 1);
    static constexpr u32 kDataBits = 256u * S - kHeaderBits;
};

// Ones among the first b bits (MSB-first, b in [0, 256]) of a 256-bit sector.
__device__ __forceinline__ u32 sector_prefix(const ulonglong4 &x, u32 b) {
    const int t = (int)b;
    return popc_top(x.x, clamp64(t)) + popc_top(x.y, clamp64(t - 64)) + popc_top(x.z, clamp64(t - 128)) +
           popc_top(x.w, clamp64(t - 192));
}

__device__ __forceinline__ u64 sector_word(const ulonglong4 &x, u32 i) {
    return i == 0 ? x.x : i == 1 ? x.y : i == 2 ? x.z : x.w;
}

// sub[s] of the header sector h (1 <= s < S).
template <int S> __device__ __forceinline__ u32 wide_sub(const ulonglong4 &h, u32 s) {
    const u32 b0 = 32u + 16u * (s - 1u);  // line bit of the field
    return (u32)(sector_word(h, b0 >> 6) >> (48u - (b0 & 63u))) & 0xffffu;
}

// rank at data position q of a line (header sector h, x = the sector holding
// q's bit, x = h when that is sector 0); *bit = the bit at q.
template <int S> __device__ __forceinline__ u32 wide_rank(const ulonglong4 &h, const ulonglong4 &x, u32 q, u32 &bit) {
    constexpr u32 H = WideShape<S>::kHeaderBits;
    const u32 t = H + q, s = t >> 8, tb = t & 255u;
    bit = (u32)(sector_word(x, tb >> 6) >> (63u - (tb & 63u))) & 1u;
    const u32 before = s ? wide_sub<S>(h, s) : 0u;
    const u32 in_sector = sector_prefix(x, tb) - (s ? 0u : sector_prefix(h, H));
    return (u32)(h.x >> 32) + before + in_sector;
}

// ------------------------------------------------------------------ poppy

template <int SB> struct PoppyShape {
    static constexpr int kLogSB = SB == 256 ? 8 : SB == 512 ? 9 : SB == 1024 ? 10 : SB == 2048 ? 11 : 12;
    static constexpr int kLogBB = kLogSB - 2;
    static constexpr int kWordsBB = SB / 256;             // u64 words per basic block
    static constexpr int kLogHyper = SB == 4096 ? 31 : 32;  // rank_data_structures.hpp:64-66
    static constexpr int kRelShift = SB == 4096 ? 33 : 32;
};

// Ones of the basic blocks of superblock entry e that precede basic block b
// (include/gpu/rank_kernel.hpp:253-296).
template <int SB, int KIND>
__device__ __forceinline__ u64 poppy_before_bb(u64 e, u32 b) {
    if (KIND == 1) {
        if (SB == 4096) {
            const u64 bc = shr_clamp(e & 0x1ffffffffull, (3u - b) * 11u);
            return (e >> 33) + ((bc & 0x7ffu) + ((bc >> 11) & 0x7ffu) + (bc >> 22));
        }
        const u32 bc = shr_clamp32((u32)(e & 0x3fffffffu), (3u - b) * 10u);
        return (e >> 32) + ((bc & 0x3ffu) + ((bc >> 10) & 0x3ffu) + ((bc >> 20) & 0x3ffu));
    }
    if (SB == 2048) {
        const u32 bc = shr_clamp32((u32)(e & 0xffffffffu), (3u - b) * 11u);
        return (e >> 32) + (bc & 0x7ffu);
    }
    const u32 bc = shr_clamp32((u32)(e & 0x3fffffffu), (3u - b) * 10u);
    return (e >> 32) + (bc & 0x3ffu);
}

// Ones of word j of a basic block that precede position i (word iw holds i).
__device__ __forceinline__ u32 bb_word_prefix(u64 w, u32 j, u32 iw, u32 i63) {
    const u32 s = (j == iw) ? (64u - i63) : (j > iw ? 64u : 0u);
    return __popcll(shr_clamp(w, s));
}

}  // namespace dev
}  // namespace sbwt
