// stream.cuh -- select on the line layout and the backward step of the run
// walk (device side).  No reference counterpart: the reference searches every
// k-mer from scratch (include/gpu/search_kernel.hpp:61-104).
//
// SBWT facts used (plain-matrix SBWT, nodes in colex order):
//  * the nodes whose labels share their last k-1 letters y form a contiguous
//    "group", ordered by first letter ($ < A < C < G < T), at most 5 nodes;
//  * the outgoing edges of a group are marked only in the column of its
//    first node, so the node y.b is C[b] + rank_b(u0) for that first node u0,
//    and conversely u0 = select_b(v - C[b]) for the node v of y.b.
// So from the node v of the k-mer y.b, the node of the k-mer a.y (one letter
// to the left in the read) is the member of the group starting at
// select_b(v - C[b]) whose first letter is a, if there is one.  Per node the
// engine keeps four bits, two nodes per byte (even node in the low half): its
// first letter (0 = $, 1..4 = A..T) and a flag for the first node of its
// group (bit 3); and the backward table: per node v, pred(v) with the set of
// first letters of pred(v)'s group, so that a backward step is one load.
// select_c uses the line counts plus a sample of the line holding every 64th
// one.
#pragma once
#include "device.cuh"

namespace sbwt {
namespace dev {

constexpr u32 kSelLog = 6;          // one select sample per 64 ones
constexpr uint8_t kGroupStart = 8;  // node nibble: bit 3 = first node of its group
constexpr u32 kNoNode = 0;          // node 0 (the all-$ root) is never a k-mer's node

// Backward steps through the 8-byte-per-column backward table (1) or through
// select + node nibbles (0).
#ifndef SBWT_BACK_TABLE
#define SBWT_BACK_TABLE 1
#endif

// Position of the (i+1)-th one (0-based i) of the 64-bit MSB-first word w.
__device__ __forceinline__ u32 msb_select(u64 w, u32 i) {
    u32 pos = 0;
#pragma unroll
    for (u32 s = 32; s; s >>= 1) {
        const u32 c = __popcll(w >> (64u - s));
        if (i >= c) {
            i -= c;
            w <<= s;
            pos += s;
        }
    }
    return pos;
}

// select_c(i): position of the one of rank i in vector c, given its lines,
// their count and its select samples (sel[s] = line of the one of rank 64 s,
// n_samples = ceil(ones / 64)).  Returns ~0u if i is not the rank of a one.
__device__ __forceinline__ u32 line_select(const ulonglong4 *__restrict__ lines, u32 lpc, const u32 *__restrict__ sel,
                                           u32 n_samples, u32 i) {
    const u32 s = i >> kSelLog;
    if (s >= n_samples) return ~0u;
    u32 lo = __ldg(sel + s);
    u32 hi = s + 1 < n_samples ? __ldg(sel + s + 1) : lpc - 1;
    // last line in [lo, hi] whose count is <= i (its count word is the line's first 8 bytes)
    while (lo < hi) {
        const u32 mid = (lo + hi + 1) >> 1;
        if ((u32)(ld_nc(reinterpret_cast<const u64 *>(lines + mid)) >> 32) <= i) lo = mid;
        else hi = mid - 1;
    }
    const ulonglong4 w = ld_line(lines + lo);
    u32 r = i - (u32)(w.x >> 32);
    const u64 w0 = w.x << 32;  // data bits 0..31 at the top
    const u32 p0 = __popcll(w0), p1 = __popcll(w.y), p2 = __popcll(w.z), p3 = __popcll(w.w);
    u32 base;
    u64 x;
    if (r < p0) {
        base = 0, x = w0;
    } else if ((r -= p0) < p1) {
        base = 32, x = w.y;
    } else if ((r -= p1) < p2) {
        base = 96, x = w.z;
    } else if ((r -= p2) < p3) {
        base = 160, x = w.w;
    } else {
        return ~0u;
    }
    return lo * kLineBits + base + msb_select(x, r);
}

struct StreamView {
    const ulonglong4 *lines;
    u32 lpc;
    const u32 *sel;        // 4 sample arrays, vector c at sel + sel_off[c]
    u32 sel_off[4];
    u32 sel_n[4];
    const uint8_t *node;   // per node a nibble (first letter | kGroupStart), two per byte
    const u64 *back;       // backward table: per node pred(v) | group_letters(pred(v)) << 32
    u32 n;                 // nodes
    u32 C[4];

    __device__ __forceinline__ u32 last_letter(u32 v) const {
        return v >= C[3] ? 3u : v >= C[2] ? 2u : v >= C[1] ? 1u : 0u;
    }

    // First node of the group of v's predecessor: select_b(v - C[b]), b = last letter of v (v >= 1).
    __device__ __forceinline__ u32 pred(u32 v) const {
        const u32 b = last_letter(v);
        const u32 cb = b == 0 ? C[0] : b == 1 ? C[1] : b == 2 ? C[2] : C[3];
        return line_select(lines + (u64)b * lpc, lpc, sel + sel_off[b], sel_n[b], v - cb);
    }

    // Letters present as first letters in the group that starts at u0 (bit 0 = $, bit 1 + c = letter c).
    __device__ __forceinline__ u32 group_letters(u32 u0) const {
        u32 m = 0;
        u32 u = u0;
#pragma unroll 1
        for (u32 g = 0; g < 5u && u < n; g++, u++) {
            const u32 f = (u32)(__ldg(node + (u >> 1)) >> ((u & 1u) << 2)) & 15u;
            if (g && (f & kGroupStart)) break;
            m |= 1u << (f & 7u);
        }
        return m;
    }

#if SBWT_BACK_TABLE
    // Node of the k-mer a.y given the node v of the k-mer y.b, or kNoNode: one
    // load of v's entry u0 | group_letters(u0) << 32 (the backward table); the
    // member with first letter a sits after the members with smaller ones.
    __device__ __forceinline__ u32 back_step(u32 v, u32 a, bool ef, u64 pol) const {
        const u64 e = ld_gather_u64(back + v, ef, pol);
        const u32 m = (u32)(e >> 32);
        if (!((m >> (a + 1u)) & 1u)) return kNoNode;
        return (u32)e + (u32)__popc(m & ((1u << (a + 1u)) - 1u));
    }
#else
    // Node of the k-mer a.y given the node v of the k-mer y.b, or kNoNode.
    __device__ __forceinline__ u32 back_step(u32 v, u32 a, bool, u64) const {
        u32 u = pred(v);
        if (u >= n) return kNoNode;
        const u32 want = a + 1u;
#pragma unroll 1
        for (u32 g = 0; g < 5u && u < n; g++, u++) {
            const u32 f = (u32)(__ldg(node + (u >> 1)) >> ((u & 1u) << 2)) & 15u;
            if (g && (f & kGroupStart)) break;
            const u32 first = f & 7u;
            if (first == want) return u;
            if (first > want) break;
        }
        return kNoNode;
    }
#endif
};

}  // namespace dev
}  // namespace sbwt
