// rank.cuh -- one search step (a rank pair) on either layout, split into a
// fetch phase (issue every load) and a finish phase (popcounts), so that a
// thread can keep the loads of several k-mers in flight at once.
//
// A step with letter c maps the interval [l, r] to
//   l' = C[c] + rank_c(l),  r' = C[c] + rank_c(r + 1) - 1
// (include/gpu/search_kernel.hpp:86-88, include/gpu/presearch_kernel.hpp:
// 138-140).  TPK lanes may share one step: each loads 1/TPK of the words and
// the partial counts are summed with __shfl_xor_sync inside the lane group
// (the reference's "shuffles" variants, include/gpu/rank_kernel.hpp:298-396).
#pragma once
#include "device.cuh"

namespace sbwt {
namespace dev {

// ------------------------------------------------------------------ LINES

template <int TPK = 1>
struct LinesRankerT {
    using IT = u32;
    static constexpr int W = 4 / TPK;  // u64 words of a line held by one lane
    const ulonglong4 *lines;
    u32 lpc;

    // TPK == 1: whole lines in registers.  A single-node interval (l == r, the
    // common case once a k-mer is matched) needs one line: rank(r+1) =
    // rank(l) + bit(l), whichever line l+1 falls in.
    struct Fetch {
        ulonglong4 a, b;
        u64 pa[W], pb[W];  // TPK > 1: this lane's words
        u32 qa, qb;
        bool two, single;
    };

    __device__ __forceinline__ static void load_part(const ulonglong4 *line, u32 sub, u64 (&w)[W]) {
        if constexpr (TPK == 2) {
            const ulonglong2 v = ld_nc2(reinterpret_cast<const ulonglong2 *>(line) + sub);
            w[0] = v.x;
            w[1] = v.y;
        } else {
            w[0] = ld_nc(reinterpret_cast<const u64 *>(line) + sub);
        }
    }

    // count word of the line (word 0) + ones of this lane's words before q
    __device__ __forceinline__ static u32 part(const u64 (&w)[W], u32 sub, u32 q) {
        u32 s = 0;
#pragma unroll
        for (int t = 0; t < W; t++) {
            const u32 wi = sub * W + t;
            s += word_prefix(w[t], wi, q);
            if (wi == 0) s += (u32)(w[t] >> 32);
        }
        return s;
    }

    __device__ __forceinline__ Fetch fetch(u32 c, u32 l, u32 r, u32 sub) const {
        Fetch f;
        const ulonglong4 *base = lines + (u64)c * lpc;
        u32 la, lb;
        line_split(l, la, f.qa);
        line_split(r + 1u, lb, f.qb);
        f.two = lb != la;
        if constexpr (TPK == 1) {
            f.single = l == r;
            f.a = ld_line(base + la);
            if (!f.single && f.two) f.b = ld_line(base + lb);
        } else {
            f.single = false;
            load_part(base + la, sub, f.pa);
            if (f.two) load_part(base + lb, sub, f.pb);
        }
        return f;
    }

    __device__ __forceinline__ void finish(const Fetch &f, u32 Cc, u32 &l, u32 &r, u32 sub, u32 gmask) const {
        if constexpr (TPK == 1) {
            const LineSums sa = line_sums(f.a);
            u32 bit;
            const u32 ra = sums_rank(sa, f.qa, bit);
            l = Cc + ra;
            if (f.single) {
                r = Cc + ra + bit - 1u;
            } else {
                u32 bb;
                const u32 rb = f.two ? sums_rank(line_sums(f.b), f.qb, bb) : sums_rank(sa, f.qb, bb);
                r = Cc + rb - 1u;
            }
        } else {
            u32 ra = part(f.pa, sub, f.qa);
            u32 rb = f.two ? part(f.pb, sub, f.qb) : part(f.pa, sub, f.qb);
#pragma unroll
            for (int o = 1; o < TPK; o <<= 1) {
                ra += __shfl_xor_sync(gmask, ra, o);
                rb += __shfl_xor_sync(gmask, rb, o);
            }
            l = Cc + ra;
            r = Cc + rb - 1u;
        }
    }

    __device__ __forceinline__ void step(u32 c, u32 Cc, u32 &l, u32 &r) const {
        const Fetch f = fetch(c, l, r, 0);
        finish(f, Cc, l, r, 0, 0xffffffffu);
    }
};
using LinesRanker = LinesRankerT<1>;

// ------------------------------------------------------------- WIDE lines

template <int S>
struct WideRanker {
    using IT = u32;
    using Sh = WideShape<S>;
    const ulonglong4 *lines;  // vector c's line j at lines + (c * lpc + j) * S
    u32 lpc;

    // Per rank: the header sector of its line and the sector holding its bit
    // (the header again when that is sector 0).  A single-node interval
    // (l == r) needs one rank: rank(r+1) = rank(l) + bit(l).
    struct Fetch {
        ulonglong4 ha, xa, hb, xb;
        u32 qa, qb;
        bool single;
    };

    __device__ __forceinline__ void load(const ulonglong4 *base, u32 x, u32 &q, ulonglong4 &h, ulonglong4 &d) const {
        const u32 line = x / Sh::kDataBits;
        q = x - line * Sh::kDataBits;
        const ulonglong4 *ln = base + (u64)line * S;
        const u32 sec = (Sh::kHeaderBits + q) >> 8;
        h = ld_line(ln);
        d = sec ? ld_line(ln + sec) : h;
    }

    __device__ __forceinline__ Fetch fetch(u32 c, u32 l, u32 r, u32) const {
        Fetch f;
        const ulonglong4 *base = lines + (u64)c * lpc * S;
        f.single = l == r;
        load(base, l, f.qa, f.ha, f.xa);
        if (!f.single) load(base, r + 1u, f.qb, f.hb, f.xb);
        return f;
    }

    __device__ __forceinline__ void finish(const Fetch &f, u32 Cc, u32 &l, u32 &r, u32, u32) const {
        u32 bit;
        const u32 ra = wide_rank<S>(f.ha, f.xa, f.qa, bit);
        l = Cc + ra;
        if (f.single) {
            r = Cc + ra + bit - 1u;
        } else {
            u32 bb;
            r = Cc + wide_rank<S>(f.hb, f.xb, f.qb, bb) - 1u;
        }
    }

    __device__ __forceinline__ void step(u32 c, u32 Cc, u32 &l, u32 &r) const {
        const Fetch f = fetch(c, l, r, 0);
        finish(f, Cc, l, r, 0, 0xffffffffu);
    }
};

// ------------------------------------------------------------------ POPPY

template <int SB, int KIND, class ITT, int TPK = 1>
struct PoppyRanker {
    using IT = ITT;
    using S = PoppyShape<SB>;
    static constexpr int W = (S::kWordsBB / TPK) > 0 ? (S::kWordsBB / TPK) : 1;  // words per lane
    const u64 *bits;
    const u64 *L0;
    const u64 *L12;
    u64 wpv, l0w, l12w;

    struct One {
        u64 e, l0;
        u64 w[W];
        u64 i;
    };
    struct Fetch {
        One a, b;
    };

    __device__ __forceinline__ One load(u32 c, u64 i, u32 sub) const {
        One o;
        o.i = i;
        o.e = ld_nc(L12 + (u64)c * l12w + (i >> S::kLogSB));
        o.l0 = ld_nc(L0 + (u64)c * l0w + (i >> S::kLogHyper));
        const u64 *blk = bits + (u64)c * wpv + (i >> S::kLogBB) * (u64)S::kWordsBB + (u64)sub * W;
        if constexpr (W == 1) {
            o.w[0] = ld_nc(blk);
        } else {
#pragma unroll
            for (int t = 0; t < W; t += 2) {
                const ulonglong2 v = ld_nc2(reinterpret_cast<const ulonglong2 *>(blk) + t / 2);
                o.w[t] = v.x;
                o.w[(t + 1) % W] = v.y;
            }
        }
        return o;
    }

    // ones of this lane's words of the basic block that precede i
    __device__ __forceinline__ static u64 part(const One &o, u32 sub) {
        const u32 iw = (u32)((o.i >> 6) & (S::kWordsBB - 1));
        const u32 i63 = (u32)(o.i & 63u);
        u64 s = 0;
#pragma unroll
        for (int t = 0; t < W; t++) s += bb_word_prefix(o.w[t], sub * W + t, iw, i63);
        return s;
    }

    __device__ __forceinline__ static u64 before(const One &o) {
        const u32 b = (u32)((o.i & (SB - 1)) >> S::kLogBB);
        return o.l0 + poppy_before_bb<SB, KIND>(o.e, b);
    }

    __device__ __forceinline__ Fetch fetch(u32 c, IT l, IT r, u32 sub) const {
        Fetch f;
        f.a = load(c, (u64)l, sub);
        f.b = load(c, (u64)r + 1ull, sub);
        return f;
    }

    __device__ __forceinline__ void finish(const Fetch &f, IT Cc, IT &l, IT &r, u32 sub, u32 gmask) const {
        u64 pa = part(f.a, sub), pb = part(f.b, sub);
#pragma unroll
        for (int o = 1; o < TPK; o <<= 1) {
            pa += __shfl_xor_sync(gmask, pa, o);
            pb += __shfl_xor_sync(gmask, pb, o);
        }
        l = Cc + (IT)(before(f.a) + pa);
        r = Cc + (IT)(before(f.b) + pb) - (IT)1;
    }

    __device__ __forceinline__ void step(u32 c, IT Cc, IT &l, IT &r) const {
        const Fetch f = fetch(c, l, r, 0);
        finish(f, Cc, l, r, 0, 0xffffffffu);
    }
};

}  // namespace dev
}  // namespace sbwt
