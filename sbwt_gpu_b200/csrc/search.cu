// search.cu -- the per-k-mer SBWT search (the hot path).
//
// Replaces epic::gpu::search (include/gpu/search_kernel.hpp:61-104), launched
// one thread per k-mer by launch_search_kernel (include/gpu/
// search_and_presearch_launchers.hpp:21-60), together with the per-read
// positions kernel (include/gpu/positions_kernel.hpp:18-36).
//
// Semantics kept from the reference, per k-mer:
//   kmer  = 64 bits from letter offset pos (search_kernel.hpp:66-68)
//   [l,r] = presearch entry of its first p letters, or [0, C[4]-1] without
//           presearch (:71-82)
//   for i = p..k-1: one rank-pair step with letter i, stop once l > r (:84-96)
//   answer = l if l <= r else 0xFFFF_FFFF_FFFF_FFFF (:98-103)
// An interval that is already empty is not stepped (an empty interval stays
// empty, so the answer is the same).
//
// Launch shape (this engine's own): a persistent grid of (#SMs x resident
// blocks).  Each warp takes chunks of consecutive k-mer indices from a global
// atomic cursor (work stealing), and each lane keeps KPT k-mers in flight in
// registers; a lane whose k-mer finishes takes the next index of its warp's
// chunk at once (ballot + popc), so lanes never idle behind a long k-mer.
// With TPK > 1, TPK lanes share one k-mer and split every 32-byte line.
// K-mers are located either through the reference's positions array
// (sbwt_search_packed) or through a per-row table (sbwt_search_reads): no
// positions array is materialised there.
#include <algorithm>
#include <type_traits>

#include "device.cuh"
#include "internal.h"
#include "mlp_kernels.cuh"
#include "rank.cuh"

namespace sbwt {
namespace {

using namespace dev;

constexpr u32 kFull = 0xffffffffu;
constexpr u32 kDone = 0xffffffffu;

template <class IT> struct PairOf;
template <> struct PairOf<u32> { using T = uint2; };
template <> struct PairOf<u64> { using T = ulonglong2; };

// Register budget per k-mer slot count: at least this many 256-thread blocks
// stay resident per SM.
template <int KPT> struct MinBlocks { static constexpr int value = KPT <= 1 ? 4 : KPT == 2 ? 3 : KPT <= 4 ? 2 : 1; };

template <class R, int KPT, int TPK>
__global__ void __launch_bounds__(256, MinBlocks<KPT>::value) search_kernel(const R rk, const SearchArgs a) {
    if (a.runs_dev && runs_usable(*a.runs_dev, a.n_kmers)) return;  // the run walk takes this kernel-contract call
    using IT = typename R::IT;
    using PT = typename PairOf<IT>::T;
    const u32 lane = threadIdx.x & 31u;
    const u32 sub = lane & (u32)(TPK - 1);
    const u32 lead = lane - sub;
    const u32 lead_lt = (1u << lead) - 1u;
    const u32 gmask = TPK == 1 ? kFull : (((1u << TPK) - 1u) << lead);
    const u32 k = a.k, p = a.p;
    const IT C0 = (IT)a.C[0], C1 = (IT)a.C[1], C2 = (IT)a.C[2], C3 = (IT)a.C[3];
    const IT rootR = (IT)(a.C[4] - 1ull);
    const PT *pre = reinterpret_cast<const PT *>(a.pre);

    u64 kmer[KPT], J[KPT];
    IT L[KPT], R_[KPT];
    u32 I[KPT];
#pragma unroll
    for (int s = 0; s < KPT; s++) { I[s] = kDone; kmer[s] = 0; J[s] = 0; L[s] = 0; R_[s] = 0; }

    // k-mers of this launch; in read mode never more than the row table holds
    const bool read_mode = !a.positions && !a.kmer_list;
    const u64 n_eff = read_mode ? min(a.n_kmers, a.kstart[a.n_rows]) : a.n_kmers;
    const mlp::Bloom bloom{a.bloom_bits, a.bloom_mask, a.bloom_hashes};
    u64 q_next = 0, q_end = 0, row = 0;
    bool more = true;

    for (;;) {
        // ---- refill empty slots from the warp's chunk (work stealing)
#pragma unroll
        for (int s = 0; s < KPT; s++) {
            while (more) {
                const bool need = I[s] == kDone;
                const u32 m = __ballot_sync(kFull, need && sub == 0);
                if (m == 0) break;
                if (q_next >= q_end) {
                    unsigned long long base = 0;
                    if (lane == 0) base = atomicAdd(a.counter, (unsigned long long)a.chunk);
                    base = __shfl_sync(kFull, base, 0);
                    if (base >= n_eff) { more = false; break; }
                    q_next = base;
                    q_end = min((u64)base + a.chunk, n_eff);
                    if (read_mode) row = a.chunk_row[base / a.chunk];
                }
                const u32 take = (u32)min((u64)__popc(m), q_end - q_next);
                const u32 rk_ = __popc(m & lead_lt);
                const bool got = need && rk_ < take;
                u64 rr = row;
                bool skip = false;
                if (got) {
                    const u64 j = q_next + rk_;
                    u64 km;
                    if (a.kmer_list) {
                        km = a.kmer_list[j];
                    } else {
                        u64 pos;
                        if (a.positions) {
                            pos = a.positions[j];
                        } else {
                            while (rr + 1 < a.n_rows && a.kstart[rr + 1] <= j) rr++;
                            pos = a.row_starts[rr] + (j - a.kstart[rr]);
                        }
                        pos = min(pos, a.max_pos);  // a bad offset reads garbage, never out of bounds
                        const u64 b = pos << 1;  // search_kernel.hpp:66-68
                        const u64 w0 = a.words[b >> 6], w1 = a.words[(b >> 6) + 1];
                        const u32 sh = (u32)(b & 63u);
                        km = (w0 << sh) | (shr_clamp(w1, 63u - sh) >> 1);
                    }
                    // learned-Bloom sandwich: answered "absent" only if both reject
                    if (a.logits && __ldg(a.logits + j) < a.tau && !bloom.probe(mlp::kmer_key(km, k))) {
                        skip = true;
                        if (sub == 0) a.answers[j] = ~0ull;
                    }
                    kmer[s] = km;
                    J[s] = j;
                    if (p) {
                        const PT e = pre[km >> (64u - 2u * p)];
                        L[s] = e.x;
                        R_[s] = e.y;
                    } else {
                        L[s] = 0;
                        R_[s] = rootR;
                    }
                    I[s] = skip ? kDone : p;
                }
                if (a.skipped) {
                    const u32 sk = __ballot_sync(kFull, skip && sub == 0);
                    if (lane == 0 && sk) atomicAdd(a.skipped, (unsigned long long)__popc(sk));
                }
                if (read_mode) {
                    const u32 lastm = __ballot_sync(kFull, got && sub == 0 && rk_ == take - 1u);
                    row = __shfl_sync(kFull, rr, __ffs(lastm) - 1);
                }
                q_next += take;
            }
        }
        bool act = false;
#pragma unroll
        for (int s = 0; s < KPT; s++) act |= I[s] != kDone;
        if (!__any_sync(kFull, act)) break;

        // ---- fetch: issue the loads of every stepping slot
        typename R::Fetch F[KPT];
        u32 cc[KPT];
#pragma unroll
        for (int s = 0; s < KPT; s++) {
            cc[s] = 0;
            if (I[s] < k && L[s] <= R_[s]) {
                cc[s] = (u32)((kmer[s] >> (62u - 2u * I[s])) & 3u);
                F[s] = rk.fetch(cc[s], L[s], R_[s], sub);
            }
        }
        // ---- finish: popcounts, interval update, answers
#pragma unroll
        for (int s = 0; s < KPT; s++) {
            if (I[s] < k && L[s] <= R_[s]) {
                const u32 c = cc[s];
                const IT Cc = c == 0 ? C0 : c == 1 ? C1 : c == 2 ? C2 : C3;
                rk.finish(F[s], Cc, L[s], R_[s], sub, gmask);
                I[s]++;
            }
            if (I[s] != kDone && (L[s] > R_[s] || I[s] >= k)) {
                if (sub == 0) a.answers[J[s]] = (L[s] <= R_[s]) ? (u64)L[s] : ~0ull;
                I[s] = kDone;
            }
        }
    }
}


// ------------------------------------------------- queue-fed single-slot form
//
// One k-mer per lane, with the per-k-mer set-up done cooperatively: when its
// queue in shared memory runs low, a whole warp takes the next 32 indices of
// its chunk at once (position, k-mer, presearch entry, prefilter check, all
// 32 lanes active) and enqueues the k-mers that still need steps; a lane
// whose k-mer finishes pops the next entry (ballot + popc).  K-mers settled
// by the presearch entry alone (empty interval, or p = k) are answered
// during the fill and never enqueued.

constexpr u32 kQueue = 64;         // entries per warp (power of two)
constexpr u32 kQueueWarps = 4;     // 128-thread blocks

struct QEntry {
    u64 kmer, j;
    u32 l, r;
};

// Resident blocks per SM the line ranker's queue kernel is compiled for: with C
// read from shared memory it fits 10 (48 registers, no spill).  Measured on the
// large workload, every k-mer searched: 40.1 ms against 42.5 at the compiler's 9
// blocks; 12 blocks (40 registers, 48 bytes of spill) 44.2.
template <class R> struct QueueMinBlocks { static constexpr int value = 1; };
template <int TPK> struct QueueMinBlocks<LinesRankerT<TPK>> { static constexpr int value = 10; };

template <class R>
__global__ void __launch_bounds__(128, QueueMinBlocks<R>::value) search_queue_kernel(const R rk, const SearchArgs a) {
    if (a.runs_dev && runs_usable(*a.runs_dev, a.n_kmers)) return;  // the run walk takes this kernel-contract call
    static_assert(sizeof(typename R::IT) == 4, "the queue form serves 32-bit intervals");
    __shared__ QEntry queue[kQueueWarps][kQueue];
    using PT = uint2;
    const u32 lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const u32 lt = (1u << lane) - 1u;
    const u32 k = a.k, p = a.p;
    __shared__ u32 sC[4];  // C in shared memory: registers kept for the search state
    if (threadIdx.x < 4) sC[threadIdx.x] = (u32)a.C[threadIdx.x];
    __syncthreads();
    const u32 rootR = (u32)(a.C[4] - 1ull);
    const PT *pre = reinterpret_cast<const PT *>(a.pre);
    const bool read_mode = !a.positions && !a.kmer_list;
    const u64 n_eff = read_mode ? min(a.n_kmers, a.kstart[a.n_rows]) : a.n_kmers;
    const mlp::Bloom bloom{a.bloom_bits, a.bloom_mask, a.bloom_hashes};
    QEntry *q = queue[warp];

    // warp-uniform queue / chunk state
    u32 head = 0, tail = 0;
    u64 c_next = 0, c_end = 0, row = 0;
    bool more = true;
    // lane state
    u64 kmer = 0, J = 0;
    u32 L = 0, Rr = 0, I = kDone;

    for (;;) {
        // ---- cooperative fill
        if (more && tail - head < 32u) {
            if (c_next >= c_end) {
                unsigned long long base = 0;
                if (lane == 0) base = atomicAdd(a.counter, (unsigned long long)a.chunk);
                base = __shfl_sync(kFull, base, 0);
                if (base >= n_eff) {
                    more = false;
                } else {
                    c_next = base;
                    c_end = min((u64)base + a.chunk, n_eff);
                    if (read_mode) row = a.chunk_row[base / a.chunk];
                }
            }
            if (more) {
                const u64 j = c_next + lane;
                const bool valid = j < c_end;
                const u32 cnt = (u32)min((u64)32, c_end - c_next);
                u64 km = 0, rr = row;
                u32 l = 0, r = 0;
                bool enq = false;
                if (valid) {
                    if (a.kmer_list) {
                        km = a.kmer_list[j];
                    } else {
                        u64 pos;
                        if (a.positions) {
                            pos = a.positions[j];
                        } else {
                            while (rr + 1 < a.n_rows && a.kstart[rr + 1] <= j) rr++;
                            pos = a.row_starts[rr] + (j - a.kstart[rr]);
                        }
                        pos = min(pos, a.max_pos);
                        const u64 b = pos << 1;  // search_kernel.hpp:66-68
                        const u64 w0 = a.words[b >> 6], w1 = a.words[(b >> 6) + 1];
                        const u32 sh = (u32)(b & 63u);
                        km = (w0 << sh) | (shr_clamp(w1, 63u - sh) >> 1);
                    }
                    bool skip = false;
                    if (a.logits && __ldg(a.logits + j) < a.tau && !bloom.probe(mlp::kmer_key(km, k))) skip = true;
                    if (!skip) {
                        if (p) {
                            const PT e = pre[km >> (64u - 2u * p)];
                            l = e.x;
                            r = e.y;
                        } else {
                            l = 0;
                            r = rootR;
                        }
                    }
                    if (skip || l > r) {
                        a.answers[j] = ~0ull;
                    } else if (p >= k) {
                        a.answers[j] = (u64)l;
                    } else {
                        enq = true;
                    }
                    if (a.skipped) {
                        const u32 sk = __ballot_sync(__activemask(), skip);
                        if (sk && lane == __ffs(__activemask()) - 1) atomicAdd(a.skipped, (unsigned long long)__popc(sk));
                    }
                }
                const u32 em = __ballot_sync(kFull, enq);
                if (enq) {
                    QEntry &e = q[(tail + __popc(em & lt)) & (kQueue - 1)];
                    e.kmer = km;
                    e.j = j;
                    e.l = l;
                    e.r = r;
                }
                tail += __popc(em);
                if (read_mode) row = __shfl_sync(kFull, rr, cnt - 1);
                c_next += cnt;
                __syncwarp();
            }
        }
        // ---- idle lanes pop
        const bool need = I == kDone;
        const u32 m = __ballot_sync(kFull, need);
        const u32 avail = tail - head;
        if (m == kFull && avail == 0 && !more) break;
        const u32 take = min((u32)__popc(m), avail);
        const u32 rank = __popc(m & lt);
        if (need && rank < take) {
            const QEntry &e = q[(head + rank) & (kQueue - 1)];
            kmer = e.kmer;
            J = e.j;
            L = e.l;
            Rr = e.r;
            I = p;
        }
        head += take;
        __syncwarp();
        // ---- one step for every active lane
        if (I != kDone) {
            const u32 c = (u32)((kmer >> (62u - 2u * I)) & 3u);
            const typename R::Fetch f = rk.fetch(c, L, Rr, 0);
            const u32 Cc = sC[c];
            rk.finish(f, Cc, L, Rr, 0, kFull);
            I++;
            if (L > Rr || I >= k) {
                a.answers[J] = (L <= Rr) ? (u64)L : ~0ull;
                I = kDone;
            }
        }
    }
}

// ------------------------------------------------------- absent-run skip
//
// Reads only.  The search of a string s (|s| <= k) ends with a non-empty
// interval exactly when s is a substring of some indexed k-mer: the interval
// holds the nodes whose label ends with s, and every substring of an indexed
// k-mer ends the label of some node (follow predecessor k-mers leftwards;
// a k-mer without one keeps its $-padded prefixes as dummy nodes).  So when
// the search of the k-mer starting at j empties after m letters, x[j, j+m)
// lies in no indexed k-mer, and no k-mer containing it is indexed: the
// k-mers starting at j+m-k .. j are all absent.  An empty presearch entry
// gives m = p.  This kernel walks each run of k-mers of one row from right
// to left and, after a search that fails at m letters, moves left by k-m+1
// k-mers at once and answers ~0 for all of them, so every answer equals the
// reference's per-k-mer search.
//
// With STREAM, a found k-mer's node also gives the node of the k-mer one
// letter to its left by one backward step (stream.cuh) instead of a search
// (presearch entry + k-p rank-pair steps); a failed backward step means that
// k-mer is absent, and the next one is searched again.
//
// Work split: a warp takes 32 windows of kWin consecutive k-mer indices from
// the global cursor and writes zero to their membership words (coalesced).
// Each lane cuts its window at row ends into runs
// and enqueues one run per fill into the warp's shared-memory queue; an idle
// lane pops a run.  Every loop iteration a lane either starts its run's next
// k-mer (backward step, or letters + presearch entry followed by its first
// rank-pair step) or takes one rank-pair step.

// k-mers per window (a multiple of 32; also the granularity of chunk_row and
// the longest run).  Longer runs mean fewer fresh searches per read (one per
// run start, plus one per absent stretch) and a longer walk per lane.
// Measured on the large, batched and pangenome workloads: 128 beats 32 by
// 9-16 % (fewer run starts), 256 starts to lose to the longer tail.  The
// line layout also serves 64 and 256 (KernelShape.window, set by the
// autotuner); the other layouts use 128.
constexpr u32 kWin = 128;

// Answers are written once, a 32-byte sector (4 answers) at a time.  A lane
// settles its run's k-mers strictly right to left and without gaps, so it
// stages the answers of the sector it is in (shared memory, 4 x u64 per
// lane) and stores the sector with one 256-bit streaming store once its
// lowest k-mer is settled; sectors that a long absent stretch covers whole
// go out directly.  Only the sectors at the two ends of a run (row ends)
// are stored answer by answer.  The stores carry the streaming (evict-first)
// hint.  Build option SBWT_ANSWER_WRITE_ONCE=1.  The default form instead
// writes ~0 over a warp's 32 windows when it takes them (coalesced, 256
// bytes a store instruction) and overwrites the found answers later.
// Measured on the large workload (ncu, 60M k-mers, full index): the
// write-once form writes 7.9 instead of 8.7 bytes per k-mer but reads 25.5
// instead of 22.5 and runs 10.3 ms instead of 8.3 ms a launch (more
// instructions per settled k-mer, one store instruction per sector).
#ifndef SBWT_ANSWER_WRITE_ONCE
#define SBWT_ANSWER_WRITE_ONCE 0
#endif

#if SBWT_ANSWER_WRITE_ONCE
__device__ __forceinline__ void st_stream4(u64 *p, u64 a, u64 b, u64 c, u64 d) {
    asm volatile("st.global.cs.v4.u64 [%0], {%1, %2, %3, %4};" ::"l"(p), "l"(a), "l"(b), "l"(c), "l"(d) : "memory");
}
__device__ __forceinline__ void st_stream(u64 *p, u64 a) {
    asm volatile("st.global.cs.u64 [%0], %1;" ::"l"(p), "l"(a) : "memory");
}

// One lane's staged sector, in shared memory: slot[0..3] and, in slot[4],
// the last (rightmost) k-mer of the lane's current run.  Sector boundaries
// are where the answer's address is a multiple of 32 bytes: k-mer x sits in
// slot (x + aoff) & 3, aoff = (answers address / 8) mod 4.  The answer
// pointer is read from the kernel parameters at each use, so the stage
// costs the walk no registers.
__device__ __forceinline__ u32 stage_slot(const u64 *ans, u64 x) {
    return (u32)(x + (reinterpret_cast<uintptr_t>(ans) >> 3)) & 3u;
}

// Store the staged slots s .. top of the sector whose slot s holds k-mer x
// (x is the lowest settled k-mer of that sector).
__device__ __forceinline__ void stage_flush(u64 *ans, const u64 *slot, u64 x, u32 s) {
    const u32 top = min(3u, s + (u32)min(slot[4] - x, (u64)3));
    if (s == 0 && top == 3) {
        const ulonglong2 v0 = *reinterpret_cast<const ulonglong2 *>(slot);
        const ulonglong2 v1 = *reinterpret_cast<const ulonglong2 *>(slot + 2);
        st_stream4(ans + x, v0.x, v0.y, v1.x, v1.y);
    } else {
        for (u32 t = s; t <= top; t++) st_stream(ans + (x - s + t), slot[t]);
    }
}

// k-mer x found with node v; lo = the run's first k-mer.
__device__ __forceinline__ void stage_found(u64 *ans, u64 *slot, u64 x, u64 v, u64 lo) {
    const u32 s = stage_slot(ans, x);
    slot[s] = v;
    if (s == 0 || x == lo) stage_flush(ans, slot, x, s);
}

// k-mers b .. x absent (b >= lo, the run's first k-mer).
__device__ __forceinline__ void stage_absent(u64 *ans, u64 *slot, u64 x, u64 b, u64 lo) {
#pragma unroll 1
    for (;;) {
        const u32 s = stage_slot(ans, x);
        const u64 a = x - min((u64)s, x - b);  // lowest k-mer of this sector in [b, x]
        const u32 sa = s - (u32)(x - a);
        if (sa == 0 && s == 3) {
            st_stream4(ans + a, ~0ull, ~0ull, ~0ull, ~0ull);  // the whole sector
        } else {
            for (u32 t = sa; t <= s; t++) slot[t] = ~0ull;
            if (sa == 0 || a == lo) stage_flush(ans, slot, a, sa);
        }
        if (a == b) break;
        x = a - 1u;
    }
}

#endif  // SBWT_ANSWER_WRITE_ONCE

// Resident 128-thread blocks per SM the run-walking kernel is compiled for
// (a register cap), measured on the large workload: 9 for the line ranker
// (56 registers; 8 blocks at the compiler's 60 registers was 13 % slower),
// 10 for the poppy ranker with basic blocks of up to 256 bits (48 registers);
// the larger poppy blocks keep the compiler's choice (a cap spills there).
// The form with 32-bit k-mer and letter indices (IX = u32, batches below 4G
// letters), with C in shared memory, fits 10 blocks (48 registers, 8 bytes
// of spill).  Measured on the large workload, p = 12: 7.99 ms against 8.26
// at 9 blocks (the 64-bit form: 8.32); with C in registers 10 blocks spilled
// 20 bytes and ran 8.32, 12 blocks (40 registers, 82 bytes) 8.94.
#ifndef SBWT_RUNS_BLOCKS32
#define SBWT_RUNS_BLOCKS32 10
#endif
// The same for the poppy ranker with basic blocks of up to 512 bits (44-46
// registers at 10 blocks, no spill): basic blocks of 512 bits, 10 blocks
// 8.16 / 7.44 ms, 12 blocks 8.32 / 7.68.
#ifndef SBWT_RUNS_BLOCKS32_POPPY
#define SBWT_RUNS_BLOCKS32_POPPY 10
#endif
template <class R, class IX> struct RunsMinBlocks { static constexpr int value = 1; };
template <int TPK> struct RunsMinBlocks<LinesRankerT<TPK>, u64> { static constexpr int value = 9; };
template <int TPK> struct RunsMinBlocks<LinesRankerT<TPK>, u32> { static constexpr int value = SBWT_RUNS_BLOCKS32; };
template <int S, class IX> struct RunsMinBlocks<WideRanker<S>, IX> { static constexpr int value = 8; };
template <int SB, int KIND, class IT, int TPK, class IX> struct RunsMinBlocks<PoppyRanker<SB, KIND, IT, TPK>, IX> {
    static constexpr int value = SB <= 512 && sizeof(IX) == 4 ? SBWT_RUNS_BLOCKS32_POPPY : SB <= 1024 ? 10 : 1;
};
constexpr u32 kStart = 0xfffffffeu; // lane state: start the run's current k-mer

struct RunEntry {
    u64 pos;  // letter offset of the run's last (rightmost) k-mer
    u64 j;    // k-mer index of that k-mer
    u32 len;  // k-mers in the run, 1..WIN
};

// FILTER: the learned prefilter's reject bitmap (a.reject) is read before
// each search from scratch; a rejected k-mer is answered absent unsearched
// (the learned-Bloom sandwich: rejected by the model and by the backup Bloom
// filter over the indexed k-mers the model rejects, so never a present one),
// and the walk goes on with the k-mer to its left.
//
// IX: the type of the k-mer and letter indices the lanes carry (u32 when the
// batch's letters, k-mers and rows stay below 2^32 - 2^16, run32_ok; else u64).
template <class R, bool STREAM, bool FILTER, u32 WIN, class IX>
__global__ void __launch_bounds__(128, RunsMinBlocks<R, IX>::value) search_runs_kernel(const R rk, const SearchArgs a) {
    // kernel contract: the run count is on the device; too few runs and the per-k-mer search takes the call
    const u64 n_rows = a.runs_dev ? *a.runs_dev : a.n_rows;
    if (a.runs_dev && !runs_usable(n_rows, a.n_kmers)) return;
    static_assert(sizeof(typename R::IT) == 4, "the run form serves 32-bit intervals");
    static_assert(WIN % 32 == 0, "windows cover whole bitmap words");
    __shared__ RunEntry queue[kQueueWarps][kQueue];
#if SBWT_ANSWER_WRITE_ONCE
    // per lane: 4 staged answers, the run's last k-mer, pending membership bits
    __shared__ __align__(16) u64 staged[kQueueWarps * 32][6];
#endif
    using PT = uint2;
    const u32 lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const u32 lt = (1u << lane) - 1u;
    const u32 k = a.k, p = a.p;
    // C in shared memory and the cache policy made at each gather: registers kept for the
    // run state, so that the 32-bit form fits 10 blocks per SM
    __shared__ u32 sC[4];
    if (threadIdx.x < 4) sC[threadIdx.x] = (u32)a.C[threadIdx.x];
    __syncthreads();
    const u32 rootR = (u32)(a.C[4] - 1ull);
    const PT *pre = reinterpret_cast<const PT *>(a.pre);
    const IX n_eff = (IX)min(a.n_kmers, a.kstart[n_rows]);
    uint32_t *const member = a.member;
    RunEntry *q = queue[warp];
#if SBWT_ANSWER_WRITE_ONCE
    u64 *const slot = staged[threadIdx.x];
    slot[5] = 0;
#endif

    u32 head = 0, tail = 0;  // warp-uniform
    bool more = true;
    IX pj = 0, pe = 0, prow = 0;  // this lane's window: next k-mer to cut, end, row of pj
    u64 kmer = 0;                 // current k-mer of this lane's run:
    IX J = 0, pos = 0;            // its index and letter offset
    u32 left = 0;                  // k-mers of the run left of J
    u32 L = 0, Rr = 0, I = kDone;
    u32 V = dev::kNoNode;          // STREAM: node of the k-mer right of J (found), or kNoNode
    u32 n_skip = 0;                            // FILTER: k-mers answered from the reject bitmap

    for (;;) {
        // ---- fill: new windows once every lane's window is cut, then one run per lane
        if (more && tail - head < 32u) {
            if (__ballot_sync(kFull, pj < pe) == 0) {
                unsigned long long base = 0;
                if (lane == 0) base = atomicAdd(a.counter, (unsigned long long)(32u * WIN));
                base = __shfl_sync(kFull, base, 0);
                if (base >= n_eff) {
                    more = false;
                } else {
                    const IX end = (IX)min((u64)base + 32u * WIN, (u64)n_eff);
#if !SBWT_ANSWER_WRITE_ONCE
                    if (a.answers)  // NULL: membership bitmap only
                        for (u64 t = base + lane; t < end; t += 32u) a.answers[t] = ~0ull;
#endif
                    pj = (IX)min((u64)base + (u64)lane * WIN, (u64)end);
                    pe = min(pj + WIN, end);
                    if (pj < pe) {
                        prow = a.chunk_row[pj / WIN];
                        if (member)
                            for (IX w = pj / 32u; w < (pe + 31u) / 32u; w++) member[w] = 0u;
                    }
                }
                __syncwarp();
            }
            if (more) {
                const bool emit = pj < pe;
                RunEntry e;
                if (emit) {
                    while (a.kstart[prow + 1] <= pj) prow++;  // rows shorter than k hold no k-mers
                    const IX last = (IX)(min((u64)pe, a.kstart[prow + 1]) - 1u);
                    e.pos = a.row_starts[prow] + (last - a.kstart[prow]);
                    e.j = last;
                    e.len = (u32)(last - pj + 1u);
                    pj = last + 1u;
                }
                const u32 em = __ballot_sync(kFull, emit);
                if (emit) q[(tail + __popc(em & lt)) & (kQueue - 1)] = e;
                tail += __popc(em);
                __syncwarp();
            }
        }
        // ---- idle lanes pop a run
        const bool need = I == kDone;
        const u32 m = __ballot_sync(kFull, need);
        const u32 avail = tail - head;
        if (m == kFull && avail == 0 && !more) break;
        const u32 take = min((u32)__popc(m), avail);
        const u32 rank = __popc(m & lt);
        if (need && rank < take) {
            const RunEntry &e = q[(head + rank) & (kQueue - 1)];
            pos = (IX)e.pos;
            J = (IX)e.j;
            left = e.len - 1u;
            I = kStart;
            V = dev::kNoNode;
#if SBWT_ANSWER_WRITE_ONCE
            slot[4] = e.j;
#endif
        }
        head += take;
        __syncwarp();
        u32 adv = 0;      // k-mers settled at and left of J
        u32 found = ~0u;  // node of k-mer J if found now
        if (I == kStart) {
            if (STREAM && V != dev::kNoNode) {
                // ---- backward step: k-mer J = x[J] . (first k-1 letters of k-mer J+1)
                const u32 letter = (u32)(a.words[pos >> 5] >> (62u - 2u * (u32)(pos & 31u))) & 3u;
                const u32 u = a.sv.back_step(V, letter, a.ef_back, l2_evict_first_policy());
                adv = 1;
                if (u != dev::kNoNode) found = u;
            } else if (FILTER && ((__ldg(a.reject + (J >> 5)) >> (J & 31u)) & 1u)) {
                adv = 1;  // rejected by the prefilter: absent, unsearched
                n_skip++;
            } else {
                // ---- start: letters (search_kernel.hpp:66-68) and presearch entry (:71-82)
                const u64 b = min((u64)pos, a.max_pos) << 1;
                const u64 w0 = a.words[b >> 6], w1 = a.words[(b >> 6) + 1];
                const u32 sh = (u32)(b & 63u);
                kmer = (w0 << sh) | (shr_clamp(w1, 63u - sh) >> 1);
                if (p) {
                    const u64 idx = kmer >> (64u - 2u * p);
                    u32 w = kPreEscape;
                    if (a.pre32) {  // compact entry; the 8-byte one only for intervals too wide for it
                        const u32 c = __ldg(a.pre32 + idx);
                        w = c >> kPreLBits;
                        L = c & ((1u << kPreLBits) - 1u);
                        Rr = L + w - 1u;
                        if (w == 0) L = 1u, Rr = 0u;
                    }
                    if (w == kPreEscape) {
                        const PT e = ld_gather_u32x2(pre + idx, a.ef_pre, l2_evict_first_policy());
                        L = e.x;
                        Rr = e.y;
                    }
                } else {
                    L = 0;
                    Rr = rootR;
                }
                if (L > Rr) {
                    adv = k - p + 1u;  // x[J, J+p) is in no indexed k-mer
                } else if (p >= k) {
                    found = L;
                    adv = 1;
                } else {
                    I = p;
                }
            }
        }
        // ---- one rank-pair step (:84-96)
        if (I < k) {
            const u32 c = (u32)((kmer >> (62u - 2u * I)) & 3u);
            const typename R::Fetch f = rk.fetch(c, L, Rr, 0);
            const u32 Cc = sC[c];
            rk.finish(f, Cc, L, Rr, 0, kFull);
            I++;
            if (L > Rr) {
                adv = k - I + 1u;  // x[J, J+I) is in no indexed k-mer
            } else if (I == k) {
                found = L;
                adv = 1;
            }
        }
#if SBWT_ANSWER_WRITE_ONCE
        if (adv) {
            const u64 lo = J - left;  // the run's first k-mer
            u32 &mword = *reinterpret_cast<u32 *>(slot + 5);  // found bits not yet or-ed into their word
            if (found != ~0u) {
                if (a.answers) stage_found(a.answers, slot, J, (u64)found, lo);
                if (member) {
                    const u32 m = mword | 1u << (J & 31u);
                    if ((J & 31u) == 0 || J == lo) {
                        atomicOr(member + (J >> 5), m);
                        mword = 0;
                    } else {
                        mword = m;
                    }
                }
            } else {
                const u64 b = adv > left ? lo : J - (adv - 1u);  // k-mers b .. J are absent
                if (a.answers) stage_absent(a.answers, slot, J, b, lo);
                if (member && ((b >> 5) != (J >> 5) || (b & 31u) == 0 || b == lo)) {
                    const u32 m = mword;
                    if (m) {
                        atomicOr(member + (J >> 5), m);
                        mword = 0;
                    }
                }
            }
        }
#else
        if (found != ~0u) {
            if (a.answers) a.answers[J] = (u64)found;
            if (member) atomicOr(member + (J >> 5), 1u << (J & 31u));
        }
#endif
        if (adv) {
            if (STREAM) V = found != ~0u ? found : dev::kNoNode;
            if (adv > left) {
                I = kDone;
            } else {
                left -= adv;
                J -= adv;
                pos -= adv;
                I = kStart;
            }
        }
    }
    if (FILTER && a.skipped) {
        for (u32 o = 16; o; o >>= 1) n_skip += __shfl_xor_sync(kFull, n_skip, o);
        if (lane == 0 && n_skip) atomicAdd(a.skipped, (unsigned long long)n_skip);
    }
}

// -------------------------------------------------------------- dispatch

// Launches a search kernel with the L2 access-policy window of the index's
// rank lines, where one applies (l2_window).
template <class K, class R>
int launch_kernel(K kern, u32 blocks, u32 threads, cudaStream_t s, const sbwt_index *ix, const R &rk,
                  const SearchArgs &a) {
    cudaLaunchAttribute attr[1];
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(blocks);
    cfg.blockDim = dim3(threads);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cfg.numAttrs = 0;
    if (l2_window(ix, &attr[0].val.accessPolicyWindow)) {
        attr[0].id = cudaLaunchAttributeAccessPolicyWindow;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
    }
    SBWT_CHECK_CUDA(cudaLaunchKernelEx(&cfg, kern, rk, a));
    return 0;
}

template <class R, int KPT, int TPK>
int launch_one(const R &rk, SearchArgs &a, const sbwt_index *ix, cudaStream_t s, u32 tpb, u32 *blocks_out) {
    auto kern = search_kernel<R, KPT, TPK>;
    int per_sm = 0;
    SBWT_CHECK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, (int)tpb, 0));
    if (per_sm < 1) per_sm = 1;
    const u32 blocks = (u32)per_sm * (u32)ix->num_sms;
    if (blocks_out) *blocks_out = blocks;
    SBWT_CHECK_CUDA(cudaMemsetAsync(a.counter, 0, sizeof(unsigned long long), s));
    SBWT_TRY(launch_kernel(kern, blocks, tpb, s, ix, rk, a));
    return 0;
}

// The batch fits the 32-bit form of the walk: every k-mer index, letter
// offset and row index with a window's slack below 2^32 (a letter offset
// read from a bad row table is still clamped to max_pos).  SBWT_RUN_INDEX64=1
// in the environment when an index is created keeps its walks on the 64-bit
// form.
bool run32_ok(const SearchArgs &a) {
    const u64 lim = (1ull << 32) - (1ull << 16);
    return !a.index64 && a.n_kmers < lim && a.max_pos < lim && a.n_rows < lim;
}

template <class R, u32 WIN, class IX>
auto runs_kernel_ix(const SearchArgs &a) {
    if constexpr (std::is_same<R, LinesRankerT<1>>::value) {  // the prefiltered walk: line layout only
        if (a.reject)
            return a.stream ? search_runs_kernel<R, true, true, WIN, IX> : search_runs_kernel<R, false, true, WIN, IX>;
    }
    return a.stream ? search_runs_kernel<R, true, false, WIN, IX> : search_runs_kernel<R, false, false, WIN, IX>;
}

template <class R, u32 WIN>
auto runs_kernel(const SearchArgs &a) {
    return run32_ok(a) ? runs_kernel_ix<R, WIN, u32>(a) : runs_kernel_ix<R, WIN, u64>(a);
}

template <class R>
int launch_queue(const R &rk, SearchArgs &a, const sbwt_index *ix, cudaStream_t s, u32 *blocks_out) {
    auto kern = search_queue_kernel<R>;
    if (a.runs) {
        if constexpr (std::is_same<R, LinesRankerT<1>>::value) {
            switch (a.chunk) {
            case 64: kern = runs_kernel<R, 64>(a); break;
            case 128: kern = runs_kernel<R, 128>(a); break;
            case 256: kern = runs_kernel<R, 256>(a); break;
            default: return set_error("window must be 64, 128 or 256 k-mers (got %u)", a.chunk);
            }
        } else {
            if (a.chunk != kWin) return set_error("this layout walks windows of %u k-mers", kWin);
            kern = runs_kernel<R, kWin>(a);
        }
    }
    if (a.reject && (!a.runs || !std::is_same<R, LinesRankerT<1>>::value))
        return set_error("the prefiltered search of reads needs the run walk on the line layout");
    int per_sm = 0;
    SBWT_CHECK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 128, 0));
    if (per_sm < 1) per_sm = 1;
    if (ix->shape.blocks_per_sm && (int)ix->shape.blocks_per_sm < per_sm) per_sm = (int)ix->shape.blocks_per_sm;
    const u32 blocks = (u32)per_sm * (u32)ix->num_sms;
    if (blocks_out) *blocks_out = blocks;
    SBWT_CHECK_CUDA(cudaMemsetAsync(a.counter, 0, sizeof(unsigned long long), s));
    SBWT_TRY(launch_kernel(kern, blocks, 128u, s, ix, rk, a));
    return 0;
}

template <int TPK>
int lines_kpt(const sbwt_index *ix, SearchArgs &a, cudaStream_t s, u32 kpt, u32 tpb, u32 *blocks) {
    LinesRankerT<TPK> rk{ix->d_lines, ix->lpc};
    if constexpr (TPK == 1) {
        if (kpt == 0) return launch_queue(rk, a, ix, s, blocks);  // kpt 0: the queue-fed form
    }
    if (kpt == 0) kpt = 1;
    switch (kpt) {
    case 1: return launch_one<LinesRankerT<TPK>, 1, TPK>(rk, a, ix, s, tpb, blocks);
    case 2: return launch_one<LinesRankerT<TPK>, 2, TPK>(rk, a, ix, s, tpb, blocks);
    case 3: return launch_one<LinesRankerT<TPK>, 3, TPK>(rk, a, ix, s, tpb, blocks);
    case 4: return launch_one<LinesRankerT<TPK>, 4, TPK>(rk, a, ix, s, tpb, blocks);
    case 6: return launch_one<LinesRankerT<TPK>, 6, TPK>(rk, a, ix, s, tpb, blocks);
    case 8: return launch_one<LinesRankerT<TPK>, 8, TPK>(rk, a, ix, s, tpb, blocks);
    default: return set_error("kmers_per_thread must be 1, 2, 3, 4, 6 or 8 (got %u)", kpt);
    }
}

template <int S>
int wide_launch(const sbwt_index *ix, SearchArgs &a, cudaStream_t s, const KernelShape &sh, u32 *blocks) {
    if (sh.kpt != 0 || sh.tpk != 1)
        return set_error("the wide-line layouts serve the queue-fed kernels (kmers_per_thread 0, threads_per_kmer 1)");
    WideRanker<S> rk{ix->d_wide, ix->wide_lpc};
    return launch_queue(rk, a, ix, s, blocks);
}

template <int SB, int KIND, class IT, int TPK>
int poppy_kpt(const sbwt_index *ix, SearchArgs &a, cudaStream_t s, u32 kpt, u32 tpb, u32 *blocks) {
    PoppyRanker<SB, KIND, IT, TPK> rk{ix->d_bits, ix->d_L0, ix->d_L12, ix->wpv, ix->l0w, ix->l12w};
    using R = PoppyRanker<SB, KIND, IT, TPK>;
    if constexpr (sizeof(IT) == 4 && TPK == 1) {
        if (kpt == 0) return launch_queue(rk, a, ix, s, blocks);
    }
    if (kpt >= 2 && sizeof(IT) == 4) return launch_one<R, 2, TPK>(rk, a, ix, s, tpb, blocks);
    return launch_one<R, 1, TPK>(rk, a, ix, s, tpb, blocks);
}

template <int SB, int KIND>
int poppy_sb(const sbwt_index *ix, SearchArgs &a, cudaStream_t s, const KernelShape &sh, u32 *blocks) {
    const bool wide = ix->n >= (1ull << 32);
    if (wide) return poppy_kpt<SB, KIND, u64, 1>(ix, a, s, 1, sh.tpb, blocks);
    // the reference's shuffle variants exist for SB 1024 (2 lanes) and 2048 (4 lanes),
    // include/gpu/rank_kernel.hpp:298-407
    if (sh.shuffles && SB == 1024) return poppy_kpt<SB, KIND, u32, 2>(ix, a, s, sh.kpt, sh.tpb, blocks);
    if (sh.shuffles && SB == 2048) return poppy_kpt<SB, KIND, u32, 4>(ix, a, s, sh.kpt, sh.tpb, blocks);
    return poppy_kpt<SB, KIND, u32, 1>(ix, a, s, sh.kpt, sh.tpb, blocks);
}

}  // namespace

bool runs_form(const sbwt_index *ix) {
    const KernelShape &sh = ix->shape;
    if (sh.mode == SBWT_SEARCH_EVERY_KMER || sh.kpt != 0) return false;
    if (sh.layout == SBWT_LAYOUT_LINES) return ix->lines_ok && sh.tpk == 1;
    if (wide_sectors(sh.layout)) return ix->wide_s == wide_sectors(sh.layout) && sh.tpk == 1;
    // poppy: the queue-fed forms are the 32-bit single-lane ones
    return ix->n < (1ull << 32) && !(sh.shuffles && (ix->sb == 1024 || ix->sb == 2048));
}

bool stream_form(const sbwt_index *ix) {
    return runs_form(ix) && ix->shape.mode == SBWT_SEARCH_STREAM && ix->stream_ok;
}

u32 search_chunk(const sbwt_index *ix, bool rows) {
    const KernelShape &sh = ix->shape;
    if (rows && runs_form(ix)) return sh.layout == SBWT_LAYOUT_LINES && sh.window ? sh.window : kWin;
    const u32 groups = 32u / (sh.layout == SBWT_LAYOUT_LINES ? sh.tpk : 1u);
    if (sh.kpt == 0) return 32u * 16u;  // queue-fed form: 16 fills of 32 per chunk
    return groups * std::max(sh.kpt, 1u) * 8u;
}

int launch_search(const sbwt_index *ix, SearchArgs &a, cudaStream_t s, uint32_t *blocks) {
    const KernelShape &sh = ix->shape;
    if (a.n_kmers == 0) return 0;
    if (a.reject && !(a.runs && sh.layout == SBWT_LAYOUT_LINES && sh.tpk == 1 && sh.kpt == 0))
        return set_error("the prefiltered search of reads needs the run walk on the line layout "
                         "(search mode stream or skip, one lane per k-mer, queue-fed)");
    if (sh.tpb == 0 || sh.tpb % 32 != 0 || sh.tpb > 256)
        return set_error("threads_per_block must be a multiple of 32 in [32, 256] (got %u)", sh.tpb);
    if (sh.layout == SBWT_LAYOUT_LINES) {
        if (!ix->lines_ok) return set_error("the line layout is not available for this index");
        switch (sh.tpk) {
        case 1: return lines_kpt<1>(ix, a, s, sh.kpt, sh.tpb, blocks);
        case 2: return lines_kpt<2>(ix, a, s, sh.kpt, sh.tpb, blocks);
        case 4: return lines_kpt<4>(ix, a, s, sh.kpt, sh.tpb, blocks);
        default: return set_error("threads_per_kmer must be 1, 2 or 4 (got %u)", sh.tpk);
        }
    }
    if (wide_sectors(sh.layout)) {
        if (ix->wide_s != wide_sectors(sh.layout)) return set_error("the wide-line layout has not been built");
        return ix->wide_s == 2 ? wide_launch<2>(ix, a, s, sh, blocks) : wide_launch<8>(ix, a, s, sh, blocks);
    }
    if (!ix->poppy_ok) return set_error("the poppy layout has not been built");
    if (ix->kind == SBWT_POPPY) {
        switch (ix->sb) {
        case 256: return poppy_sb<256, 1>(ix, a, s, sh, blocks);
        case 512: return poppy_sb<512, 1>(ix, a, s, sh, blocks);
        case 1024: return poppy_sb<1024, 1>(ix, a, s, sh, blocks);
        case 2048: return poppy_sb<2048, 1>(ix, a, s, sh, blocks);
        default: return poppy_sb<4096, 1>(ix, a, s, sh, blocks);
        }
    }
    switch (ix->sb) {
    case 256: return poppy_sb<256, 2>(ix, a, s, sh, blocks);
    case 512: return poppy_sb<512, 2>(ix, a, s, sh, blocks);
    case 1024: return poppy_sb<1024, 2>(ix, a, s, sh, blocks);
    default: return poppy_sb<2048, 2>(ix, a, s, sh, blocks);
    }
}

}  // namespace sbwt
