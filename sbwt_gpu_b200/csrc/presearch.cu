// presearch.cu -- the [l, r] interval table for all 4^p prefixes.
//
// Replaces PreSearch::call_presearch (include/presearch.hpp:32-130) and its
// kernel (include/gpu/presearch_kernel.hpp:19-37).  The reference runs one
// thread per p-mer doing p-1 rank-pair steps from the first letter's
// C-interval (4^p * (p-1) steps).  Here the table is built level by level:
// the entry of x.c (index 4*idx(x) + c, first letter most significant) is one
// step with letter c from the entry of x, so level j+1 costs 4^(j+1) steps and
// the whole table about 4^p * 4/3.  The recurrence and its order are the
// reference's, so every entry -- empty intervals included (l = r + 1, no early
// exit) -- is bit-identical to what the reference writes.
#include <cstdlib>
#include <vector>

#include "device.cuh"
#include "internal.h"
#include "rank.cuh"

namespace sbwt {
namespace {

using namespace dev;

template <class IT> struct Pair;
template <> struct Pair<u32> { using T = uint2; };
template <> struct Pair<u64> { using T = ulonglong2; };

template <class IT>
__global__ void level1_kernel(u64 C0, u64 C1, u64 C2, u64 C3, u64 C4, typename Pair<IT>::T *out) {
    const int c = threadIdx.x;
    if (c >= 4) return;
    const u64 C[5] = {C0, C1, C2, C3, C4};
    typename Pair<IT>::T e;
    e.x = (IT)C[c];
    e.y = (IT)(C[c + 1] - 1ull);  // presearch_kernel.hpp:25-26
    out[c] = e;
}

template <class R>
__global__ void level_kernel(R rk, u64 C0, u64 C1, u64 C2, u64 C3, const typename Pair<typename R::IT>::T *parent,
                             typename Pair<typename R::IT>::T *out, u64 count) {
    using IT = typename R::IT;
    const u64 t = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count) return;
    const typename Pair<IT>::T e = parent[t >> 2];
    const u32 c = (u32)(t & 3u);
    const u64 Cc = c == 0 ? C0 : c == 1 ? C1 : c == 2 ? C2 : C3;
    IT l = e.x, r = e.y;
    rk.step(c, (IT)Cc, l, r);  // presearch_kernel.hpp:29-34
    typename Pair<IT>::T o;
    o.x = l;
    o.y = r;
    out[t] = o;
}

template <class R>
int run_levels(sbwt_index *ix, const R &rk, u32 p, void *table, cudaStream_t s) {
    using PT = typename Pair<typename R::IT>::T;
    PT *scratch = nullptr;
    const u64 half = p >= 2 ? (1ull << (2 * (p - 1))) : 0;  // largest intermediate level
    if (p >= 2) SBWT_CHECK_CUDA(cudaMalloc(&scratch, 2 * half * sizeof(PT)));
    PT *bufs[2] = {scratch, scratch ? scratch + half : nullptr};
    PT *prev = (p == 1) ? (PT *)table : bufs[0];
    level1_kernel<typename R::IT><<<1, 32, 0, s>>>(ix->C[0], ix->C[1], ix->C[2], ix->C[3], ix->C[4], prev);
    for (u32 j = 2; j <= p; j++) {
        const u64 count = 1ull << (2 * j);
        PT *dst = (j == p) ? (PT *)table : bufs[(j - 1) & 1];
        const unsigned blocks = (unsigned)((count + 255) / 256);
        level_kernel<R><<<blocks, 256, 0, s>>>(rk, ix->C[0], ix->C[1], ix->C[2], ix->C[3], prev, dst, count);
        prev = dst;
    }
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (scratch) cudaFree(scratch);
    if (e != cudaSuccess) return set_error("presearch failed: %s", cudaGetErrorString(e));
    return 0;
}

template <int SB, int KIND>
int run_poppy_levels(sbwt_index *ix, u32 p, void *table, cudaStream_t s) {
    if (ix->pre64) {
        PoppyRanker<SB, KIND, u64> rk{ix->d_bits, ix->d_L0, ix->d_L12, ix->wpv, ix->l0w, ix->l12w};
        return run_levels(ix, rk, p, table, s);
    }
    PoppyRanker<SB, KIND, u32> rk{ix->d_bits, ix->d_L0, ix->d_L12, ix->wpv, ix->l0w, ix->l12w};
    return run_levels(ix, rk, p, table, s);
}

__global__ void pre_compact_kernel(const uint2 *__restrict__ pre, u64 count, uint32_t *__restrict__ out) {
    const u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) {
        const uint2 e = pre[i];
        out[i] = dev::pre_compact(e.x, e.y);
    }
}

// The compact table of the run walk is built when the index is small enough
// for it and the autotuner chose it, or (no choice made) the environment
// variable SBWT_PRESEARCH_COMPACT is "1".
// Measured on the large workload (p = 12, 100.2M columns): 8.375 ms per
// search against 8.317 ms with the 8-byte entries alone, so it is off by
// default.
bool compact_presearch(const sbwt_index *ix) {
    if (ix->n >= dev::kPreMaxColumns) return false;
    if (ix->compact_pre >= 0) return ix->compact_pre == 1;  // the autotuner's choice
    const char *e = std::getenv("SBWT_PRESEARCH_COMPACT");
    return e && e[0] == '1' && e[1] == 0;
}

}  // namespace

int run_presearch(sbwt_index *ix, uint32_t p, cudaStream_t s) {
    ix->gen++;
    if (ix->d_pre) cudaFree(ix->d_pre);
    ix->d_pre = nullptr;
    if (ix->d_pre32) cudaFree(ix->d_pre32);
    ix->d_pre32 = nullptr;
    ix->p = 0;
    if (p == 0) return 0;  // search without presearch (parameters.hpp:555, search_kernel.hpp:79-81)
    if (p > ix->k) return set_error("presearch depth p=%u exceeds k=%u", p, ix->k);
    if (p > 16) return set_error("presearch depth p=%u is larger than 16 (a 4^p-entry table)", p);
    ix->pre64 = ix->n >= (1ull << 32);
    const size_t esz = ix->pre64 ? sizeof(ulonglong2) : sizeof(uint2);
    const u64 count = 1ull << (2 * p);
    SBWT_CHECK_CUDA(cudaMalloc(&ix->d_pre, count * esz));
    int rc;
    if (ix->lines_ok) {
        LinesRanker rk{ix->d_lines, ix->lpc};
        rc = run_levels(ix, rk, p, ix->d_pre, s);
    } else if (ix->poppy_ok) {
        const int kind = ix->kind;
        switch (ix->sb) {
        case 256: rc = kind == SBWT_POPPY ? run_poppy_levels<256, 1>(ix, p, ix->d_pre, s)
                                          : run_poppy_levels<256, 2>(ix, p, ix->d_pre, s); break;
        case 512: rc = kind == SBWT_POPPY ? run_poppy_levels<512, 1>(ix, p, ix->d_pre, s)
                                          : run_poppy_levels<512, 2>(ix, p, ix->d_pre, s); break;
        case 1024: rc = kind == SBWT_POPPY ? run_poppy_levels<1024, 1>(ix, p, ix->d_pre, s)
                                           : run_poppy_levels<1024, 2>(ix, p, ix->d_pre, s); break;
        case 2048: rc = kind == SBWT_POPPY ? run_poppy_levels<2048, 1>(ix, p, ix->d_pre, s)
                                           : run_poppy_levels<2048, 2>(ix, p, ix->d_pre, s); break;
        default: rc = run_poppy_levels<4096, 1>(ix, p, ix->d_pre, s); break;
        }
    } else {
        rc = set_error("presearch: the index has no rank structure");
    }
    if (rc == 0 && !ix->pre64 && compact_presearch(ix)) {
        const cudaError_t e = cudaMalloc(&ix->d_pre32, count * sizeof(uint32_t));
        if (e != cudaSuccess) {
            rc = set_error("presearch: %s", cudaGetErrorString(e));
        } else {
            pre_compact_kernel<<<(unsigned)((count + 255) / 256), 256, 0, s>>>(
                static_cast<const uint2 *>(ix->d_pre), count, ix->d_pre32);
            const cudaError_t e2 = cudaGetLastError();
            if (e2 != cudaSuccess) rc = set_error("presearch: %s", cudaGetErrorString(e2));
        }
    }
    if (rc) {
        cudaFree(ix->d_pre);
        cudaFree(ix->d_pre32);
        ix->d_pre = nullptr;
        ix->d_pre32 = nullptr;
        return rc;
    }
    ix->p = p;
    return 0;
}

int export_presearch(const sbwt_index *ix, uint64_t *lefts, uint64_t *rights, uint64_t count) {
    if (ix->p == 0 || !ix->d_pre) return set_error("the index has no presearch table");
    const u64 want = 1ull << (2 * ix->p);
    if (count != want) return set_error("presearch export: count must be 4^p = %llu", (unsigned long long)want);
    if (ix->pre64) {
        std::vector<ulonglong2> h(count);
        SBWT_CHECK_CUDA(cudaMemcpy(h.data(), ix->d_pre, count * sizeof(ulonglong2), cudaMemcpyDeviceToHost));
        for (u64 i = 0; i < count; i++) { lefts[i] = h[i].x; rights[i] = h[i].y; }
    } else {
        std::vector<uint2> h(count);
        SBWT_CHECK_CUDA(cudaMemcpy(h.data(), ix->d_pre, count * sizeof(uint2), cudaMemcpyDeviceToHost));
        for (u64 i = 0; i < count; i++) { lefts[i] = h[i].x; rights[i] = h[i].y; }
    }
    return 0;
}

}  // namespace sbwt
