// rank_build.cu -- rank structures built on the GPU from the raw vectors.
//
// Replaces the single-threaded CPU pass of RankDataStructures::precount_the_
// structures_based_on_words_in_basicblock (include/rank_data_structures.hpp:
// 142-198, run as four OpenMP tasks in include/matrix_sbwt.hpp:70-110) with
// device-wide warp scans (scan.cuh):
//   * LINES: the per-line 32-bit counts of this engine's search layout;
//   * POPPY: the reference's L0 / L12 words, identical word for word to what
//     the reference computes (including the sentinel L12 entry, :158-161).
#include <cstdio>

#include "device.cuh"
#include "internal.h"
#include "scan.cuh"

namespace sbwt {
namespace {

using namespace dev;

// ------------------------------------------------------------------ LINES

struct LinesBuild {
    const u64 *src;  // one vector, reference word layout
    u64 wsrc;        // readable words
    ulonglong4 *dst;
    struct Item {
        u64 g0, g1, g2, g3;  // 256 bits starting at the block's first position
    };
    __device__ __forceinline__ u64 word(u64 wi) const { return wi < wsrc ? src[wi] : 0ull; }
    __device__ __forceinline__ Item load(u64 li) const {
        const u64 P = li * kLineBits;
        const u64 wi = P >> 6;
        const u32 off = (u32)(P & 63u);  // 0 or 32
        const u64 a0 = word(wi), a1 = word(wi + 1), a2 = word(wi + 2), a3 = word(wi + 3);
        Item it;
        if (off == 0) {
            it.g0 = a0; it.g1 = a1; it.g2 = a2; it.g3 = a3;
        } else {
            const u64 a4 = word(wi + 4);
            it.g0 = (a0 << 32) | (a1 >> 32);
            it.g1 = (a1 << 32) | (a2 >> 32);
            it.g2 = (a2 << 32) | (a3 >> 32);
            it.g3 = (a3 << 32) | (a4 >> 32);
        }
        return it;
    }
    __device__ __forceinline__ u64 value(const Item &it) const {
        return (u64)(__popcll(it.g0) + __popcll(it.g1) + __popcll(it.g2) + __popcll(it.g3 >> 32));
    }
    __device__ __forceinline__ void emit(u64 li, u64 prefix, const Item &it) const {
        ulonglong4 w;
        w.x = (prefix << 32) | (it.g0 >> 32);
        w.y = (it.g0 << 32) | (it.g1 >> 32);
        w.z = (it.g1 << 32) | (it.g2 >> 32);
        w.w = (it.g2 << 32) | (it.g3 >> 32);
        dst[li] = w;
    }
};

// ------------------------------------------------------------- wide lines

// Line li of a wide layout (device.cuh WideShape): the scan value is the
// line's ones; emit reassembles its data bits from the raw vector, adds the
// per-sector counts and writes the S sectors.
template <int S>
struct WideBuild {
    using Sh = WideShape<S>;
    static constexpr u32 kWords = 4u * S;
    const u64 *src;  // one vector, reference word layout
    u64 wsrc;        // readable words
    ulonglong4 *dst;
    struct Item {
        u32 ones;
    };
    __device__ __forceinline__ u64 word(u64 wi) const { return wi < wsrc ? src[wi] : 0ull; }
    // 64 source bits starting at bit position P (MSB-first)
    __device__ __forceinline__ u64 bits64(u64 P) const {
        const u64 wi = P >> 6;
        const u32 off = (u32)(P & 63u);
        const u64 a = word(wi);
        return off ? (a << off) | (word(wi + 1) >> (64u - off)) : a;
    }
    // line word i's data bits (header bits zero)
    __device__ __forceinline__ u64 data_word(u64 li, u32 i) const {
        constexpr u32 H = Sh::kHeaderBits;
        const u64 P0 = li * Sh::kDataBits;
        if (64u * (i + 1) <= H) return 0ull;
        if (64u * i < H) return bits64(P0) >> (H - 64u * i);
        return bits64(P0 + (64u * i - H));  // the data bits end with the line (H + D = 256 S)
    }
    __device__ __forceinline__ Item load(u64 li) const {
        u32 c = 0;
#pragma unroll 4
        for (u32 i = 0; i < kWords; i++) c += __popcll(data_word(li, i));
        return Item{c};
    }
    __device__ __forceinline__ u64 value(const Item &it) const { return it.ones; }
    __device__ __forceinline__ void emit(u64 li, u64 prefix, const Item &) const {
        u64 *out = reinterpret_cast<u64 *>(dst + li * S);
        u64 head[3] = {prefix << 32, 0ull, 0ull};  // the header lies in line words 0..2
        u32 run = 0;                               // ones in the sectors before the current one
#pragma unroll 1
        for (u32 sec = 0; sec < (u32)S; sec++) {
            if (sec) {  // sub[sec] = ones of the data bits in sectors 0..sec-1, 16 bits at line bit 32 + 16 (sec-1)
                const u32 b0 = 32u + 16u * (sec - 1u);
                head[b0 >> 6] |= (u64)run << (48u - (b0 & 63u));
            }
            for (u32 i = 4u * sec; i < 4u * sec + 4u; i++) run += __popcll(data_word(li, i));
        }
        for (u32 i = 0; i < kWords; i++) out[i] = data_word(li, i) | (i < 3 ? head[i] : 0ull);
    }
};

// ------------------------------------------------------------------ POPPY

template <int SB, int KIND>
struct PoppyBuild {
    using S = PoppyShape<SB>;
    const u64 *src;
    const u64 *L0;
    u64 *L12;
    struct Item {
        u32 bb[4];
    };
    __device__ __forceinline__ Item load(u64 s) const {
        Item it;
        const u64 *w = src + s * (u64)(SB / 64);
#pragma unroll
        for (int b = 0; b < 4; b++) {
            u32 c = 0;
#pragma unroll
            for (int j = 0; j < S::kWordsBB; j++) c += __popcll(w[b * S::kWordsBB + j]);
            it.bb[b] = c;
        }
        return it;
    }
    __device__ __forceinline__ u64 value(const Item &it) const {
        return (u64)(it.bb[0] + it.bb[1] + it.bb[2] + it.bb[3]);
    }
    // rank_data_structures.hpp:170-190
    __device__ __forceinline__ void emit(u64 s, u64 prefix, const Item &it) const {
        const u64 h = (s * (u64)SB) >> S::kLogHyper;
        const u64 rel = prefix - L0[h];
        u64 e;
        if (KIND == SBWT_POPPY) {
            const u32 one = (SB == 4096);
            e = (rel << (32 + one)) | ((u64)it.bb[0] << (20 + 2 * one)) | ((u64)it.bb[1] << (10 + one)) |
                (u64)it.bb[2];
        } else if (SB < 2048) {
            e = (rel << 32) | ((u64)it.bb[0] << 20) | ((u64)(it.bb[0] + it.bb[1]) << 10) |
                (u64)(it.bb[0] + it.bb[1] + it.bb[2]);
        } else {
            e = (rel << 32) | ((u64)it.bb[0] << 22) | ((u64)(it.bb[0] + it.bb[1]) << 11) |
                (u64)(it.bb[0] + it.bb[1] + it.bb[2]);
        }
        L12[s] = e;
    }
};

// L0[h] = ones before hyperblock h = scan prefix at superblock h * SPH
// (SPH = 2^logH / SB superblocks, a multiple of kItemsPerBlock).
__global__ void poppy_l0_kernel(const u64 *bsum, u64 nb, const u64 *total, u64 *L0, u64 l0w, u64 sph_blocks) {
    const u64 h = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= l0w) return;
    const u64 b = h * sph_blocks;
    L0[h] = b < nb ? bsum[b] : *total;
}

// The sentinel entry L12[n_sb] = (ones before it, relative to its
// hyperblock) << 32 (<< 33 for SB 4096), rank_data_structures.hpp:158-161.
__global__ void poppy_sentinel_kernel(const u64 *total, const u64 *L0, u64 *L12, u64 n_sb, u64 l0w, u32 sb,
                                      u32 log_hyper) {
    u64 h = (n_sb * (u64)sb) >> log_hyper;
    if (h >= l0w) h = l0w - 1;
    const u32 shift = sb == 4096 ? 33 : 32;
    L12[n_sb] = (*total - L0[h]) << shift;
}

template <int SB, int KIND>
int poppy_one(sbwt_index *ix, int c, cudaStream_t s) {
    using S = PoppyShape<SB>;
    const u64 n_sb = (ix->n + SB - 1) / SB;
    PoppyBuild<SB, KIND> f;
    f.src = ix->d_bits + (u64)c * ix->wpv;
    f.L0 = ix->d_L0 + (u64)c * ix->l0w;
    f.L12 = ix->d_L12 + (u64)c * ix->l12w;
    u64 *bsum = ix->d_scan;
    u64 *total = ix->d_scan + ix->scan_cap - 1;
    const u64 nb = scan_blocks(n_sb);
    if (nb) {
        scan_phase1<PoppyBuild<SB, KIND>><<<(unsigned)nb, kScanThreads, 0, s>>>(f, n_sb, bsum);
        scan_phase2<<<1, 1024, 0, s>>>(bsum, nb, total);
    } else {
        SBWT_CHECK_CUDA(cudaMemsetAsync(total, 0, sizeof(u64), s));
    }
    const u64 sph = (1ull << S::kLogHyper) / SB;
    const u64 sph_blocks = sph / kItemsPerBlock;
    poppy_l0_kernel<<<(unsigned)((ix->l0w + 127) / 128), 128, 0, s>>>(bsum, nb, total, (u64 *)f.L0, ix->l0w,
                                                                      sph_blocks);
    if (nb) scan_phase3<PoppyBuild<SB, KIND>><<<(unsigned)nb, kScanThreads, 0, s>>>(f, n_sb, bsum);
    poppy_sentinel_kernel<<<1, 1, 0, s>>>(total, f.L0, f.L12, n_sb, ix->l0w, SB, S::kLogHyper);
    SBWT_CHECK_CUDA(cudaGetLastError());
    return 0;
}

template <int SB, int KIND>
int poppy_all(sbwt_index *ix, cudaStream_t s) {
    for (int c = 0; c < 4; c++) SBWT_TRY((poppy_one<SB, KIND>(ix, c, s)));
    return 0;
}

}  // namespace

int ensure_scan_scratch(sbwt_index *ix, uint64_t n_items) {
    const size_t need = (size_t)scan_blocks(n_items) + 2;
    if (ix->scan_cap >= need) return 0;
    if (ix->d_scan) cudaFree(ix->d_scan);
    ix->d_scan = nullptr;
    ix->scan_cap = 0;
    SBWT_CHECK_CUDA(cudaMalloc(&ix->d_scan, need * sizeof(u64)));
    ix->scan_cap = need;
    return 0;
}

int build_lines(sbwt_index *ix, cudaStream_t s, uint64_t ones[4]) {
    const u64 nl = (u64)ix->lpc;
    SBWT_TRY(ensure_scan_scratch(ix, nl));
    u64 *totals = nullptr;
    SBWT_CHECK_CUDA(cudaMalloc(&totals, 4 * sizeof(u64)));
    int rc = 0;
    for (int c = 0; c < 4 && rc == 0; c++) {
        LinesBuild f;
        f.src = ix->d_bits + (u64)c * ix->wpv;
        f.wsrc = ix->wpv;
        f.dst = ix->d_lines + (u64)c * nl;
        cudaError_t e = device_scan(f, nl, ix->d_scan, totals + c, s);
        if (e != cudaSuccess) rc = set_error("line build launch failed: %s", cudaGetErrorString(e));
    }
    if (rc == 0) {
        cudaError_t e = cudaMemcpyAsync(ones, totals, 4 * sizeof(u64), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) rc = set_error("line build failed: %s", cudaGetErrorString(e));
    }
    cudaFree(totals);
    return rc;
}

template <int S>
int wide_all(sbwt_index *ix, cudaStream_t s) {
    const u64 nl = ix->wide_lpc;
    SBWT_TRY(ensure_scan_scratch(ix, nl));
    u64 *totals = nullptr;
    SBWT_CHECK_CUDA(cudaMalloc(&totals, 4 * sizeof(u64)));
    int rc = 0;
    for (int c = 0; c < 4 && rc == 0; c++) {
        WideBuild<S> f;
        f.src = ix->d_bits + (u64)c * ix->wpv;
        f.wsrc = ix->wpv;
        f.dst = ix->d_wide + (u64)c * nl * S;
        cudaError_t e = device_scan(f, nl, ix->d_scan, totals + c, s);
        if (e != cudaSuccess) rc = set_error("wide line build launch failed: %s", cudaGetErrorString(e));
    }
    if (rc == 0) {
        const cudaError_t e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) rc = set_error("wide line build failed: %s", cudaGetErrorString(e));
    }
    cudaFree(totals);
    return rc;
}

int build_wide(sbwt_index *ix, uint32_t sectors, cudaStream_t s) {
    if (sectors != 2 && sectors != 8) return set_error("wide lines have 2 or 8 sectors (got %u)", sectors);
    const u64 data = sectors == 2 ? WideShape<2>::kDataBits : WideShape<8>::kDataBits;
    const u64 nl = (ix->n / data + 1 + 7) / 8 * 8;
    if (ix->n >= (1ull << 32) || nl > 0xffffffffull) return set_error("wide lines serve indexes below 2^32 columns");
    ix->gen++;
    if (ix->d_wide) cudaFree(ix->d_wide);
    ix->d_wide = nullptr;
    ix->wide_s = 0;
    SBWT_CHECK_CUDA(cudaMalloc(&ix->d_wide, 4ull * nl * sectors * sizeof(ulonglong4)));
    ix->wide_lpc = (u32)nl;
    SBWT_TRY(sectors == 2 ? wide_all<2>(ix, s) : wide_all<8>(ix, s));
    ix->wide_s = sectors;
    return 0;
}

int build_poppy(sbwt_index *ix, uint32_t sb, int kind, cudaStream_t s) {
    if (!(sb == 256 || sb == 512 || sb == 1024 || sb == 2048 || sb == 4096))
        return set_error("bits_in_superblock must be 256, 512, 1024, 2048 or 4096 (got %u)", sb);
    if (kind != SBWT_POPPY && kind != SBWT_CUM_POPPY)
        return set_error("rank_structure must be poppy (1) or cum_poppy (2) (got %d)", kind);
    if (sb == 4096 && kind != SBWT_POPPY)
        return set_error("Superblock size 4096 bits is supported only in the rank structure version poppy.");
    ix->gen++;
    const u32 log_hyper = sb == 4096 ? 31 : 32;
    const u64 l0w = 1ull + (ix->n >> log_hyper);                  // rank_data_structures.hpp:67
    const u64 l12w = 1ull + ((ix->n + sb - 1ull) / sb * sb) / sb;  // rank_data_structures.hpp:68
    if (ix->d_L0) cudaFree(ix->d_L0);
    if (ix->d_L12) cudaFree(ix->d_L12);
    ix->d_L0 = ix->d_L12 = nullptr;
    ix->poppy_ok = false;
    SBWT_CHECK_CUDA(cudaMalloc(&ix->d_L0, 4 * l0w * sizeof(u64)));
    SBWT_CHECK_CUDA(cudaMalloc(&ix->d_L12, 4 * l12w * sizeof(u64)));
    ix->l0w = l0w;
    ix->l12w = l12w;
    SBWT_TRY(ensure_scan_scratch(ix, l12w));
    int rc;
    if (kind == SBWT_POPPY) {
        switch (sb) {
        case 256: rc = poppy_all<256, SBWT_POPPY>(ix, s); break;
        case 512: rc = poppy_all<512, SBWT_POPPY>(ix, s); break;
        case 1024: rc = poppy_all<1024, SBWT_POPPY>(ix, s); break;
        case 2048: rc = poppy_all<2048, SBWT_POPPY>(ix, s); break;
        default: rc = poppy_all<4096, SBWT_POPPY>(ix, s); break;
        }
    } else {
        switch (sb) {
        case 256: rc = poppy_all<256, SBWT_CUM_POPPY>(ix, s); break;
        case 512: rc = poppy_all<512, SBWT_CUM_POPPY>(ix, s); break;
        case 1024: rc = poppy_all<1024, SBWT_CUM_POPPY>(ix, s); break;
        default: rc = poppy_all<2048, SBWT_CUM_POPPY>(ix, s); break;
        }
    }
    if (rc) return rc;
    SBWT_CHECK_CUDA(cudaStreamSynchronize(s));
    ix->sb = sb;
    ix->kind = kind;
    ix->poppy_ok = true;
    return 0;
}

}  // namespace sbwt
