// mlp.cu -- kernels of the learned prefilter (no reference counterpart):
//   * gemm_tn_kernel: D = A * B^T on the tensor cores (tcgen05.mma, BF16 in
//     shared memory, FP32 accumulators in TMEM), used by training;
//   * mlp_infer_kernel: the fused inference pass -- one-hot tile built in
//     shared memory, layer 1 on the tensor cores, bias + ReLU + BF16 written
//     back into TMEM, layer 2 with its A operand read from TMEM, bias + ReLU +
//     the 256 -> 1 dot in the epilogue; weights stay resident in shared
//     memory for the whole (persistent) launch;
//   * training helpers (one-hot batches, transposes, loss, masks, Adam),
//     k-mer sampling from the index by select walks, and the Bloom filter.
#include <algorithm>
#include <cstdio>

#include "internal.h"
#include "mlp.h"
#include "mlp_kernels.cuh"

namespace sbwt {
namespace mlp {

using namespace tc;

// ------------------------------------------------------------------ GEMM

// D[M x N] (+)= A[M x K] * B[N x K]^T for the K range of blockIdx.z; A and B
// row-major BF16, M a multiple of 128, N of BN, K of 64.  128 threads.
template <u32 BN>
__global__ void __launch_bounds__(128) gemm_tn_kernel(const bf16 *__restrict__ A, const bf16 *__restrict__ B,
                                                      float *__restrict__ D, u32 N, u32 K, u32 kps, int atomic,
                                                      int *err) {
    extern __shared__ __align__(1024) uint8_t smem[];
    __shared__ uint64_t bar;
    __shared__ u32 tmem_s;
    uint8_t *sA = smem;
    uint8_t *sB = smem + 128 * 64 * 2;
    const u32 tid = threadIdx.x, warp = tid >> 5, lane = tid & 31u;
    const u32 m0 = blockIdx.x * 128u, n0 = blockIdx.y * BN;
    const u32 kbeg = blockIdx.z * kps, kend = min(K, kbeg + kps);
    constexpr u32 kCols = BN < 32 ? 32 : BN;
    if (warp == 0) tmem_alloc(&tmem_s, kCols);
    if (tid == 0) mbar_init(&bar, 1);
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    const u32 tmem = tmem_s;
    u32 phase = 0;
    bool ok = true;
    for (u32 kb = kbeg; kb < kend && ok; kb += 64) {
        for (u32 i = tid; i < 128u * 8u; i += 128u) {
            const u32 r = i >> 3, kc = i & 7u;
            const uint4 v = *reinterpret_cast<const uint4 *>(A + (size_t)(m0 + r) * K + kb + kc * 8u);
            *reinterpret_cast<uint4 *>(sA + canon_offset(128, r, kc * 8u)) = v;
        }
        for (u32 i = tid; i < BN * 8u; i += 128u) {
            const u32 r = i >> 3, kc = i & 7u;
            const uint4 v = *reinterpret_cast<const uint4 *>(B + (size_t)(n0 + r) * K + kb + kc * 8u);
            *reinterpret_cast<uint4 *>(sB + canon_offset(BN, r, kc * 8u)) = v;
        }
        fence_smem_to_async();
        __syncthreads();
        if (tid == 0) {
            fence_after_sync();
#pragma unroll
            for (u32 s = 0; s < 4; s++) {
                const u64 da = smem_desc(smem_addr(sA) + s * 2u * 128u * 16u, 128u * 16u, 128u);
                const u64 db = smem_desc(smem_addr(sB) + s * 2u * BN * 16u, BN * 16u, 128u);
                mma_ss(tmem, da, db, idesc_bf16(128, BN), kb > kbeg || s > 0);
            }
            mma_commit(&bar);
        }
        const bool got = mbar_wait(&bar, phase, err, kErrGemmWait);
        phase ^= 1u;
        fence_after_sync();
        ok = __syncthreads_and(got);
    }
    if (ok && kend > kbeg) {
        const u32 row = m0 + warp * 32u + lane;
        for (u32 c = 0; c < BN; c += 16) {
            u32 v[16];
            tmem_ld16(tmem + ((warp * 32u) << 16) + c, v);
            tmem_wait_ld();
            float *dst = D + (size_t)row * N + n0 + c;
            if (atomic) {
#pragma unroll
                for (int j = 0; j < 16; j++) atomicAdd(dst + j, __uint_as_float(v[j]));
            } else {
#pragma unroll
                for (int j = 0; j < 16; j += 4)
                    *reinterpret_cast<float4 *>(dst + j) = make_float4(__uint_as_float(v[j]), __uint_as_float(v[j + 1]),
                                                                       __uint_as_float(v[j + 2]), __uint_as_float(v[j + 3]));
            }
        }
    }
    if (!ok && tid == 0) mbar_wait(&bar, phase ^ 1u, err, kErrGemmWait);  // let an MMA still in flight land
    fence_before_sync();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, kCols);
}

// --------------------------------------------------------- fused inference

// W1, W2, the one-hot tile and the per-column-group partial dots: 226 KiB
constexpr u32 kInferThreads = 512;
constexpr u32 kColGroups = kInferThreads / kTileM;  // 4
constexpr u32 kGroupCols = kHid / kColGroups;       // 64
constexpr u32 kInferSmem = kHid * kIn * 2 + kHid * kHid * 2 + kTileM * kIn * 2 + kColGroups * kTileM * 4;

// One-hot chunks q0..q1-1 of row r: chunk q holds inputs 8q..8q+7 = letters
// 2q and 2q+1 (4 one-hot inputs each).
__device__ __forceinline__ void onehot_chunks(uint8_t *tile, u32 R, u32 r, u64 kmer, u32 k, u32 q0, u32 q1) {
#pragma unroll
    for (u32 q = q0; q < q1; q++) {
        const u32 i0 = 2 * q, i1 = 2 * q + 1;
        const u32 c0 = i0 < k ? letter(kmer, i0) : 4u;
        const u32 c1 = i1 < k ? letter(kmer, i1) : 4u;
        uint4 w;
        const u32 one = 0x3F80u;  // bf16 1.0
        w.x = (c0 == 0 ? one : 0u) | ((c0 == 1 ? one : 0u) << 16);
        w.y = (c0 == 2 ? one : 0u) | ((c0 == 3 ? one : 0u) << 16);
        w.z = (c1 == 0 ? one : 0u) | ((c1 == 1 ? one : 0u) << 16);
        w.w = (c1 == 2 ? one : 0u) | ((c1 == 3 ? one : 0u) << 16);
        *reinterpret_cast<uint4 *>(tile + canon_offset(R, r, 8 * q)) = w;
    }
}

// One CTA per SM (226 KiB of shared memory, all 512 TMEM columns), 512
// threads = 16 warps.  The biases and w3 come by value in the parameter
// space (InferBias, read as float4 through the constant cache).  Warp w
// reaches TMEM lanes 32*(w%4)..+31 (rows of the 128-k-mer tile) and handles
// hidden columns 64*(w/4)..+63 of them in both epilogues, so four warps
// share each row and the epilogues run on all 16 warps; layer 2's 256 -> 1
// dot is summed over the four column groups in shared memory.
//
// Pipelined over tiles with the TMEM columns in two halves of 256: tile t
// accumulates in half h (layer 1, then layer 2 over it) and keeps its
// layer-1 activations (layer 2's A operand, BF16 pairs) in the first 128
// columns of the other half.  Once layer 2 of tile t has run, that other
// half is free, so tile t+1's layer-1 MMA runs there while the threads do
// tile t's layer-2 epilogue, and tile t+1's one-hot tile is built while
// tile t's layer-2 MMA runs:
//   epi1(t) -> MMA2(t) || one-hot(t+1) -> MMA1(t+1) || epi2(t) -> epi1(t+1) ...
// Two mbarriers (layer 1, layer 2), each with its own phase.
__device__ __forceinline__ void infer_epi1(u32 tacc, u32 ta2, u32 lane_base, u32 c0, const InferBias &bias) {
    u32 v[4][16];
#pragma unroll
    for (u32 j = 0; j < 4; j++) tmem_ld16(tacc + lane_base + c0 + 16u * j, v[j]);
    tmem_wait_ld();
#pragma unroll
    for (u32 j = 0; j < 4; j++) {
        tmem_tie(v[j]);
        u32 packed[8];
#pragma unroll
        for (int t = 0; t < 16; t += 4) {
            // the same 4 biases for every lane of the warp, from the parameter space
            const float4 bb = *reinterpret_cast<const float4 *>(bias.b1 + c0 + 16u * j + t);
            packed[t / 2] = pack_bf16x2(fmaxf(__uint_as_float(v[j][t]) + bb.x, 0.0f),
                                        fmaxf(__uint_as_float(v[j][t + 1]) + bb.y, 0.0f));
            packed[t / 2 + 1] = pack_bf16x2(fmaxf(__uint_as_float(v[j][t + 2]) + bb.z, 0.0f),
                                            fmaxf(__uint_as_float(v[j][t + 3]) + bb.w, 0.0f));
        }
        tmem_st8(ta2 + lane_base + (c0 + 16u * j) / 2u, packed);
    }
    tmem_wait_st();
}

// Partial dot of one row's 64 layer-2 activations (bias, ReLU, BF16) with w3.
__device__ __forceinline__ float infer_epi2(u32 tacc, u32 lane_base, u32 c0, const InferBias &bias) {
    u32 v[4][16];
#pragma unroll
    for (u32 j = 0; j < 4; j++) tmem_ld16(tacc + lane_base + c0 + 16u * j, v[j]);
    tmem_wait_ld();
    float acc = 0.0f;
#pragma unroll
    for (u32 j = 0; j < 4; j++) {
        tmem_tie(v[j]);
#pragma unroll
        for (int t = 0; t < 16; t += 4) {
            const u32 c = c0 + 16u * j + t;
            const float4 bb = *reinterpret_cast<const float4 *>(bias.b2 + c);
            const float4 ww = *reinterpret_cast<const float4 *>(bias.w3 + c);
            acc = fmaf(bf16_round(fmaxf(__uint_as_float(v[j][t]) + bb.x, 0.0f)), ww.x, acc);
            acc = fmaf(bf16_round(fmaxf(__uint_as_float(v[j][t + 1]) + bb.y, 0.0f)), ww.y, acc);
            acc = fmaf(bf16_round(fmaxf(__uint_as_float(v[j][t + 2]) + bb.z, 0.0f)), ww.z, acc);
            acc = fmaf(bf16_round(fmaxf(__uint_as_float(v[j][t + 3]) + bb.w, 0.0f)), ww.w, acc);
        }
    }
    return acc;
}

__global__ void __launch_bounds__(kInferThreads, 1)
    mlp_infer_kernel(const u64 *__restrict__ kmers, u64 n, u32 k, const bf16 *__restrict__ W1b,
                     const bf16 *__restrict__ W2b, const InferBias bias, const InferOut out, int *err) {
    extern __shared__ __align__(1024) uint8_t smem[];
    __shared__ uint64_t bar1, bar2;
    __shared__ u32 tmem_s;
    uint8_t *sW1 = smem;
    uint8_t *sW2 = smem + kHid * kIn * 2;
    uint8_t *sX = sW2 + kHid * kHid * 2;
    float *sRed = reinterpret_cast<float *>(sX + kTileM * kIn * 2);  // [kColGroups][kTileM] partial dots
    const u32 tid = threadIdx.x, warp = tid >> 5, lane = tid & 31u;
    const u32 quarter = warp & 3u, cg = warp >> 2;
    const u32 trow = quarter * 32u + lane;  // this thread's row of the tile
    const u32 c0 = cg * kGroupCols;         // its first hidden column
    const u32 xr = tid & (kTileM - 1u), xg = tid / kTileM;  // one-hot: row, chunk group
    constexpr u32 kChunks = kIn / 8 / kColGroups;             // 4 of the 16 chunks of a row
    // weights into the canonical K-major layouts (once per launch)
    for (u32 i = tid; i < kHid * (kIn / 8); i += kInferThreads) {
        const u32 r = i / (kIn / 8), kc = i % (kIn / 8);
        *reinterpret_cast<uint4 *>(sW1 + canon_offset(kHid, r, kc * 8)) =
            *reinterpret_cast<const uint4 *>(W1b + (size_t)r * kIn + kc * 8);
    }
    for (u32 i = tid; i < kHid * (kHid / 8); i += kInferThreads) {
        const u32 r = i / (kHid / 8), kc = i % (kHid / 8);
        *reinterpret_cast<uint4 *>(sW2 + canon_offset(kHid, r, kc * 8)) =
            *reinterpret_cast<const uint4 *>(W2b + (size_t)r * kHid + kc * 8);
    }
    if (warp == 0) tmem_alloc(&tmem_s, 512);
    if (tid == 0) {
        mbar_init(&bar1, 1);
        mbar_init(&bar2, 1);
    }
    // the first tile's one-hot tile
    u64 tile = blockIdx.x;
    {
        const u64 row = tile * kTileM + xr;
        onehot_chunks(sX, kTileM, xr, row < n ? kmers[row] : 0ull, k, xg * kChunks, (xg + 1) * kChunks);
    }
    fence_smem_to_async();
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    const u32 T0 = tmem_s;
    const u32 lane_base = (quarter * 32u) << 16;
    const float bias3 = bias.b3;
    auto mma1 = [&](u32 tacc) {  // layer 1: one-hot tile x W1^T into tacc (thread 0, after a thread sync)
        fence_after_sync();
#pragma unroll
        for (u32 s = 0; s < kIn / 16; s++) {
            const u64 da = smem_desc(smem_addr(sX) + s * 2u * kTileM * 16u, kTileM * 16u, 128u);
            const u64 db = smem_desc(smem_addr(sW1) + s * 2u * kHid * 16u, kHid * 16u, 128u);
            mma_ss(tacc, da, db, idesc_bf16(kTileM, kHid), s > 0);
        }
        mma_commit(&bar1);
    };
    u32 ph1 = 0, ph2 = 0;
    bool pend1 = false, pend2 = false;  // an MMA commit outstanding on bar1 / bar2
    bool ok = true;
    u32 half = 0;  // this tile accumulates in columns [256 half, +256), its A2 at the other half
    if (tid == 0) mma1(T0);
    pend1 = true;
    for (;;) {
        const u32 tacc = T0 + 256u * half, ta2 = T0 + 256u * (half ^ 1u);
        // ---- layer 1 done: bias, ReLU, BF16 into the other half's first 128 columns
        bool got = mbar_wait(&bar1, ph1, err, kErrInferWait1);
        ph1 ^= 1u;
        pend1 = false;
        fence_after_sync();
        if (!__syncthreads_and(got)) { ok = false; break; }
        infer_epi1(tacc, ta2, lane_base, c0, bias);
        fence_before_sync();
        __syncthreads();
        if (tid == 0) {
            fence_after_sync();
#pragma unroll
            for (u32 s = 0; s < kHid / 16; s++) {
                const u64 db = smem_desc(smem_addr(sW2) + s * 2u * kHid * 16u, kHid * 16u, 128u);
                mma_ts(tacc, ta2 + s * 8u, db, idesc_bf16(kTileM, kHid), s > 0);
            }
            mma_commit(&bar2);
        }
        pend2 = true;
        // ---- while layer 2 runs: the next tile's one-hot tile (layer 1 has read this one)
        const u64 next = tile + gridDim.x;
        const bool has_next = next * kTileM < n;
        if (has_next) {
            const u64 row = next * kTileM + xr;
            onehot_chunks(sX, kTileM, xr, row < n ? kmers[row] : 0ull, k, xg * kChunks, (xg + 1) * kChunks);
        }
        fence_smem_to_async();
        got = mbar_wait(&bar2, ph2, err, kErrInferWait2);
        ph2 ^= 1u;
        pend2 = false;
        fence_after_sync();
        if (!__syncthreads_and(got)) { ok = false; break; }
        // ---- layer 2 done: the next tile's layer 1 into the other half (this tile's A2 is spent)
        if (has_next) {
            if (tid == 0) mma1(ta2);
            pend1 = true;
        }
        // ---- this tile's layer-2 epilogue while the next tile's layer 1 runs
        sRed[cg * kTileM + trow] = infer_epi2(tacc, lane_base, c0, bias);
        fence_before_sync();
        __syncthreads();
        if (cg == 0) {
            const u64 row = tile * kTileM + trow;
            float sum = 0.0f;
#pragma unroll
            for (u32 g = 0; g < kColGroups; g++) sum += sRed[g * kTileM + trow];
            const float lg = sum + bias3;
            if (out.logits && row < n) out.logits[row] = lg;
            if (out.reject) {
                // the sandwich's decision: rejected by the model at tau and by the backup Bloom filter
                const Bloom bloom{out.bloom_bits, out.bloom_mask, out.bloom_hashes};
                const bool rej = row < n && lg < out.tau && !bloom.probe(kmer_key(kmers[row], k));
                const u32 bits = __ballot_sync(0xffffffffu, rej);
                const u64 first = tile * kTileM + quarter * 32u;  // this warp's 32 rows
                if (lane == 0 && first < n) out.reject[first >> 5] = bits;
            }
        }
        // sRed is reused and this half's columns take the next tile's A2 only after every thread is here
        __syncthreads();
        fence_after_sync();
        if (!has_next) break;
        tile = next;
        half ^= 1u;
    }
    if (!ok && tid == 0) {  // let the MMAs still in flight land before the columns are freed
        if (pend1) mbar_wait(&bar1, ph1, err, kErrInferWait1);
        if (pend2) mbar_wait(&bar2, ph2, err, kErrInferWait2);
    }
    fence_before_sync();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem_s, 512);
}

// ------------------------------------------------------- training helpers

// X[b] = one-hot of k-mer (batch_start + b), Y[b] = its label.
__global__ void onehot_batch_kernel(const u64 *__restrict__ kmers, const uint8_t *__restrict__ labels, u64 n_train,
                                    const unsigned long long *step, u32 batch, u32 k, bf16 *__restrict__ X,
                                    float *__restrict__ Y) {
    const u32 b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= batch) return;
    const u64 start = ((u64)*step * batch) % (n_train - batch + 1);
    const u64 kmer = kmers[start + b];
    Y[b] = (float)labels[start + b];
    uint16_t *row = reinterpret_cast<uint16_t *>(X + (size_t)b * kIn);
    for (u32 i = 0; i < kIn / 4; i++) {
        const u32 c = i < k ? letter(kmer, i) : 4u;
#pragma unroll
        for (u32 j = 0; j < 4; j++) row[4 * i + j] = (c == j) ? 0x3F80 : 0;
    }
}

// dst[c][r] = src[r][c] (bf16, 32x32 tiles through shared memory)
__global__ void transpose_kernel(const bf16 *__restrict__ src, bf16 *__restrict__ dst, u32 R, u32 C) {
    __shared__ bf16 t[32][33];
    const u32 c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
    for (u32 i = threadIdx.y; i < 32; i += blockDim.y) {
        const u32 r = r0 + i, c = c0 + threadIdx.x;
        if (r < R && c < C) t[i][threadIdx.x] = src[(size_t)r * C + c];
    }
    __syncthreads();
    for (u32 i = threadIdx.y; i < 32; i += blockDim.y) {
        const u32 c = c0 + i, r = r0 + threadIdx.x;
        if (r < R && c < C) dst[(size_t)c * R + r] = t[threadIdx.x][i];
    }
}

// H = bf16(ReLU(Z + bias)), Z [rows][256] fp32
__global__ void bias_relu_kernel(const float *__restrict__ Z, const float *__restrict__ bias, bf16 *__restrict__ H,
                                 u64 count) {
    const u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    H[i] = __float2bfloat16_rn(fmaxf(Z[i] + bias[i % kHid], 0.0f));
}

// Per row: h2 = bf16(ReLU(z2 + b2)), logit = h2 . w3 + b3, BCE loss;
// dZ2 = dlogit * w3 * [h2 > 0] (bf16), and the gradients of w3, b3, b2
// (block-reduced, then atomically added).  One warp per row, 8 rows/block.
__global__ void __launch_bounds__(256) head_kernel(const float *__restrict__ Z2, const float *__restrict__ theta,
                                                   const float *__restrict__ Y, u32 batch, bf16 *__restrict__ dZ2,
                                                   float *__restrict__ grad, float *__restrict__ loss_sum,
                                                   const MlpOffsets off) {
    __shared__ float s_dw3[kHid], s_db2[kHid], s_db3;
    const u32 warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    for (u32 i = threadIdx.x; i < kHid; i += blockDim.x) { s_dw3[i] = 0.0f; s_db2[i] = 0.0f; }
    if (threadIdx.x == 0) s_db3 = 0.0f;
    __syncthreads();
    const float *b2 = theta + off.b2, *w3 = theta + off.w3;
    const float b3 = theta[off.b3];
    const u32 r = blockIdx.x * 8 + warp;
    if (r < batch) {
        float h[8], s = 0.0f;
#pragma unroll
        for (int j = 0; j < 8; j++) {
            const u32 c = lane * 8 + j;
            h[j] = bf16_round(fmaxf(Z2[(size_t)r * kHid + c] + b2[c], 0.0f));
            s = fmaf(h[j], w3[c], s);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        const float z = s + b3, y = Y[r];
        // BCE with logits: softplus(z) - y z;  d/dz = sigmoid(z) - y
        const float sp = z > 0 ? z + log1pf(expf(-z)) : log1pf(expf(z));
        const float sig = 1.0f / (1.0f + expf(-z));
        const float dz = (sig - y) / (float)batch;
        if (lane == 0) {
            atomicAdd(loss_sum, (sp - y * z) / (float)batch);
            atomicAdd(&s_db3, dz);
        }
#pragma unroll
        for (int j = 0; j < 8; j++) {
            const u32 c = lane * 8 + j;
            const float g = h[j] > 0.0f ? dz * w3[c] : 0.0f;
            dZ2[(size_t)r * kHid + c] = __float2bfloat16_rn(g);
            atomicAdd(&s_dw3[c], dz * h[j]);
            atomicAdd(&s_db2[c], bf16_round(g));
        }
    }
    __syncthreads();
    for (u32 i = threadIdx.x; i < kHid; i += blockDim.x) {
        atomicAdd(grad + off.w3 + i, s_dw3[i]);
        atomicAdd(grad + off.b2 + i, s_db2[i]);
    }
    if (threadIdx.x == 0) atomicAdd(grad + off.b3, s_db3);
}

// dZ1 = bf16(dH1 * [h1 > 0]); db1 += column sums.  One warp per row.
__global__ void __launch_bounds__(256) relu_grad_kernel(const float *__restrict__ dH1, const bf16 *__restrict__ H1,
                                                        u32 batch, bf16 *__restrict__ dZ1, float *__restrict__ grad,
                                                        const MlpOffsets off) {
    __shared__ float s_db1[kHid];
    const u32 warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    for (u32 i = threadIdx.x; i < kHid; i += blockDim.x) s_db1[i] = 0.0f;
    __syncthreads();
    const u32 r = blockIdx.x * 8 + warp;
    if (r < batch) {
#pragma unroll
        for (int j = 0; j < 8; j++) {
            const u32 c = lane * 8 + j;
            const size_t i = (size_t)r * kHid + c;
            const float g = __bfloat162float(H1[i]) > 0.0f ? dH1[i] : 0.0f;
            const bf16 gb = __float2bfloat16_rn(g);
            dZ1[i] = gb;
            atomicAdd(&s_db1[c], __bfloat162float(gb));
        }
    }
    __syncthreads();
    for (u32 i = threadIdx.x; i < kHid; i += blockDim.x) atomicAdd(grad + off.b1 + i, s_db1[i]);
}

// Adam (Kingma & Ba 2015) over the whole parameter vector, then the BF16
// operand copies of W1 and W2; inputs past 4k of W1 stay zero.
__global__ void adam_kernel(float *__restrict__ theta, const float *__restrict__ grad, float *__restrict__ m,
                            float *__restrict__ v, const unsigned long long *step, u32 count, float lr, u32 k,
                            bf16 *__restrict__ W1b, bf16 *__restrict__ W2b, const MlpOffsets off) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const float t = (float)(*step + 1);
    float g = grad[i];
    if (i < off.b1 && (i % kIn) >= 4 * k) g = 0.0f;  // padded inputs of W1
    const float mi = b1 * m[i] + (1.0f - b1) * g;
    const float vi = b2 * v[i] + (1.0f - b2) * g * g;
    m[i] = mi;
    v[i] = vi;
    const float mh = mi / (1.0f - powf(b1, t)), vh = vi / (1.0f - powf(b2, t));
    const float p = theta[i] - lr * mh / (sqrtf(vh) + eps);
    theta[i] = p;
    if (i < off.b1) W1b[i] = __float2bfloat16_rn(p);
    else if (i >= off.W2 && i < off.b2) W2b[i - off.W2] = __float2bfloat16_rn(p);
}

__global__ void step_kernel(unsigned long long *step, float *loss_hist, const float *loss_sum, u32 hist_every) {
    const unsigned long long s = *step;
    if (hist_every && s % hist_every == 0) loss_hist[s / hist_every] = *loss_sum;
    *step = s + 1;
}

__global__ void to_bf16_kernel(const float *__restrict__ src, bf16 *__restrict__ dst, u32 count) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) dst[i] = __float2bfloat16_rn(src[i]);
}

// ------------------------------------------------- k-mers from the index

// select_c(j): position of the j-th 1 (0-based) of vector c in the LINES
// layout: binary search over the line counts, then within the line.
__device__ u32 line_select(const ulonglong4 *lines_c, u32 lpc, u32 j) {
    u32 lo = 0, hi = lpc - 1;  // last line whose count <= j
    while (lo < hi) {
        const u32 mid = (lo + hi + 1) >> 1;
        const u32 cnt = (u32)(lines_c[mid].x >> 32);
        if (cnt <= j) lo = mid; else hi = mid - 1;
    }
    const ulonglong4 w = lines_c[lo];
    u32 rem = j - (u32)(w.x >> 32);
    const u64 words[4] = {w.x & 0xffffffffull, w.y, w.z, w.w};
    for (u32 wi = 0; wi < 4; wi++) {
        const u32 pc = __popcll(words[wi]);
        if (rem < pc) {
            u64 x = words[wi];
            for (int b = 63; b >= 0; b--) {
                if ((x >> b) & 1ull) {
                    if (rem == 0) return lo * dev::kLineBits + (wi * 64u + (63u - (u32)b)) - 32u;
                    rem--;
                }
            }
        }
        rem -= pc;
    }
    return 0xffffffffu;  // unreachable for j < ones(c)
}

// The k-mer of node v by k select steps back along its incoming edges;
// false for a dummy node (the walk reaches the root first).
__device__ bool node_kmer(const ulonglong4 *lines, u32 lpc, const u64 *C, u32 k, u32 v, u64 &kmer) {
    u64 x = 0;
    for (u32 t = 0; t < k; t++) {
        if (v == 0) return false;
        const u32 c = v < C[1] ? 0u : v < C[2] ? 1u : v < C[3] ? 2u : 3u;
        x |= (u64)c << (62u - 2u * (k - 1u - t));
        v = line_select(lines + (u64)c * lpc, lpc, v - (u32)C[c]);
    }
    kmer = x;
    return true;
}

// Training candidates: with probability n_pos/(n_pos+n_neg) an indexed
// k-mer (a random node, resampled if it is a dummy), else half uniform
// random k-mers and half indexed k-mers with 1-3 substitutions.
__global__ void sample_kernel(const ulonglong4 *lines, u32 lpc, C5 C5v, u32 n_nodes, u32 k, u64 n_pos, u64 n_neg,
                              u64 seed, u64 count, u64 *__restrict__ out) {
    const u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const u64 C[5] = {C5v.c[0], C5v.c[1], C5v.c[2], C5v.c[3], C5v.c[4]};
    u64 h = mix64(seed ^ (i * 0x9E3779B97F4A7C15ull));
    const u64 kmask = k == 32 ? ~0ull : ~((1ull << (64 - 2 * k)) - 1ull);
    const bool pos = (h % (n_pos + n_neg)) < n_pos;
    h = mix64(h);
    if (!pos && (h & 1ull)) {
        out[i] = mix64(h) & kmask;
        return;
    }
    u64 x = 0;
    for (int attempt = 0; attempt < 64; attempt++) {
        h = mix64(h);
        const u32 v = 1u + (u32)(h % (u64)(n_nodes - 1));
        if (node_kmer(lines, lpc, C, k, v, x)) break;
    }
    if (!pos) {
        h = mix64(h);
        const u32 subs = 1u + (u32)(h % 3u);
        for (u32 s = 0; s < subs; s++) {
            h = mix64(h);
            const u32 p = (u32)(h % k);
            const u32 old = letter(x, p);
            const u32 nw = (old + 1u + (u32)((h >> 32) % 3u)) & 3u;
            const u32 sh = 62u - 2u * p;
            x = (x & ~(3ull << sh)) | ((u64)nw << sh);
        }
    }
    out[i] = x;
}

// Every indexed k-mer: node v in [1, n) -> its k-mer, or ~0 for a dummy.
__global__ void enumerate_kernel(const ulonglong4 *lines, u32 lpc, C5 C5v, u32 n_nodes, u32 k, u64 *__restrict__ out) {
    const u32 v = blockIdx.x * blockDim.x + threadIdx.x + 1u;
    if (v >= n_nodes) return;
    const u64 C[5] = {C5v.c[0], C5v.c[1], C5v.c[2], C5v.c[3], C5v.c[4]};
    u64 x;
    out[v - 1] = node_kmer(lines, lpc, C, k, v, x) ? x : ~0ull;
}

// labels[i] = answers[i] found (labels == NULL: only count them, for lists
// longer than any label array).
__global__ void labels_kernel(const u64 *__restrict__ answers, u64 n, uint8_t *__restrict__ labels,
                              unsigned long long *positives) {
    const u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    const bool hit = i < n && answers[i] != ~0ull;
    if (labels && i < n) labels[i] = hit ? 1 : 0;
    const u32 m = __ballot_sync(0xffffffffu, hit);
    if ((threadIdx.x & 31u) == 0 && m) atomicAdd(positives, (unsigned long long)__popc(m));
}

// Indexed k-mers the model rejects (logit < tau) go into the Bloom filter;
// `rejected` counts them (pass 1 counts only, bits == nullptr).
__global__ void bloom_build_kernel(const u64 *__restrict__ kmers, const float *__restrict__ logits, u64 n, float tau,
                                   u32 k, u32 *bits, u64 mask, u32 hashes, unsigned long long *rejected) {
    const u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    const bool rej = i < n && kmers[i] != ~0ull && logits[i] < tau;
    if (rej && bits) bloom_insert(bits, mask, hashes, kmer_key(kmers[i], k));
    const u32 m = __ballot_sync(0xffffffffu, rej);
    if ((threadIdx.x & 31u) == 0 && m) atomicAdd(rejected, (unsigned long long)__popc(m));
}

// Accuracy of the trained model on a labelled set at threshold tau.
__global__ void accuracy_kernel(const float *__restrict__ logits, const uint8_t *__restrict__ labels, u64 n, float tau,
                                unsigned long long *correct) {
    const u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    const bool ok = i < n && ((logits[i] >= tau) == (labels[i] != 0));
    const u32 m = __ballot_sync(0xffffffffu, ok);
    if ((threadIdx.x & 31u) == 0 && m) atomicAdd(correct, (unsigned long long)__popc(m));
}

// ------------------------------------------------------------ launchers

int gemm_tn(const bf16 *A, const bf16 *B, float *D, u32 M, u32 N, u32 K, u32 splits, int *err, cudaStream_t s) {
    if (M % 128 || K % 64 || (N != 128 && N != 256)) return set_error("gemm_tn: unsupported shape %ux%ux%u", M, N, K);
    const u32 ksteps = K / 64;
    splits = std::max(1u, std::min(splits, ksteps));
    const u32 kps = ((ksteps + splits - 1) / splits) * 64;
    splits = (K + kps - 1) / kps;
    const dim3 grid(M / 128, 1, splits);
    const int atomic = splits > 1;
    static bool attr_set = false;  // 48 KiB of dynamic shared memory needs the opt-in
    if (!attr_set) {
        SBWT_CHECK_CUDA(cudaFuncSetAttribute(gemm_tn_kernel<256>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             128 * 64 * 2 + 256 * 64 * 2));
        SBWT_CHECK_CUDA(cudaFuncSetAttribute(gemm_tn_kernel<128>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             128 * 64 * 2 + 128 * 64 * 2));
        attr_set = true;
    }
    if (atomic) SBWT_CHECK_CUDA(cudaMemsetAsync(D, 0, (size_t)M * N * sizeof(float), s));
    if (N == 256) {
        const u32 smem = 128 * 64 * 2 + 256 * 64 * 2;
        gemm_tn_kernel<256><<<grid, 128, smem, s>>>(A, B, D, N, K, kps, atomic, err);
    } else {
        const u32 smem = 128 * 64 * 2 + 128 * 64 * 2;
        gemm_tn_kernel<128><<<grid, 128, smem, s>>>(A, B, D, N, K, kps, atomic, err);
    }
    SBWT_CHECK_CUDA(cudaGetLastError());
    return 0;
}

int infer(const u64 *kmers, u64 n, u32 k, const bf16 *W1b, const bf16 *W2b, const InferBias &bias,
          const InferOut &out, int *err, int num_sms, cudaStream_t s) {
    if (n == 0) return 0;
    // the shared-memory opt-in is a per-device function attribute
    int dev = 0;
    SBWT_CHECK_CUDA(cudaGetDevice(&dev));
    static bool attr_set[kMaxDevicesAttr] = {};
    if (dev < 0 || dev >= kMaxDevicesAttr) return set_error("device %d out of range", dev);
    if (!attr_set[dev]) {
        SBWT_CHECK_CUDA(cudaFuncSetAttribute(mlp_infer_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kInferSmem));
        attr_set[dev] = true;
    }
    const u64 tiles = (n + kTileM - 1) / kTileM;
    const u32 grid = (u32)std::min<u64>(tiles, (u64)num_sms);
    mlp_infer_kernel<<<grid, kInferThreads, kInferSmem, s>>>(kmers, n, k, W1b, W2b, bias, out, err);
    SBWT_CHECK_CUDA(cudaGetLastError());
    return 0;
}

int transpose(const bf16 *src, bf16 *dst, u32 R, u32 C, cudaStream_t s) {
    transpose_kernel<<<dim3((C + 31) / 32, (R + 31) / 32), dim3(32, 8), 0, s>>>(src, dst, R, C);
    SBWT_CHECK_CUDA(cudaGetLastError());
    return 0;
}

}  // namespace mlp
}  // namespace sbwt
