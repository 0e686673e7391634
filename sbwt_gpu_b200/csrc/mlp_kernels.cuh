// mlp_kernels.cuh -- device code of the learned prefilter (no reference
// counterpart).  Model: one-hot k-mer (4 x k <= 128 inputs) -> 256 ReLU ->
// 256 ReLU -> 1 logit; BF16 weights and activations, FP32 accumulation on
// the tensor cores (tcgen05.mma kind::f16, accumulators in TMEM).
#pragma once
#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "device.cuh"
#include "tc.cuh"

namespace sbwt {
namespace mlp {

using u32 = uint32_t;
using u64 = uint64_t;
using bf16 = __nv_bfloat16;

constexpr u32 kIn = 128;    // 4 x k one-hot inputs, zero-padded to 128
constexpr u32 kHid = 256;   // hidden width (both layers)
constexpr u32 kTileM = 128; // rows per MMA tile (TMEM lanes)

// Error codes written to the device error flag.
constexpr int kErrGemmWait = 101;
constexpr int kErrInferWait1 = 102;
constexpr int kErrInferWait2 = 103;

__device__ __forceinline__ float bf16_round(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

// 64-bit mixer (splitmix64 finaliser), for sampling and Bloom hashing.
__device__ __host__ __forceinline__ u64 mix64(u64 x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

// The k letters of an MSB-first k-mer word (letter i at bits 63-2i..62-2i).
__device__ __forceinline__ u32 letter(u64 kmer, u32 i) { return (u32)(kmer >> (62u - 2u * i)) & 3u; }

// Canonical key of a k-mer for hashing: only its top 2k bits.
__device__ __forceinline__ u64 kmer_key(u64 kmer, u32 k) { return k == 32 ? kmer : (kmer >> (64u - 2u * k)); }

// ------------------------------------------------------------ Bloom filter

struct Bloom {
    const u32 *bits;  // m bits, m a power of two
    u64 mask;         // m - 1
    u32 hashes;
    __device__ __forceinline__ bool probe(u64 key) const {
        const u64 h = mix64(key ^ 0x5851F42D4C957F2Dull);
        const u64 h1 = h & 0xffffffffull, h2 = (h >> 32) | 1ull;
        for (u32 i = 0; i < hashes; i++) {
            const u64 b = (h1 + i * h2) & mask;
            if (!((__ldg(bits + (b >> 5)) >> (b & 31)) & 1u)) return false;
        }
        return true;
    }
};

__device__ __forceinline__ void bloom_insert(u32 *bits, u64 mask, u32 hashes, u64 key) {
    const u64 h = mix64(key ^ 0x5851F42D4C957F2Dull);
    const u64 h1 = h & 0xffffffffull, h2 = (h >> 32) | 1ull;
    for (u32 i = 0; i < hashes; i++) {
        const u64 b = (h1 + i * h2) & mask;
        atomicOr(bits + (b >> 5), 1u << (b & 31));
    }
}

}  // namespace mlp
}  // namespace sbwt
