// scan.cuh -- device-wide exclusive prefix sum in three launches, built from
// warp scans (__shfl_up_sync) and a shared-memory pass over warp totals.
//
//   phase 1: every block reduces its kItemsPerBlock items -> bsum[block]
//   phase 2: one block scans bsum (exclusive, in place) and writes the total
//   phase 3: every block scans its items again and hands each item its
//            exclusive prefix (bsum[block] + in-block prefix) to an emitter
//
// A functor F supplies `Item load(u64 idx)`, `u64 value(const Item&)` and
// `void emit(u64 idx, u64 prefix, const Item&)`; indices >= n are never
// loaded or emitted.  No inter-block waiting is involved (no spin loops).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace sbwt {
namespace dev {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 4;
constexpr int kItemsPerBlock = kScanThreads * kScanItems;

// Exclusive block scan of one u64 per thread; returns the prefix and writes
// the block total to *total (all threads).
__device__ __forceinline__ uint64_t block_exclusive_scan(uint64_t v, uint64_t *total) {
    __shared__ uint64_t warp_tot[32];
    __shared__ uint64_t tot_s;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nwarps = (blockDim.x + 31) >> 5;
    uint64_t inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint64_t y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += y;
    }
    if (lane == 31) warp_tot[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        uint64_t t = lane < nwarps ? warp_tot[lane] : 0;
        uint64_t ti = t;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint64_t y = __shfl_up_sync(0xffffffffu, ti, o);
            if (lane >= o) ti += y;
        }
        if (lane < nwarps) warp_tot[lane] = ti - t;  // exclusive warp offsets
        if (lane == 31) tot_s = ti;  // lanes >= nwarps add 0: lane 31 holds the total
    }
    __syncthreads();
    const uint64_t res = warp_tot[warp] + inc - v;
    *total = tot_s;
    __syncthreads();
    return res;
}

template <class F>
__global__ void __launch_bounds__(kScanThreads) scan_phase1(F f, uint64_t n, uint64_t *bsum) {
    const uint64_t base = (uint64_t)blockIdx.x * kItemsPerBlock + (uint64_t)threadIdx.x * kScanItems;
    uint64_t s = 0;
#pragma unroll
    for (int t = 0; t < kScanItems; t++)
        if (base + t < n) s += f.value(f.load(base + t));
    uint64_t total;
    block_exclusive_scan(s, &total);
    if (threadIdx.x == 0) bsum[blockIdx.x] = total;
}

static __global__ void __launch_bounds__(1024) scan_phase2(uint64_t *bsum, uint64_t nb, uint64_t *total_out) {
    uint64_t carry = 0;
    for (uint64_t b = 0; b < nb; b += blockDim.x) {
        const uint64_t i = b + threadIdx.x;
        const uint64_t v = i < nb ? bsum[i] : 0;
        uint64_t tot;
        const uint64_t ex = block_exclusive_scan(v, &tot);
        if (i < nb) bsum[i] = carry + ex;
        carry += tot;
    }
    if (threadIdx.x == 0 && total_out) *total_out = carry;
}

template <class F>
__global__ void __launch_bounds__(kScanThreads) scan_phase3(F f, uint64_t n, const uint64_t *bsum) {
    using Item = typename F::Item;
    const uint64_t base = (uint64_t)blockIdx.x * kItemsPerBlock + (uint64_t)threadIdx.x * kScanItems;
    Item it[kScanItems];
    uint64_t v[kScanItems];
    uint64_t s = 0;
#pragma unroll
    for (int t = 0; t < kScanItems; t++) {
        if (base + t < n) {
            it[t] = f.load(base + t);
            v[t] = f.value(it[t]);
        } else {
            v[t] = 0;
        }
        s += v[t];
    }
    uint64_t total;
    uint64_t pre = block_exclusive_scan(s, &total) + bsum[blockIdx.x];
#pragma unroll
    for (int t = 0; t < kScanItems; t++) {
        if (base + t < n) f.emit(base + t, pre, it[t]);
        pre += v[t];
    }
}

inline uint64_t scan_blocks(uint64_t n) { return (n + kItemsPerBlock - 1) / kItemsPerBlock; }

// Runs the three phases on `stream`.  bsum must hold scan_blocks(n) words;
// total (device, optional) receives the sum of all values.
template <class F>
cudaError_t device_scan(const F &f, uint64_t n, uint64_t *bsum, uint64_t *total, cudaStream_t stream) {
    const uint64_t nb = scan_blocks(n);
    if (nb == 0) {
        if (total) return cudaMemsetAsync(total, 0, sizeof(uint64_t), stream);
        return cudaSuccess;
    }
    scan_phase1<F><<<(unsigned)nb, kScanThreads, 0, stream>>>(f, n, bsum);
    scan_phase2<<<1, 1024, 0, stream>>>(bsum, nb, total);
    scan_phase3<F><<<(unsigned)nb, kScanThreads, 0, stream>>>(f, n, bsum);
    return cudaGetLastError();
}

}  // namespace dev
}  // namespace sbwt
