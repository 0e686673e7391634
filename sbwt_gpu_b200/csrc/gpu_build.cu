// gpu_build.cu -- plain-matrix SBWT construction on the GPU.
//
// The reference loads four bit vectors written by an external SBWT tool
// (include/matrix_sbwt.hpp:44-55) and ships no construction code; builder.cpp
// holds this project's host builder.  This file computes the same four
// vectors on the GPU (bit for bit: tests compare the two builders) with the
// same definitions (see builder.cpp):
//   nodes = distinct k-mers + the $-padded prefixes of every source k-mer,
//   colex order by (key, len), key = reversed 2-bit string ($ = 0), len = real
//   letters; column v row c = 1 iff v is the first node of its group (nodes
//   sharing their last k-1 letters) and (those letters).c is a node.
//
// Steps, each a kernel or a CUB primitive:
//   1. runs of ACGT letters: B[i] = i+1 after a non-ACGT letter, i at a
//      sequence start; M = inclusive max-scan of B; the k-mer ending at i is
//      valid iff i + 1 - M[i] >= k.  Its key comes from the 2-bit packed
//      letters (pack_kernel) by a bit reversal;
//   2. radix sort of the keys (2k bits) and unique;
//   3. sources: k-mers whose (k-1)-prefix is no k-mer's (k-1)-suffix (binary
//      search over the sorted keys, whose suffixes are sorted too);
//   4. dummies: k per source, stable-sorted by len then key, deduplicated;
//   5. node order: every k-mer and dummy finds its place by binary search in
//      the other list and is scattered;
//   6. group-first nodes; then each non-root node w sets bit c (its last
//      letter) of the first node of the group (w's first k-1 letters, len-1),
//      found by binary search, with atomicOr.
#include <cub/cub.cuh>

#include <cstdlib>
#include <cstring>
#include <vector>

#include "internal.h"

namespace sbwt {
namespace {

constexpr int kThreads = 256;

inline unsigned blocks_for(u64 n) { return (unsigned)((n + kThreads - 1) / kThreads); }

// device allocations released together
struct DevPool {
    std::vector<void *> ptrs;
    ~DevPool() {
        for (void *p : ptrs) cudaFree(p);
    }
    template <class T> cudaError_t get(T **p, size_t count) {
        *p = nullptr;
        const cudaError_t e = cudaMalloc((void **)p, (count ? count : 1) * sizeof(T));
        if (e == cudaSuccess) ptrs.push_back((void *)*p);
        return e;
    }
    void release(void *p) {
        for (auto &q : ptrs)
            if (q == p) {
                cudaFree(q);
                q = nullptr;
            }
    }
};

__device__ __forceinline__ bool is_acgt(uint8_t ch) {
    switch (ch) {
    case 'A': case 'a': case 'C': case 'c': case 'G': case 'g': case 'T': case 't': return true;
    default: return false;
    }
}

__global__ void breaks_kernel(const uint8_t *__restrict__ letters, u64 n, u64 *__restrict__ B) {
    const u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) B[i] = is_acgt(letters[i]) ? 0ull : i + 1;
}

__global__ void seq_starts_kernel(const u64 *__restrict__ starts, u64 n_seqs, u64 n, u64 *__restrict__ B) {
    const u64 s = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n_seqs) return;
    const u64 i = starts[s];
    if (i < n && B[i] < i) B[i] = i;  // an invalid letter there already gives i + 1
}

// 2-bit groups of a 64-bit word in reverse order (group t -> group 31 - t).
__device__ __forceinline__ u64 reverse_pairs(u64 w) {
    w = __brevll(w);
    return ((w & 0x5555555555555555ull) << 1) | ((w >> 1) & 0x5555555555555555ull);
}

__global__ void keys_kernel(const u64 *__restrict__ words, const u64 *__restrict__ M, u64 n, u32 k,
                            u64 *__restrict__ keys, uint8_t *__restrict__ flags) {
    const u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const bool valid = i + 1 >= M[i] + k;
    flags[i] = valid;
    u64 key = 0;
    if (valid) {
        const u64 b = (i + 1 - k) << 1;  // bit offset of the k-mer's first letter
        const u64 w0 = words[b >> 6], w1 = words[(b >> 6) + 1];
        const u32 sh = (u32)(b & 63u);
        const u64 fwd = (w0 << sh) | (dev::shr_clamp(w1, 63u - sh) >> 1);  // first letter in bits 63..62
        key = reverse_pairs(fwd);  // letter t at bits 2t+1..2t
        if (k < 32) key &= (1ull << (2u * k)) - 1ull;
    }
    keys[i] = key;
}

// first index in a[0, n) with a[idx] >= x
__device__ __forceinline__ u64 lower_bound_u64(const u64 *__restrict__ a, u64 n, u64 x) {
    u64 lo = 0, hi = n;
    while (lo < hi) {
        const u64 mid = (lo + hi) >> 1;
        if (a[mid] < x) lo = mid + 1; else hi = mid;
    }
    return lo;
}

__device__ __forceinline__ u64 upper_bound_u64(const u64 *__restrict__ a, u64 n, u64 x) {
    u64 lo = 0, hi = n;
    while (lo < hi) {
        const u64 mid = (lo + hi) >> 1;
        if (a[mid] <= x) lo = mid + 1; else hi = mid;
    }
    return lo;
}

__global__ void sources_kernel(const u64 *__restrict__ keys, u64 nk, u32 k, uint8_t *__restrict__ src) {
    const u64 x = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= nk) return;
    const u64 mask_km1 = (1ull << (2u * (k - 1u))) - 1ull;
    const u64 pre = keys[x] & mask_km1;
    // keys are sorted, so are their (k-1)-suffixes key >> 2: is pre among them?
    const u64 y = lower_bound_u64(keys, nk, pre << 2);
    src[x] = !(y < nk && (keys[y] >> 2) == pre);
}

__global__ void dummies_kernel(const u64 *__restrict__ sources, u64 ns, u32 k, u64 *__restrict__ dkey,
                               uint8_t *__restrict__ dlen) {
    const u64 t = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ns * k) return;
    const u64 s = t / k;
    const u32 i = (u32)(t - s * k);
    const u64 x = sources[s];
    dkey[t] = i == 0 ? 0ull : ((x & ((1ull << (2u * i)) - 1ull)) << (2u * (k - i)));
    dlen[t] = (uint8_t)i;
}

__global__ void dedup_flags_kernel(const u64 *__restrict__ key, const uint8_t *__restrict__ len, u64 n,
                                   uint8_t *__restrict__ keep) {
    const u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) keep[i] = i == 0 || key[i] != key[i - 1] || len[i] != len[i - 1];
}

__global__ void place_kmers_kernel(const u64 *__restrict__ keys, u64 nk, const u64 *__restrict__ dkey, u64 nd, u32 k,
                                   u64 *__restrict__ nkey, uint8_t *__restrict__ nlen) {
    const u64 x = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= nk) return;
    const u64 key = keys[x];
    const u64 v = x + upper_bound_u64(dkey, nd, key);  // dummies with an equal key sort first (shorter)
    nkey[v] = key;
    nlen[v] = (uint8_t)k;
}

__global__ void place_dummies_kernel(const u64 *__restrict__ dkey, const uint8_t *__restrict__ dlen, u64 nd,
                                     const u64 *__restrict__ keys, u64 nk, u64 *__restrict__ nkey,
                                     uint8_t *__restrict__ nlen) {
    const u64 d = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= nd) return;
    const u64 key = dkey[d];
    const u64 v = d + lower_bound_u64(keys, nk, key);
    nkey[v] = key;
    nlen[v] = dlen[d];
}

__global__ void group_first_kernel(const u64 *__restrict__ nkey, const uint8_t *__restrict__ nlen, u64 n, u32 k,
                                   uint8_t *__restrict__ first, u64 *__restrict__ idx) {
    const u64 v = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    bool f = v == 0;
    if (!f) {
        f = (nkey[v] >> 2) != (nkey[v - 1] >> 2) || min((u32)nlen[v], k - 1u) != min((u32)nlen[v - 1], k - 1u);
    }
    first[v] = f;
    idx[v] = v;
}

__global__ void group_ids_kernel(const u64 *__restrict__ G, u64 ng, const u64 *__restrict__ nkey,
                                 const uint8_t *__restrict__ nlen, u32 k, u64 *__restrict__ gkey,
                                 uint8_t *__restrict__ glen) {
    const u64 g = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= ng) return;
    const u64 v = G[g];
    gkey[g] = nkey[v] >> 2;
    glen[g] = (uint8_t)min((u32)nlen[v], k - 1u);
}

__global__ void edges_kernel(const u64 *__restrict__ nkey, const uint8_t *__restrict__ nlen, u64 n, u32 k,
                             const u64 *__restrict__ G, const u64 *__restrict__ gkey, const uint8_t *__restrict__ glen,
                             u64 ng, unsigned long long *__restrict__ bits, u64 nw,
                             unsigned long long *__restrict__ bad) {
    const u64 w = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (w == 0 || w >= n) return;  // node 0 is the root
    const u64 key = nkey[w];
    const u32 len = nlen[w];
    const u32 c = (u32)(key >> (2u * (k - 1u))) & 3u;
    const u64 mask_km1 = (1ull << (2u * (k - 1u))) - 1ull;
    const u64 tk = key & mask_km1;
    const u32 tl = len - 1u;
    // lexicographic lower bound of (tk, tl) among the group ids
    u64 lo = 0, hi = ng;
    while (lo < hi) {
        const u64 mid = (lo + hi) >> 1;
        const u64 a = gkey[mid];
        if (a < tk || (a == tk && glen[mid] < tl)) lo = mid + 1; else hi = mid;
    }
    if (lo >= ng || gkey[lo] != tk || glen[lo] != tl) {
        atomicAdd(bad, 1ull);
        return;
    }
    const u64 u = G[lo];
    atomicOr(bits + (u64)c * nw + (u >> 6), 1ull << (63u - (u32)(u & 63u)));
}

#define BUILD_TRY(expr)                                                                               \
    do {                                                                                              \
        const cudaError_t e_ = (expr);                                                                \
        if (e_ != cudaSuccess) return set_error("sbwt_build_gpu: %s: %s", #expr, cudaGetErrorString(e_)); \
    } while (0)

// Runs a CUB call twice: size query, then the call with scratch from the pool.
template <class F> cudaError_t cub_call(DevPool &pool, F &&f) {
    size_t bytes = 0;
    cudaError_t e = f(nullptr, bytes);
    if (e != cudaSuccess) return e;
    void *tmp = nullptr;
    e = pool.get((unsigned char **)&tmp, bytes);
    if (e != cudaSuccess) return e;
    e = f(tmp, bytes);
    pool.release(tmp);
    return e;
}

template <class T> T read_back(const T *d) {
    T h{};
    cudaMemcpy(&h, d, sizeof(T), cudaMemcpyDeviceToHost);
    return h;
}

int build_gpu(const uint8_t *seqs, const uint64_t *seq_starts, uint64_t n_seqs, uint32_t k, sbwt_built *out) {
    std::memset(out, 0, sizeof(*out));
    if (k < 3 || k > 32) return set_error("sbwt_build_gpu: k must be in [3, 32], got %u", k);
    const u64 n_letters = n_seqs ? seq_starts[n_seqs] - seq_starts[0] : 0;
    if (n_seqs == 0 || n_letters == 0) return set_error("sbwt_build_gpu: the input holds no k-mer of length %u", k);
    const u64 base = seq_starts[0];
    DevPool pool;
    cudaStream_t s = 0;
    // 1. letters, starts, runs, keys
    uint8_t *d_letters = nullptr;
    u64 *d_starts = nullptr, *d_words = nullptr, *d_B = nullptr, *d_M = nullptr;
    BUILD_TRY(pool.get(&d_letters, n_letters + 16));
    BUILD_TRY(cudaMemcpy(d_letters, seqs + base, n_letters, cudaMemcpyHostToDevice));
    std::vector<u64> rel(n_seqs);
    for (u64 i = 0; i < n_seqs; i++) rel[i] = seq_starts[i] - base;
    BUILD_TRY(pool.get(&d_starts, n_seqs));
    BUILD_TRY(cudaMemcpy(d_starts, rel.data(), n_seqs * sizeof(u64), cudaMemcpyHostToDevice));
    const u64 n_words = (n_letters + 32 + 31) / 32;
    BUILD_TRY(pool.get(&d_words, n_words));
    SBWT_TRY(launch_pack(d_letters, n_letters, d_words, s));
    BUILD_TRY(pool.get(&d_B, n_letters));
    BUILD_TRY(pool.get(&d_M, n_letters));
    breaks_kernel<<<blocks_for(n_letters), kThreads, 0, s>>>(d_letters, n_letters, d_B);
    seq_starts_kernel<<<blocks_for(n_seqs), kThreads, 0, s>>>(d_starts, n_seqs, n_letters, d_B);
    BUILD_TRY(cudaGetLastError());
    pool.release(d_letters);
    BUILD_TRY(cub_call(pool, [&](void *t, size_t &b) {
        return cub::DeviceScan::InclusiveScan(t, b, d_B, d_M, cub::Max(), (int64_t)n_letters, s);
    }));
    pool.release(d_B);
    u64 *d_keys_all = nullptr, *d_keys = nullptr;
    uint8_t *d_flags = nullptr;
    int64_t *d_num = nullptr;
    BUILD_TRY(pool.get(&d_keys_all, n_letters));
    BUILD_TRY(pool.get(&d_flags, n_letters));
    BUILD_TRY(pool.get(&d_num, 4));
    keys_kernel<<<blocks_for(n_letters), kThreads, 0, s>>>(d_words, d_M, n_letters, k, d_keys_all, d_flags);
    BUILD_TRY(cudaGetLastError());
    pool.release(d_M);
    pool.release(d_words);
    BUILD_TRY(pool.get(&d_keys, n_letters));
    BUILD_TRY(cub_call(pool, [&](void *t, size_t &b) {
        return cub::DeviceSelect::Flagged(t, b, d_keys_all, d_flags, d_keys, d_num, (int64_t)n_letters, s);
    }));
    const u64 n_raw = (u64)read_back(d_num);
    pool.release(d_flags);
    if (n_raw == 0) return set_error("sbwt_build_gpu: the input holds no k-mer of length %u", k);
    // 2. sort + unique (d_keys_all is the sort's output buffer)
    BUILD_TRY(cub_call(pool, [&](void *t, size_t &b) {
        return cub::DeviceRadixSort::SortKeys(t, b, d_keys, d_keys_all, (int64_t)n_raw, 0, (int)(2 * k), s);
    }));
    BUILD_TRY(cub_call(pool, [&](void *t, size_t &b) {
        return cub::DeviceSelect::Unique(t, b, d_keys_all, d_keys, d_num, (int64_t)n_raw, s);
    }));
    const u64 nk = (u64)read_back(d_num);
    pool.release(d_keys_all);
    // 3. sources
    uint8_t *d_src = nullptr;
    u64 *d_sources = nullptr;
    BUILD_TRY(pool.get(&d_src, nk));
    BUILD_TRY(pool.get(&d_sources, nk));
    sources_kernel<<<blocks_for(nk), kThreads, 0, s>>>(d_keys, nk, k, d_src);
    BUILD_TRY(cudaGetLastError());
    BUILD_TRY(cub_call(pool, [&](void *t, size_t &b) {
        return cub::DeviceSelect::Flagged(t, b, d_keys, d_src, d_sources, d_num, (int64_t)nk, s);
    }));
    const u64 ns = (u64)read_back(d_num);
    pool.release(d_src);
    // 4. dummies: k per source (i = 0 is the root), sorted by (key, len), deduplicated
    u64 nd = 0;
    u64 *d_dkey = nullptr;
    uint8_t *d_dlen = nullptr;
    const u64 nd_raw = ns ? ns * k : 1;
    {
        u64 *k1 = nullptr, *k2 = nullptr;
        uint8_t *l1 = nullptr, *l2 = nullptr, *keep = nullptr;
        BUILD_TRY(pool.get(&k1, nd_raw));
        BUILD_TRY(pool.get(&k2, nd_raw));
        BUILD_TRY(pool.get(&l1, nd_raw));
        BUILD_TRY(pool.get(&l2, nd_raw));
        BUILD_TRY(pool.get(&keep, nd_raw));
        if (ns) {
            dummies_kernel<<<blocks_for(nd_raw), kThreads, 0, s>>>(d_sources, ns, k, k1, l1);
            BUILD_TRY(cudaGetLastError());
        } else {  // no source k-mer (every (k-1)-prefix continues some k-mer): the root alone
            BUILD_TRY(cudaMemset(k1, 0, sizeof(u64)));
            BUILD_TRY(cudaMemset(l1, 0, 1));
        }
        // LSD: stable by len, then stable by key
        BUILD_TRY(cub_call(pool, [&](void *t, size_t &b) {
            return cub::DeviceRadixSort::SortPairs(t, b, l1, l2, k1, k2, (int64_t)nd_raw, 0, 8, s);
        }));
        BUILD_TRY(cub_call(pool, [&](void *t, size_t &b) {
            return cub::DeviceRadixSort::SortPairs(t, b, k2, k1, l2, l1, (int64_t)nd_raw, 0, (int)(2 * k), s);
        }));
        dedup_flags_kernel<<<blocks_for(nd_raw), kThreads, 0, s>>>(k1, l1, nd_raw, keep);
        BUILD_TRY(cudaGetLastError());
        BUILD_TRY(pool.get(&d_dkey, nd_raw));
        BUILD_TRY(pool.get(&d_dlen, nd_raw));
        BUILD_TRY(cub_call(pool, [&](void *t, size_t &b) {
            return cub::DeviceSelect::Flagged(t, b, k1, keep, d_dkey, d_num, (int64_t)nd_raw, s);
        }));
        nd = (u64)read_back(d_num);
        BUILD_TRY(cub_call(pool, [&](void *t, size_t &b) {
            return cub::DeviceSelect::Flagged(t, b, l1, keep, d_dlen, d_num + 1, (int64_t)nd_raw, s);
        }));
        pool.release(k1);
        pool.release(k2);
        pool.release(l1);
        pool.release(l2);
        pool.release(keep);
    }
    pool.release(d_sources);
    // 5. merged node order
    const u64 n = nk + nd;
    u64 *d_nkey = nullptr;
    uint8_t *d_nlen = nullptr;
    BUILD_TRY(pool.get(&d_nkey, n));
    BUILD_TRY(pool.get(&d_nlen, n));
    place_kmers_kernel<<<blocks_for(nk), kThreads, 0, s>>>(d_keys, nk, d_dkey, nd, k, d_nkey, d_nlen);
    place_dummies_kernel<<<blocks_for(nd), kThreads, 0, s>>>(d_dkey, d_dlen, nd, d_keys, nk, d_nkey, d_nlen);
    BUILD_TRY(cudaGetLastError());
    pool.release(d_keys);
    pool.release(d_dkey);
    pool.release(d_dlen);
    // 6. groups and edge bits
    uint8_t *d_first = nullptr, *d_glen = nullptr;
    u64 *d_idx = nullptr, *d_G = nullptr, *d_gkey = nullptr;
    BUILD_TRY(pool.get(&d_first, n));
    BUILD_TRY(pool.get(&d_idx, n));
    group_first_kernel<<<blocks_for(n), kThreads, 0, s>>>(d_nkey, d_nlen, n, k, d_first, d_idx);
    BUILD_TRY(cudaGetLastError());
    BUILD_TRY(pool.get(&d_G, n));
    BUILD_TRY(cub_call(pool, [&](void *t, size_t &b) {
        return cub::DeviceSelect::Flagged(t, b, d_idx, d_first, d_G, d_num, (int64_t)n, s);
    }));
    const u64 ng = (u64)read_back(d_num);
    pool.release(d_idx);
    pool.release(d_first);
    BUILD_TRY(pool.get(&d_gkey, ng));
    BUILD_TRY(pool.get(&d_glen, ng));
    group_ids_kernel<<<blocks_for(ng), kThreads, 0, s>>>(d_G, ng, d_nkey, d_nlen, k, d_gkey, d_glen);
    const u64 nw = (n + 63) / 64;
    unsigned long long *d_bits = nullptr, *d_bad = nullptr;
    BUILD_TRY(pool.get(&d_bits, 4 * nw));
    BUILD_TRY(pool.get(&d_bad, 1));
    BUILD_TRY(cudaMemset(d_bits, 0, 4 * nw * sizeof(u64)));
    BUILD_TRY(cudaMemset(d_bad, 0, sizeof(u64)));
    edges_kernel<<<blocks_for(n), kThreads, 0, s>>>(d_nkey, d_nlen, n, k, d_G, d_gkey, d_glen, ng, d_bits, nw, d_bad);
    BUILD_TRY(cudaGetLastError());
    BUILD_TRY(cudaDeviceSynchronize());
    if (read_back(d_bad)) return set_error("sbwt_build_gpu: internal error: a node has no predecessor group");
    u64 *bits[4] = {nullptr, nullptr, nullptr, nullptr};
    for (int c = 0; c < 4; c++) {
        bits[c] = (u64 *)std::malloc(nw * sizeof(u64));
        if (!bits[c]) {
            for (int d = 0; d < c; d++) std::free(bits[d]);
            return set_error("sbwt_build_gpu: out of host memory for the bit vectors");
        }
        const cudaError_t e = cudaMemcpy(bits[c], d_bits + (u64)c * nw, nw * sizeof(u64), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) {
            for (int d = 0; d <= c; d++) std::free(bits[d]);
            return set_error("sbwt_build_gpu: copy of the bit vectors failed: %s", cudaGetErrorString(e));
        }
    }
    out->n_bits = n;
    out->n_kmers = nk;
    out->n_dummies = nd;
    out->n_words = nw;
    for (int c = 0; c < 4; c++) out->bits[c] = bits[c];
    return 0;
}

}  // namespace
}  // namespace sbwt

extern "C" int sbwt_build_gpu(const uint8_t *seqs, const uint64_t *seq_starts, uint64_t n_seqs, uint32_t k, int32_t device,
                              sbwt_built *out) {
    sbwt::clear_error();
    if (!out) return sbwt::set_error("sbwt_build_gpu: out is NULL");
    if (!seqs || !seq_starts) return sbwt::set_error("sbwt_build_gpu: NULL input");
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0)
        return sbwt::set_error("no CUDA device is available");
    if (device < 0 || device >= count) return sbwt::set_error("device %d out of range", device);
    SBWT_CHECK_CUDA(cudaSetDevice(device));
    return sbwt::build_gpu(seqs, seq_starts, n_seqs, k, out);
}
