// ingest.cu -- query ingest on the GPU: 2-bit packing, the per-row k-mer
// table, the chunk->row table of the search kernel, and the membership bitmap.
#include "device.cuh"
#include "internal.h"
#include "scan.cuh"

namespace sbwt {
namespace {

using namespace dev;

// Four letters (byte 0 first) -> one byte holding their 2-bit codes, first
// letter in bits 7..6.  A/a->0 C/c->1 G/g->2 T/t->3, any other byte -> 0, as
// the LUT of include/gpu/create_kmer_string.hpp:18-20.  (x | 0x20) folds case;
// only 'C'/'c' become 0x63, 'G'/'g' 0x67, 'T'/'t' 0x74.  The multiply by
// 0x40100401 moves the code of byte i to bits 30-2i..31-2i without carries
// into the top byte.
__device__ __forceinline__ u32 pack4(u32 x) {
    const u32 lo = x | 0x20202020u;
    const u32 codes = (__vcmpeq4(lo, 0x63636363u) & 0x01010101u) | (__vcmpeq4(lo, 0x67676767u) & 0x02020202u) |
                      (__vcmpeq4(lo, 0x74747474u) & 0x03030303u);
    return (codes * 0x40100401u) >> 24;
}

__device__ __forceinline__ u64 pack8x4(const uint4 &v0, const uint4 &v1) {
    return ((u64)pack4(v0.x) << 56) | ((u64)pack4(v0.y) << 48) | ((u64)pack4(v0.z) << 40) |
           ((u64)pack4(v0.w) << 32) | ((u64)pack4(v1.x) << 24) | ((u64)pack4(v1.y) << 16) |
           ((u64)pack4(v1.z) << 8) | (u64)pack4(v1.w);
}

// One thread per output word (32 letters), two 16-byte loads when the word
// lies wholly inside the letters; the word holding the end, and the padding
// words after it, are assembled byte by byte (bytes past n_letters are 0,
// i.e. 'A', as the reference's zero padding, kmer_search.hpp:292-301).
__global__ void pack_kernel(const uint8_t *__restrict__ letters, u64 n_letters, u64 *__restrict__ words, u64 n_words,
                            bool aligned) {
    const u64 w = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= n_words) return;
    const u64 first = w * 32u;
    if (aligned && first + 32u <= n_letters) {
        const uint4 *p = reinterpret_cast<const uint4 *>(letters + first);
        words[w] = pack8x4(__ldg(p), __ldg(p + 1));
        return;
    }
    u64 x = 0;
    for (u32 g = 0; g < 8; g++) {
        u32 v = 0;
        for (u32 b = 0; b < 4; b++) {
            const u64 i = first + g * 4u + b;
            const u32 ch = i < n_letters ? (u32)letters[i] : 0u;
            v |= ch << (8 * b);
        }
        x |= (u64)pack4(v) << (56 - 8 * g);
    }
    words[w] = x;
}

struct KstartScan {
    const u64 *row_starts;
    u64 *kstart;
    u32 k;
    struct Item {
        u64 v;
    };
    __device__ __forceinline__ Item load(u64 r) const {
        const u64 len = row_starts[r + 1] - row_starts[r];
        return Item{len >= k ? len - k + 1ull : 0ull};
    }
    __device__ __forceinline__ u64 value(const Item &it) const { return it.v; }
    __device__ __forceinline__ void emit(u64 r, u64 prefix, const Item &) const { kstart[r] = prefix; }
};

// chunk_row[c] = the row holding k-mer c*chunk: the first r with
// kstart[r+1] > c*chunk (rows without k-mers are skipped).
__global__ void chunk_rows_kernel(const u64 *kstart, u64 n_rows, u64 n_chunks, u32 chunk, u32 *chunk_row) {
    const u64 c = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n_chunks) return;
    const u64 j = c * chunk;
    u64 lo = 0, hi = n_rows;
    while (lo < hi) {
        const u64 mid = (lo + hi) >> 1;
        if (kstart[mid + 1] <= j) lo = mid + 1; else hi = mid;
    }
    chunk_row[c] = (u32)lo;
}

// out[t] = the MSB-first 64-bit window of k-mer j0 + t of a batch of reads
// (search_kernel.hpp:66-68 on the per-row k-mer table), t < count.
__global__ void kmer_list_kernel(const u64 *__restrict__ words, const u64 *__restrict__ row_starts,
                                 const u64 *__restrict__ kstart, const u32 *__restrict__ chunk_row, u32 chunk,
                                 u64 max_pos, u64 j0, u64 count, u64 *__restrict__ out) {
    const u64 t = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count) return;
    const u64 j = j0 + t;
    u64 r = chunk_row[j / chunk];
    while (kstart[r + 1] <= j) r++;  // rows shorter than k hold no k-mers
    const u64 b = min(row_starts[r] + (j - kstart[r]), max_pos) << 1;
    const u64 w0 = words[b >> 6], w1 = words[(b >> 6) + 1];
    const u32 sh = (u32)(b & 63u);
    out[t] = (w0 << sh) | (dev::shr_clamp(w1, 63u - sh) >> 1);
}

__global__ void member_bits_kernel(const u64 *__restrict__ answers, u64 n, uint32_t *__restrict__ bits) {
    const u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    const bool hit = i < n && answers[i] != ~0ull;
    const u32 m = __ballot_sync(0xffffffffu, hit);
    if ((threadIdx.x & 31u) == 0 && (i >> 5) < (n + 31) / 32) bits[i >> 5] = m;
}

}  // namespace

int launch_pack(const uint8_t *d_letters, uint64_t n_letters, uint64_t *d_words, cudaStream_t s) {
    const u64 n_words = (n_letters + 32u + 31u) / 32u;  // ceil((n+32)/32), kmer_search.hpp:294
    const bool aligned = ((uintptr_t)d_letters & 15u) == 0;
    const unsigned blocks = (unsigned)((n_words + 255) / 256);
    pack_kernel<<<blocks, 256, 0, s>>>(d_letters, n_letters, d_words, n_words, aligned);
    SBWT_CHECK_CUDA(cudaGetLastError());
    return 0;
}

uint64_t scan_scratch_words(uint64_t n_items) { return scan_blocks(n_items) + 2; }

int launch_kstart(const uint64_t *d_row_starts, uint64_t n_rows, uint32_t k, uint64_t *d_kstart, uint64_t *d_scan,
                  cudaStream_t s) {
    KstartScan f{d_row_starts, d_kstart, k};
    cudaError_t e = device_scan(f, n_rows, d_scan, d_kstart + n_rows, s);
    if (e != cudaSuccess) return set_error("k-mer table scan failed: %s", cudaGetErrorString(e));
    return 0;
}

int launch_chunk_rows(const uint64_t *d_kstart, uint64_t n_rows, uint64_t n_kmers, uint32_t chunk,
                      uint32_t *d_chunk_row, cudaStream_t s) {
    const u64 n_chunks = (n_kmers + chunk - 1) / chunk;
    if (n_chunks == 0) return 0;
    chunk_rows_kernel<<<(unsigned)((n_chunks + 255) / 256), 256, 0, s>>>(d_kstart, n_rows, n_chunks, chunk,
                                                                         d_chunk_row);
    SBWT_CHECK_CUDA(cudaGetLastError());
    return 0;
}

int launch_kmer_list(const SearchArgs &a, uint64_t j0, uint64_t count, uint64_t *d_out, cudaStream_t s) {
    if (count == 0) return 0;
    kmer_list_kernel<<<(unsigned)((count + 255) / 256), 256, 0, s>>>(a.words, a.row_starts, a.kstart, a.chunk_row,
                                                                     a.chunk, a.max_pos, j0, count, d_out);
    SBWT_CHECK_CUDA(cudaGetLastError());
    return 0;
}

int launch_member_bits(const uint64_t *d_answers, uint64_t n, uint32_t *d_bits, cudaStream_t s) {
    if (n == 0) return 0;
    const u64 threads = (n + 31) / 32 * 32;
    member_bits_kernel<<<(unsigned)((threads + 255) / 256), 256, 0, s>>>(d_answers, n, d_bits);
    SBWT_CHECK_CUDA(cudaGetLastError());
    return 0;
}

}  // namespace sbwt
