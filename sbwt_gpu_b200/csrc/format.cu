// format.cu -- the reference's answer text on the GPU.
//
// Replaces ResultsPersister::save_results_to_file (include/epicseq/
// results_persister.hpp:82-95): per read, each answer as a signed 64-bit
// decimal followed by one space, then '\n' (a read without k-mers gives an
// empty line).  sbwt_format_answers (queries.cpp) writes the same bytes on
// the host.
//
// Layout: item j = (newlines of the rows that end right before k-mer j) +
// (answer j's digits + ' ').  x[j] = item length (rows ending at j are
// counted by one atomicAdd per row), an exclusive scan gives each item's
// offset, and one thread per k-mer writes its item; the newlines of the rows
// ending after the last k-mer close the text.
#include <cub/cub.cuh>

#include "internal.h"

namespace sbwt {
namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ u32 decimal_len(u64 v) {
    const bool neg = (int64_t)v < 0;
    u64 m = neg ? 0ull - v : v;
    u32 d = 1;
    while (m >= 10ull) {
        m /= 10ull;
        d++;
    }
    return d + (neg ? 1u : 0u);
}

__global__ void item_len_kernel(const u64 *__restrict__ answers, u64 n, u64 *__restrict__ x) {
    const u64 j = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (j < n) x[j] = decimal_len(answers[j]) + 1u;
    if (j == n) x[n] = 0;
}

// Row r's newline goes before k-mer kstart[r+1] (or after the last k-mer).
__global__ void row_ends_kernel(const u64 *__restrict__ kstart, u64 n_rows, u64 n, u64 *__restrict__ x,
                                unsigned long long *__restrict__ tail_rows) {
    const u64 r = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n_rows) return;
    const u64 j = kstart[r + 1];
    if (j < n) atomicAdd((unsigned long long *)(x + j), 1ull);
    else atomicAdd(tail_rows, 1ull);
}

__global__ void write_items_kernel(const u64 *__restrict__ answers, u64 n, const u64 *__restrict__ off,
                                   char *__restrict__ out, const unsigned long long *__restrict__ tail_rows) {
    const u64 j = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (j == n) {  // the rows after the last k-mer
        const u64 t = *tail_rows;
        for (u64 i = 0; i < t; i++) out[off[n] + i] = '\n';
        return;
    }
    if (j > n) return;
    const u64 v = answers[j];
    const u32 len = decimal_len(v);
    u64 o = off[j];
    const u64 nl = off[j + 1] - o - len - 1u;
    for (u64 i = 0; i < nl; i++) out[o++] = '\n';
    const bool neg = (int64_t)v < 0;
    u64 m = neg ? 0ull - v : v;
    char *p = out + o + len;
    *p = ' ';
    do {
        *--p = (char)('0' + (int)(m % 10ull));
        m /= 10ull;
    } while (m);
    if (neg) *--p = '-';
}

}  // namespace
}  // namespace sbwt

using namespace sbwt;

extern "C" int sbwt_format_answers_device(const uint64_t *d_row_starts, uint64_t n_rows, uint32_t k,
                                          const uint64_t *d_answers, uint64_t n_kmers, char *d_out, uint64_t cap,
                                          uint64_t *bytes, void *stream) {
    clear_error();
    if (!bytes) return set_error("bytes is NULL");
    *bytes = 0;
    if (!d_row_starts || (!d_answers && n_kmers)) return set_error("NULL device pointer");
    if (n_rows == 0) return 0;
    const cudaStream_t s = (cudaStream_t)stream;
    u64 *x = nullptr, *kstart = nullptr, *scan = nullptr;
    unsigned long long *tail = nullptr;
    void *tmp = nullptr;
    int rc = 0;
    cudaError_t e = cudaMalloc(&x, (n_kmers + 1) * sizeof(u64));
    if (e == cudaSuccess) e = cudaMalloc(&kstart, (n_rows + 1) * sizeof(u64));
    if (e == cudaSuccess) e = cudaMalloc(&scan, scan_scratch_words(n_rows) * sizeof(u64));
    if (e == cudaSuccess) e = cudaMalloc(&tail, sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMemsetAsync(tail, 0, sizeof(unsigned long long), s);
    if (e != cudaSuccess) {
        rc = set_error("sbwt_format_answers_device: %s", cudaGetErrorString(e));
    } else if ((rc = launch_kstart(d_row_starts, n_rows, k, kstart, scan, s)) == 0) {
        u64 kmers_in_rows = 0;
        e = cudaMemcpyAsync(&kmers_in_rows, kstart + n_rows, sizeof(u64), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) {
            rc = set_error("sbwt_format_answers_device: %s", cudaGetErrorString(e));
        } else if (kmers_in_rows != n_kmers) {
            rc = set_error("the rows hold %llu k-mers, not %llu", (unsigned long long)kmers_in_rows,
                           (unsigned long long)n_kmers);
        } else {
            const unsigned bk = (unsigned)((n_kmers + 1 + kThreads - 1) / kThreads);
            const unsigned br = (unsigned)((n_rows + kThreads - 1) / kThreads);
            item_len_kernel<<<bk, kThreads, 0, s>>>(d_answers, n_kmers, x);
            row_ends_kernel<<<br, kThreads, 0, s>>>(kstart, n_rows, n_kmers, x, tail);
            size_t tb = 0;
            e = cub::DeviceScan::ExclusiveSum(nullptr, tb, x, x, (int64_t)(n_kmers + 1), s);
            if (e == cudaSuccess) e = cudaMalloc(&tmp, tb ? tb : 1);
            if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(tmp, tb, x, x, (int64_t)(n_kmers + 1), s);
            u64 head = 0;
            unsigned long long t = 0;
            if (e == cudaSuccess) e = cudaMemcpyAsync(&head, x + n_kmers, sizeof(u64), cudaMemcpyDeviceToHost, s);
            if (e == cudaSuccess) e = cudaMemcpyAsync(&t, tail, sizeof(t), cudaMemcpyDeviceToHost, s);
            if (e == cudaSuccess) e = cudaStreamSynchronize(s);
            if (e != cudaSuccess) {
                rc = set_error("sbwt_format_answers_device: %s", cudaGetErrorString(e));
            } else {
                *bytes = head + t;
                if (d_out) {
                    if (cap < *bytes) {
                        rc = set_error("the text needs %llu bytes, the buffer holds %llu", (unsigned long long)*bytes,
                                       (unsigned long long)cap);
                    } else {
                        write_items_kernel<<<bk, kThreads, 0, s>>>(d_answers, n_kmers, x, d_out, tail);
                        e = cudaGetLastError();
                        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
                        if (e != cudaSuccess) rc = set_error("sbwt_format_answers_device: %s", cudaGetErrorString(e));
                    }
                }
            }
        }
    }
    cudaFree(tmp);
    cudaFree(x);
    cudaFree(kstart);
    cudaFree(scan);
    cudaFree(tail);
    return rc;
}
