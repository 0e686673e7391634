// stream.cu -- builds the backward-step structures (stream.cuh): select
// samples, node nibbles and the backward table, on the GPU from the index's
// lines alone, so that indexes loaded from the reference's files get them
// too.  No reference counterpart.
//
// First letters and groups come from the labels: with pred(v) = the first
// node of the group of v's predecessor (stream.cuh), the last letter of
// pred^t(v) is label(v)[k-1-t] for t < k, and the chain reaches the all-$
// root exactly where the label's $ padding starts.  Pointer doubling builds,
// for every node, the last min(32, real letters) letters of its label in
// five rounds of gathers:
//   code(v) = sum_t lastletter(pred^t(v)) << 2t,  len(v) = letters before the root
// Then first letter = letter k-1 (or $ if len < k), and v starts a group iff
// its last k-1 letters (and how many of them are real) differ from v-1's.
#include <cstring>
#include <vector>

#include "internal.h"
#include "stream.cuh"

namespace sbwt {
namespace {

using namespace dev;

// sel_c[s] = line holding the one of rank 64 s of vector c.
__global__ void select_samples_kernel(const ulonglong4 *__restrict__ lines, u32 lpc, u32 *__restrict__ sel,
                                      u32 n_samples) {
    const u32 t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= lpc) return;
    const ulonglong4 w = lines[t];
    const u32 cnt = (u32)(w.x >> 32);
    const u32 ones = __popcll(w.x & 0xffffffffull) + __popcll(w.y) + __popcll(w.z) + __popcll(w.w);
    if (!ones) return;
    const u32 s_lo = (cnt + 63u) >> kSelLog, s_hi = (cnt + ones - 1u) >> kSelLog;
    for (u32 s = s_lo; s <= s_hi && s < n_samples; s++) sel[s] = t;
}

__global__ void pred_init_kernel(const StreamView sv, u32 *__restrict__ P, u64 *__restrict__ code,
                                 uint8_t *__restrict__ len, unsigned long long *__restrict__ bad) {
    const u32 v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= sv.n) return;
    if (v == 0) {
        P[0] = 0;
        code[0] = 0;
        len[0] = 0;
        return;
    }
    u32 u = sv.pred(v);
    if (u >= sv.n) {  // not an SBWT: record it, point at the root
        atomicAdd(bad, 1ull);
        u = 0;
    }
    P[v] = u;
    code[v] = sv.last_letter(v);
    len[v] = 1;
}

// One doubling round: window m -> 2m letters.
__global__ void double_kernel(u32 n, u32 m, const u32 *__restrict__ P, const u64 *__restrict__ code,
                              const uint8_t *__restrict__ len, u32 *__restrict__ P2, u64 *__restrict__ code2,
                              uint8_t *__restrict__ len2) {
    const u32 v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    const u32 l = len[v];
    const u32 u = P[v];
    if (l < m) {  // the chain reached the root inside the window
        code2[v] = code[v];
        len2[v] = (uint8_t)l;
        P2[v] = 0;
        return;
    }
    code2[v] = code[v] | (code[u] << (2u * m));
    len2[v] = (uint8_t)(m + len[u]);
    P2[v] = P[u];
}

// One thread per byte: the nibbles of nodes 2t and 2t+1.
__global__ void node_nibbles_kernel(u32 n, u32 k, const u64 *__restrict__ code, const uint8_t *__restrict__ len,
                                   uint8_t *__restrict__ node) {
    const u32 t = blockIdx.x * blockDim.x + threadIdx.x;
    if ((u64)t * 2u >= n) return;
    const u64 mask = (1ull << (2u * (k - 1u))) - 1ull;  // the last k-1 letters (k <= 32)
    u32 byte = 0;
    for (u32 h = 0; h < 2u; h++) {
        const u32 v = 2u * t + h;
        if (v >= n) break;
        const u32 l = len[v];
        const u64 c = code[v];
        const u32 first = l >= k ? (u32)((c >> (2u * (k - 1u))) & 3u) + 1u : 0u;
        bool start = v == 0;
        if (!start) {
            const u32 lp = len[v - 1];
            start = ((c ^ code[v - 1]) & mask) != 0 || min(l, k - 1u) != min(lp, k - 1u);
        }
        byte |= (first | (start ? kGroupStart : 0u)) << (4u * h);
    }
    node[t] = (uint8_t)byte;
}

// Backward table: entry v = pred(v) | group_letters(pred(v)) << 32 (node 0: 0).
__global__ void back_table_kernel(const StreamView sv, u64 *__restrict__ back) {
    const u32 v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= sv.n) return;
    u64 e = 0;
    if (v) {
        const u32 u0 = sv.pred(v);
        if (u0 < sv.n) e = (u64)u0 | ((u64)sv.group_letters(u0) << 32);
    }
    back[v] = e;
}

}  // namespace

StreamView stream_view(const sbwt_index *ix) {
    StreamView sv;
    std::memset(&sv, 0, sizeof(sv));
    sv.lines = ix->d_lines;
    sv.lpc = ix->lpc;
    sv.sel = ix->d_sel;
    for (int c = 0; c < 4; c++) {
        sv.sel_off[c] = ix->sel_off[c];
        sv.sel_n[c] = ix->sel_n[c];
        sv.C[c] = (u32)ix->C[c];
    }
    sv.node = ix->d_node;
    sv.back = ix->d_back;
    sv.n = (u32)ix->n;
    return sv;
}

int build_stream(sbwt_index *ix, cudaStream_t s) {
    if (ix->stream_ok) return 0;
    if (!ix->lines_ok) return set_error("the backward step needs the line layout");
    if (ix->k > 32 || ix->k < 2) return set_error("k out of range");
    const u32 n = (u32)ix->n;
    u64 total = 0;
    for (int c = 0; c < 4; c++) {
        const u64 ones = ix->C[c + 1] - ix->C[c];
        ix->sel_off[c] = (u32)total;
        ix->sel_n[c] = (u32)((ones + 63) >> kSelLog);
        total += ix->sel_n[c] + 1;
    }
    SBWT_CHECK_CUDA(cudaMalloc(&ix->d_sel, total * sizeof(u32)));
    SBWT_CHECK_CUDA(cudaMemsetAsync(ix->d_sel, 0, total * sizeof(u32), s));
    SBWT_CHECK_CUDA(cudaMalloc(&ix->d_node, (size_t)n / 2 + 16));
    for (int c = 0; c < 4; c++) {
        if (!ix->sel_n[c]) continue;
        select_samples_kernel<<<(ix->lpc + 255) / 256, 256, 0, s>>>(ix->d_lines + (u64)c * ix->lpc, ix->lpc,
                                                                     ix->d_sel + ix->sel_off[c], ix->sel_n[c]);
        SBWT_CHECK_CUDA(cudaGetLastError());
    }
    // scratch: P, code, len twice, plus a flag
    u32 *P[2] = {nullptr, nullptr};
    u64 *code[2] = {nullptr, nullptr};
    uint8_t *len[2] = {nullptr, nullptr};
    unsigned long long *bad = nullptr;
    int rc = 0;
    auto fail = [&](cudaError_t e) {
        rc = set_error("CUDA error while building the backward-step structures: %s", cudaGetErrorString(e));
    };
    cudaError_t e = cudaSuccess;
    for (int i = 0; i < 2 && e == cudaSuccess; i++) {
        e = cudaMalloc(&P[i], (size_t)n * sizeof(u32));
        if (e == cudaSuccess) e = cudaMalloc(&code[i], (size_t)n * sizeof(u64));
        if (e == cudaSuccess) e = cudaMalloc(&len[i], (size_t)n);
    }
    if (e == cudaSuccess) e = cudaMalloc(&bad, sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMemsetAsync(bad, 0, sizeof(unsigned long long), s);
    if (e != cudaSuccess) {
        fail(e);
    } else {
        ix->stream_ok = false;
        const StreamView sv = stream_view(ix);
        const u32 blocks = (n + 255) / 256;
        pred_init_kernel<<<blocks, 256, 0, s>>>(sv, P[0], code[0], len[0], bad);
        int cur = 0;
        for (u32 m = 1; m <= 16; m <<= 1) {
            double_kernel<<<blocks, 256, 0, s>>>(n, m, P[cur], code[cur], len[cur], P[cur ^ 1], code[cur ^ 1],
                                                 len[cur ^ 1]);
            cur ^= 1;
        }
        node_nibbles_kernel<<<(n / 2 + 1 + 255) / 256, 256, 0, s>>>(n, ix->k, code[cur], len[cur], ix->d_node);
        if (SBWT_BACK_TABLE) {
            e = cudaMalloc(&ix->d_back, (size_t)n * sizeof(u64));
            if (e == cudaSuccess) back_table_kernel<<<blocks, 256, 0, s>>>(stream_view(ix), ix->d_back);
        }
        unsigned long long h_bad = 0;
        if (e == cudaSuccess) e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaMemcpyAsync(&h_bad, bad, sizeof h_bad, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) fail(e);
        else if (h_bad) rc = set_error("the bit vectors are not an SBWT: %llu nodes have no predecessor", h_bad);
    }
    for (int i = 0; i < 2; i++) {
        cudaFree(P[i]);
        cudaFree(code[i]);
        cudaFree(len[i]);
    }
    cudaFree(bad);
    if (rc) {
        cudaFree(ix->d_node);
        cudaFree(ix->d_sel);
        cudaFree(ix->d_back);
        ix->d_node = nullptr;
        ix->d_sel = nullptr;
        ix->d_back = nullptr;
        return rc;
    }
    ix->stream_ok = true;
    ix->gen++;
    return 0;
}

}  // namespace sbwt

using namespace sbwt;

extern "C" int sbwt_node_bytes_export(sbwt_index *ix, uint8_t *out, uint64_t count) {
    clear_error();
    if (!ix || !out) return set_error("NULL argument");
    if (count != ix->n) return set_error("count must be the number of columns (%llu)", (unsigned long long)ix->n);
    SBWT_CHECK_CUDA(cudaSetDevice(ix->device));
    SBWT_TRY(build_stream(ix, 0));
    std::vector<uint8_t> packed(count / 2 + 1);
    SBWT_CHECK_CUDA(cudaMemcpy(packed.data(), ix->d_node, count / 2 + (count & 1), cudaMemcpyDeviceToHost));
    for (u64 v = 0; v < count; v++) out[v] = (uint8_t)((packed[v >> 1] >> ((v & 1) * 4)) & 15u);
    return 0;
}
