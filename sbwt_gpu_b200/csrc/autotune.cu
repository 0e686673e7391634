// autotune.cu -- this engine's autotuner (no reference counterpart: the
// reference takes its kernel variant from flags, include/parameters.hpp:
// 79-297, and picks it by template switch, include/epicseq/search_caller.hpp:
// 81-209).
//
// On a caller-supplied sample batch (device letters + row starts) the tuner
// times sbwt_search_reads for each candidate launch shape and keeps the
// fastest: the queue-fed single-slot kernel and the line layout x k-mers per
// thread {1,2,3,4,6,8} x threads per k-mer
// {1,2,4} x threads per block {128,256}; optionally the reference's poppy
// layouts (SB 512/1024/2048, with and without the cooperative "shuffles"
// rank); and optionally presearch depths p in {8,10,12,14,15} (p <= k).  Every
// candidate's answers are reduced to an order-sensitive checksum, and all
// checksums must agree: the sweep doubles as a bit-exactness check across
// shapes at full size.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "internal.h"

namespace sbwt {
namespace {

__global__ void checksum_kernel(const u64 *__restrict__ a, u64 n, unsigned long long *out) {
    u64 s = 0;
    for (u64 j = (u64)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += (u64)gridDim.x * blockDim.x)
        s += a[j] * (2ull * j + 1ull);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31u) == 0) atomicAdd(out, (unsigned long long)s);
}

struct Cand {
    int layout;
    u32 kpt, tpk, tpb, sb;
    int shuffles;
    u32 p;
    float ms;
    unsigned long long sum;
};

std::string cand_json(const Cand &c) {
    char b[256];
    std::snprintf(b, sizeof b,
                  "{\"layout\":\"%s\",\"kmers_per_thread\":%u,\"threads_per_kmer\":%u,\"threads_per_block\":%u,"
                  "\"bits_in_superblock\":%u,\"shuffles\":%d,\"p\":%u,\"ms\":%.4f}",
                  c.layout == SBWT_LAYOUT_LINES ? "lines" : "poppy", c.kpt, c.tpk, c.tpb, c.sb, c.shuffles, c.p,
                  c.ms);
    return b;
}

}  // namespace
}  // namespace sbwt

using namespace sbwt;

extern "C" int sbwt_autotune(sbwt_index *ix, const uint8_t *d_letters, uint64_t n_letters,
                             const uint64_t *d_row_starts, uint64_t n_rows, uint64_t n_kmers, uint64_t *d_answers,
                             uint32_t flags, char *report, uint64_t report_cap) {
    clear_error();
    if (!ix) return set_error("index is NULL");
    if (n_kmers == 0 || n_rows == 0) return set_error("autotune needs a non-empty sample");
    SBWT_CHECK_CUDA(cudaSetDevice(ix->device));
    cudaStream_t s = nullptr;
    SBWT_CHECK_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    unsigned long long *d_sum = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int rc = 0;
    const KernelShape saved = ix->shape;
    const u32 saved_p = ix->p;
    const bool saved_graph = ix->use_graph, saved_prof = ix->prof_on;
    ix->use_graph = false;
    ix->prof_on = false;
    std::vector<Cand> done;
    unsigned long long want_sum = 0;
    bool have_sum = false;

    auto apply = [&](const Cand &c) -> int {
        if (c.layout == SBWT_LAYOUT_POPPY) {
            if (!ix->poppy_ok || ix->sb != c.sb || ix->kind != SBWT_POPPY) SBWT_TRY(build_poppy(ix, c.sb, SBWT_POPPY, s));
        }
        ix->shape.layout = c.layout;
        ix->shape.kpt = c.kpt;
        ix->shape.tpk = c.tpk;
        ix->shape.tpb = c.tpb;
        ix->shape.sb = c.sb;
        ix->shape.kind = SBWT_POPPY;
        ix->shape.shuffles = c.shuffles;
        if (c.p != ix->p) SBWT_TRY(run_presearch(ix, c.p, s));
        return 0;
    };
    auto measure = [&](Cand &c) -> int {
        SBWT_TRY(apply(c));
        Workspace &w = ix->ws[0];
        SBWT_TRY(search_rows_device(ix, w, d_letters, n_letters, d_row_starts, n_rows, d_answers, nullptr, n_kmers, s));
        float best = 1e30f;
        for (int rep = 0; rep < 3; rep++) {
            SBWT_CHECK_CUDA(cudaEventRecord(e0, s));
            SBWT_TRY(search_rows_device(ix, w, d_letters, n_letters, d_row_starts, n_rows, d_answers, nullptr, n_kmers,
                                        s));
            SBWT_CHECK_CUDA(cudaEventRecord(e1, s));
            SBWT_CHECK_CUDA(cudaEventSynchronize(e1));
            float ms = 0;
            SBWT_CHECK_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            best = std::min(best, ms);
        }
        SBWT_CHECK_CUDA(cudaMemsetAsync(d_sum, 0, sizeof(*d_sum), s));
        checksum_kernel<<<1184, 256, 0, s>>>(d_answers, n_kmers, d_sum);
        SBWT_CHECK_CUDA(cudaGetLastError());
        SBWT_CHECK_CUDA(cudaMemcpyAsync(&c.sum, d_sum, sizeof(c.sum), cudaMemcpyDeviceToHost, s));
        SBWT_CHECK_CUDA(cudaStreamSynchronize(s));
        c.ms = best;
        if (!have_sum) {
            want_sum = c.sum;
            have_sum = true;
        } else if (c.sum != want_sum) {
            return set_error("autotune: answers of %s differ from the first candidate's", cand_json(c).c_str());
        }
        done.push_back(c);
        return 0;
    };

    do {
        if (cudaMalloc(&d_sum, sizeof(*d_sum)) != cudaSuccess || cudaEventCreate(&e0) != cudaSuccess ||
            cudaEventCreate(&e1) != cudaSuccess) {
            rc = set_error("autotune: out of device resources");
            break;
        }
        const u32 p0 = saved_p;
        std::vector<Cand> stage1;
        if (ix->lines_ok) {
            stage1.push_back(Cand{SBWT_LAYOUT_LINES, 0, 1, 128, 1024, 0, p0, 0, 0});  // queue-fed single slot
            for (u32 tpb : {128u, 256u})
                for (u32 tpk : {1u, 2u, 4u})
                    for (u32 kpt : {1u, 2u, 3u, 4u, 6u, 8u}) stage1.push_back(Cand{SBWT_LAYOUT_LINES, kpt, tpk, tpb, 1024, 0, p0, 0, 0});
        }
        if ((flags & 4u) || !ix->lines_ok)
            for (u32 sb : {512u, 1024u, 2048u})
                for (int sh : {0, 1}) {
                    if (sh && sb == 512) continue;
                    for (u32 kpt : {0u, 1u, 2u}) {
                        if (kpt == 0 && sh) continue;
                        stage1.push_back(Cand{SBWT_LAYOUT_POPPY, kpt, 1, kpt == 0 ? 128u : 256u, sb, sh, p0, 0, 0});
                    }
                }
        for (Cand &c : stage1)
            if ((rc = measure(c)) != 0) break;
        if (rc) break;
        std::vector<Cand> ranked = done;
        std::sort(ranked.begin(), ranked.end(), [](const Cand &a, const Cand &b) { return a.ms < b.ms; });
        Cand best = ranked.front();
        if (flags & 2u) {
            for (u32 p : {8u, 10u, 12u, 14u, 15u}) {
                if (p > ix->k || p == best.p) continue;
                Cand c = best;
                c.p = p;
                if ((rc = measure(c)) != 0) break;
                if (c.ms < best.ms) best = c;
            }
            if (rc) break;
            // re-rank the five best shapes at the chosen p
            for (size_t i = 0; i < ranked.size() && i < 5; i++) {
                Cand c = ranked[i];
                if (c.p == best.p) continue;
                c.p = best.p;
                if ((rc = measure(c)) != 0) break;
                if (c.ms < best.ms) best = c;
            }
            if (rc) break;
        }
        if ((rc = apply(best)) != 0) break;
        if (report && report_cap) {
            std::string j = "{\"best\":" + cand_json(best) + ",\"n_kmers\":" + std::to_string(n_kmers) +
                            ",\"checksum\":" + std::to_string(want_sum) + ",\"candidates\":[";
            for (size_t i = 0; i < done.size(); i++) j += (i ? "," : "") + cand_json(done[i]);
            j += "]}";
            if (j.size() + 1 > report_cap) {
                rc = set_error("autotune: report needs %zu bytes", j.size() + 1);
                break;
            }
            std::memcpy(report, j.c_str(), j.size() + 1);
        }
    } while (false);
    if (rc) {  // restore the previous configuration
        ix->shape = saved;
        if (ix->p != saved_p) run_presearch(ix, saved_p, s);
    }
    ix->use_graph = saved_graph;
    ix->prof_on = saved_prof;
    if (d_sum) cudaFree(d_sum);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
    return rc;
}
