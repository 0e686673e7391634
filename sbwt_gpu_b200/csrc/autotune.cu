// autotune.cu -- this engine's autotuner (no reference counterpart: the
// reference takes its kernel variant from flags, include/parameters.hpp:
// 79-297, and picks it by template switch, include/epicseq/search_caller.hpp:
// 81-209).
//
// On a caller-supplied sample batch (device letters + row starts) the tuner
// times sbwt_search_reads for candidate configurations and keeps the
// fastest, in stages:
//   1. the search layout: 32-byte lines and the 512/2048-bit wide lines
//      (the interleave granularity), with SBWT_TUNE_POPPY also the
//      reference's poppy layouts (SB 512/1024/2048), with SBWT_TUNE_SHAPES
//      also the per-k-mer kernel's register shapes (k-mers per thread
//      {1,2,3,4,6,8} x threads per k-mer {1,2,4} x threads per block
//      {128,256});
//   2. the run walk's knobs on the best layout, one at a time, each kept
//      when it is faster: window (64 / 256 k-mers against 128), resident
//      blocks per SM, the evict-first policy of the presearch and
//      backward-table gathers (never / always against by table size), the
//      rank lines held in the persisting L2 set-aside, and the compact
//      4-byte presearch entries;
//   3. with SBWT_TUNE_P the presearch depth p in {8,10,12,14,15} (p <= k),
//      then the window and the evict policy again at the chosen p.
// Every candidate's answers are reduced to an order-sensitive checksum, and
// all checksums must agree: the sweep doubles as a bit-exactness check
// across configurations at full size.
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
    u32 window, bps;
    int evict, compact, persist;
    float ms;
    unsigned long long sum;
};

const char *layout_name(int l) {
    return l == SBWT_LAYOUT_LINES ? "lines" : l == SBWT_LAYOUT_POPPY ? "poppy" : l == SBWT_LAYOUT_LINES512 ? "lines512"
                                                                                                          : "lines2048";
}

std::string cand_json(const Cand &c) {
    char b[384];
    std::snprintf(b, sizeof b,
                  "{\"layout\":\"%s\",\"kmers_per_thread\":%u,\"threads_per_kmer\":%u,\"threads_per_block\":%u,"
                  "\"bits_in_superblock\":%u,\"shuffles\":%d,\"p\":%u,\"window\":%u,\"blocks_per_sm\":%u,"
                  "\"evict\":\"%s\",\"compact_presearch\":%d,\"l2_persist\":%d,\"ms\":%.4f}",
                  layout_name(c.layout), c.kpt, c.tpk, c.tpb, c.sb, c.shuffles, c.p, c.window, c.bps,
                  c.evict == 0 ? "by table size" : c.evict == 1 ? "never" : "always", c.compact, c.persist, c.ms);
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
    const int saved_compact = ix->compact_pre;
    const bool saved_graph = ix->use_graph, saved_prof = ix->prof_on;
    ix->use_graph = false;
    ix->prof_on = false;
    std::vector<Cand> done;
    float default_ms = 0.0f;
    unsigned long long want_sum = 0;
    bool have_sum = false;

    auto apply = [&](const Cand &c) -> int {
        if (c.layout == SBWT_LAYOUT_POPPY) {
            if (!ix->poppy_ok || ix->sb != c.sb || ix->kind != SBWT_POPPY) SBWT_TRY(build_poppy(ix, c.sb, SBWT_POPPY, s));
        }
        if (wide_sectors(c.layout) && ix->wide_s != wide_sectors(c.layout)) SBWT_TRY(build_wide(ix, wide_sectors(c.layout), s));
        ix->shape.layout = c.layout;
        ix->shape.kpt = c.kpt;
        ix->shape.tpk = c.tpk;
        ix->shape.tpb = c.tpb;
        ix->shape.sb = c.sb;
        ix->shape.kind = SBWT_POPPY;
        ix->shape.shuffles = c.shuffles;
        ix->shape.window = c.window;
        ix->shape.blocks_per_sm = c.bps;
        ix->shape.evict = c.evict;
        ix->shape.l2_persist = c.persist;
        if (!c.persist && ix->l2_setaside) l2_setaside_release(ix);  // a set-aside without the window costs L2
        if (c.p != ix->p || c.compact != ix->compact_pre) {
            ix->compact_pre = c.compact;
            SBWT_TRY(run_presearch(ix, c.p, s));
        }
        ix->gen++;
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
        const int c0 = ix->compact_pre;
        // stage 1: layouts; the first candidate is the index's configuration before tuning
        std::vector<Cand> stage1;
        stage1.push_back(Cand{saved.layout, saved.kpt, saved.tpk, saved.tpb, saved.sb, saved.shuffles, p0,
                              saved.window, saved.blocks_per_sm, saved.evict, c0, saved.l2_persist, 0, 0});
        if (ix->lines_ok) {
            for (int l : {SBWT_LAYOUT_LINES, SBWT_LAYOUT_LINES512, SBWT_LAYOUT_LINES2048})
                if (!(l == saved.layout && saved.kpt == 0 && saved.tpk == 1))
                    stage1.push_back(Cand{l, 0, 1, 128, 1024, 0, p0, 128, 0, 0, c0, 0, 0, 0});
            if (flags & 8u)
                for (u32 tpb : {128u, 256u})
                    for (u32 tpk : {1u, 2u, 4u})
                        for (u32 kpt : {1u, 2u, 3u, 4u, 6u, 8u})
                            stage1.push_back(Cand{SBWT_LAYOUT_LINES, kpt, tpk, tpb, 1024, 0, p0, 128, 0, 0, c0, 0, 0, 0});
        }
        if ((flags & 4u) || !ix->lines_ok)
            for (u32 sb : {512u, 1024u, 2048u})
                for (int sh : {0, 1}) {
                    if (sh && sb == 512) continue;
                    for (u32 kpt : {0u, 1u, 2u}) {
                        if (kpt == 0 && sh) continue;
                        if (kpt && !(flags & 8u)) continue;
                        stage1.push_back(Cand{SBWT_LAYOUT_POPPY, kpt, 1, kpt == 0 ? 128u : 256u, sb, sh, p0, 128, 0, 0,
                                              c0, 0, 0, 0});
                    }
                }
        for (Cand &c : stage1)
            if ((rc = measure(c)) != 0) break;
        if (rc) break;
        default_ms = done.front().ms;
        Cand best = *std::min_element(done.begin(), done.end(), [](const Cand &a, const Cand &b) { return a.ms < b.ms; });
        // stage 2: the run walk's knobs, one at a time (kept when faster by more than 1 %)
        auto try_knob = [&](Cand c) -> int {
            SBWT_TRY(measure(c));
            if (c.ms < 0.99f * best.ms) best = c;
            return 0;
        };
        auto walk_knobs = [&](bool grid, bool compact) -> int {
            if (best.kpt != 0) return 0;  // the per-k-mer kernel has none of these knobs
            if (best.layout == SBWT_LAYOUT_LINES)
                for (u32 w : {64u, 256u}) {
                    Cand c = best;
                    c.window = w;
                    SBWT_TRY(try_knob(c));
                }
            for (int ev : {1, 2}) {
                Cand c = best;
                c.evict = ev;
                SBWT_TRY(try_knob(c));
            }
            if (grid)
                for (u32 b : {4u, 6u, 7u, 8u}) {
                    Cand c = best;
                    c.bps = b;
                    SBWT_TRY(try_knob(c));
                }
            if (best.layout != SBWT_LAYOUT_POPPY) {  // the rank lines in the L2 set-aside
                Cand c = best;
                c.persist = best.persist ? 0 : 1;
                SBWT_TRY(try_knob(c));
            }
            if (compact && ix->n < dev::kPreMaxColumns && best.p) {
                Cand c = best;
                c.compact = best.compact == 1 ? 0 : 1;
                SBWT_TRY(try_knob(c));
            }
            return 0;
        };
        if ((rc = walk_knobs(true, true)) != 0) break;
        // stage 3: presearch depth, then the knobs that depend on the tables' sizes again
        if (flags & 2u) {
            const Cand before = best;
            for (u32 p : {8u, 10u, 12u, 14u, 15u}) {
                if (p > ix->k || p == before.p) continue;
                Cand c = before;
                c.p = p;
                if ((rc = try_knob(c)) != 0) break;
            }
            if (rc) break;
            if (best.p != before.p && (rc = walk_knobs(false, true)) != 0) break;
        }
        if ((rc = apply(best)) != 0) break;
        if (report && report_cap) {
            char dm[32];
            std::snprintf(dm, sizeof dm, "%.4f", default_ms);
            std::string j = "{\"best\":" + cand_json(best) + ",\"default_ms\":" + dm +
                            ",\"n_kmers\":" + std::to_string(n_kmers) + ",\"checksum\":" + std::to_string(want_sum) +
                            ",\"candidates\":[";
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
        if (ix->p != saved_p || ix->compact_pre != saved_compact) {
            ix->compact_pre = saved_compact;
            run_presearch(ix, saved_p, s);
        }
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
