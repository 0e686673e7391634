// api.cu -- the C ABI (include/sbwt_gpu.h): index handle, device memory,
// streams, and the search entry points.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <vector>

#include "device.cuh"
#include "internal.h"

using sbwt::set_error;
using sbwt::u32;
using sbwt::u64;

namespace sbwt {

void Workspace::release() {
    cudaFree(words); cudaFree(kstart); cudaFree(chunk_row); cudaFree(scan); cudaFree(counter);
    cudaFree(letters); cudaFree(rows); cudaFree(answers); cudaFree(member); cudaFree(goff); cudaFree(nodes);
    if (h_rows) cudaFreeHost(h_rows);
    if (h_goff) cudaFreeHost(h_goff);
    if (h_nodes) cudaFreeHost(h_nodes);
    if (h_member) cudaFreeHost(h_member);
    if (h_letters) cudaFreeHost(h_letters);
    if (h_answers) cudaFreeHost(h_answers);
    if (graph) cudaGraphExecDestroy(graph);
    *this = Workspace();
}

// Grow-only device buffer of `need` elements.
template <class T>
int grow(T *&p, size_t &cap, size_t need) {
    if (cap >= need && p) return 0;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    const size_t want = std::max(need, (size_t)1);
    SBWT_CHECK_CUDA(cudaMalloc((void **)&p, want * sizeof(T)));
    cap = want;
    return 0;
}

// Grow-only pinned host buffer of `need` elements.
template <class T>
int grow_host(T *&p, size_t &cap, size_t need) {
    if (cap >= need && p) return 0;
    if (p) cudaFreeHost(p);
    p = nullptr;
    cap = 0;
    const size_t want = std::max(need, (size_t)1);
    SBWT_CHECK_CUDA(cudaHostAlloc((void **)&p, want * sizeof(T), cudaHostAllocDefault));
    cap = want;
    return 0;
}

template int grow<uint8_t>(uint8_t *&, size_t &, size_t);
template int grow<uint32_t>(uint32_t *&, size_t &, size_t);
template int grow<unsigned long long>(unsigned long long *&, size_t &, size_t);
template int grow<uint64_t>(uint64_t *&, size_t &, size_t);
template int grow_host<uint8_t>(uint8_t *&, size_t &, size_t);
template int grow_host<uint64_t>(uint64_t *&, size_t &, size_t);
template int grow_host<uint32_t>(uint32_t *&, size_t &, size_t);

namespace {

int use_device(int device) {
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0)
        return set_error("no CUDA device is available (%s); this engine has no CPU fallback",
                         e != cudaSuccess ? cudaGetErrorString(e) : "0 devices");
    if (device < 0 || device >= count) return set_error("CUDA device %d does not exist (%d devices)", device, count);
    SBWT_CHECK_CUDA(cudaSetDevice(device));
    return 0;
}

int validate_params(const sbwt_params *p) {
    if (p->k < 3 || p->k > 32) return set_error("The value of k must be at least 3 and at most 32.");
    if (p->k_presearch > p->k) return set_error("presearch depth %u exceeds k = %u", p->k_presearch, p->k);
    if (p->layout < SBWT_LAYOUT_LINES || p->layout > SBWT_LAYOUT_LINES2048) return set_error("unknown layout %d", p->layout);
    if (p->search_mode != SBWT_SEARCH_EVERY_KMER && p->search_mode != SBWT_SEARCH_SKIP_ABSENT &&
        p->search_mode != SBWT_SEARCH_STREAM)
        return set_error("unknown search mode %d", p->search_mode);
    return 0;
}

void apply_shape(sbwt_index *ix, const sbwt_params *p) {
    sbwt::KernelShape &sh = ix->shape;
    sh.layout = (p->layout >= SBWT_LAYOUT_LINES && p->layout <= SBWT_LAYOUT_LINES2048) ? p->layout : SBWT_LAYOUT_LINES;
    // defaults from the autotuner on the large workload (1 k-mer per thread,
    // 128-thread blocks: occupancy beats register-resident k-mer slots)
    sh.kpt = p->kmers_per_thread;  // 0: the queue-fed single-slot kernel
    sh.tpk = p->threads_per_kmer ? p->threads_per_kmer : 1;
    sh.tpb = p->threads_per_block ? std::min<u32>(p->threads_per_block, 256u) : 128u;
    sh.sb = p->bits_in_superblock;
    sh.kind = p->rank_structure;
    sh.shuffles = p->with_shuffles;
    sh.mode = p->search_mode;
}

// Shared tail of the two index constructors: `words[c]` hold ceil(n/64)
// words of vector c in the reference's in-memory layout.
int finish_index(sbwt_index *ix, const u64 *const words[4], const sbwt_params *prm) {
    const u64 n = ix->n;
    const u64 nw = (n + 63) / 64;
    ix->wpv = (n + 4095) / 4096 * 64 + 64;  // bit_vector.hpp:104 plus one spare block
    SBWT_CHECK_CUDA(cudaMalloc(&ix->d_bits, 4 * ix->wpv * sizeof(u64)));
    SBWT_CHECK_CUDA(cudaMemset(ix->d_bits, 0, 4 * ix->wpv * sizeof(u64)));
    for (int c = 0; c < 4; c++) {
        u64 *dst = ix->d_bits + (u64)c * ix->wpv;
        if (nw > 1) SBWT_CHECK_CUDA(cudaMemcpy(dst, words[c], (nw - 1) * sizeof(u64), cudaMemcpyHostToDevice));
        // bits past n are zero on the device whatever the caller's padding holds
        u64 last = words[c][nw - 1];
        if (n % 64) last &= ~0ull << (64 - n % 64);
        SBWT_CHECK_CUDA(cudaMemcpy(dst + nw - 1, &last, sizeof(u64), cudaMemcpyHostToDevice));
    }
    cudaStream_t s = 0;
    u64 ones[4] = {0, 0, 0, 0};
    // device time of each build phase (sbwt_build_times)
    cudaEvent_t ev[5];
    for (auto &e : ev) SBWT_CHECK_CUDA(cudaEventCreate(&e));
    struct EvFree {
        cudaEvent_t *e;
        ~EvFree() {
            for (int i = 0; i < 5; i++) cudaEventDestroy(e[i]);
        }
    } ev_free{ev};
    SBWT_CHECK_CUDA(cudaEventRecord(ev[0], s));
    if (n / sbwt::dev::kLineBits + 1 <= sbwt::dev::kMaxLinesPerChar) {
        ix->lpc = (u32)(((n / sbwt::dev::kLineBits + 1) + 7) / 8 * 8);
        SBWT_CHECK_CUDA(cudaMalloc(&ix->d_lines, 4ull * ix->lpc * sizeof(ulonglong4)));
        SBWT_TRY(sbwt::build_lines(ix, s, ones));
        ix->lines_ok = true;
    }
    SBWT_CHECK_CUDA(cudaEventRecord(ev[1], s));
    const bool want_poppy = prm->layout == SBWT_LAYOUT_POPPY || !ix->lines_ok;
    if (want_poppy) {
        SBWT_TRY(sbwt::build_poppy(ix, prm->bits_in_superblock, prm->rank_structure, s));
        if (!ix->lines_ok) {
            // ones of each vector = sum of the last L12 relative count chain: read via the sentinel
            std::vector<u64> l0(ix->l0w), l12(1);
            for (int c = 0; c < 4; c++) {
                SBWT_CHECK_CUDA(cudaMemcpy(l0.data(), ix->d_L0 + (u64)c * ix->l0w, ix->l0w * sizeof(u64),
                                           cudaMemcpyDeviceToHost));
                SBWT_CHECK_CUDA(cudaMemcpy(l12.data(), ix->d_L12 + (u64)c * ix->l12w + ix->l12w - 1, sizeof(u64),
                                           cudaMemcpyDeviceToHost));
                const u64 nsb = ix->l12w - 1;
                u64 h = (nsb * ix->sb) >> (ix->sb == 4096 ? 31 : 32);
                if (h >= ix->l0w) h = ix->l0w - 1;
                ones[c] = l0[h] + (l12[0] >> (ix->sb == 4096 ? 33 : 32));
            }
        }
    }
    // matrix_sbwt.hpp:150-157
    ix->C[0] = 1;
    for (int c = 0; c < 4; c++) ix->C[c + 1] = ix->C[c] + ones[c];
    if (ix->C[4] != n)
        return set_error("the bit vectors are not an SBWT: 1 + total ones = %llu but n = %llu",
                         (unsigned long long)ix->C[4], (unsigned long long)n);
    {
        const int persist = ix->shape.l2_persist;  // set from the environment in new_index
        apply_shape(ix, prm);
        ix->shape.l2_persist = persist;
    }
    if (ix->shape.layout != SBWT_LAYOUT_POPPY && !ix->lines_ok) ix->shape.layout = SBWT_LAYOUT_POPPY;
    if (sbwt::wide_sectors(ix->shape.layout)) SBWT_TRY(sbwt::build_wide(ix, sbwt::wide_sectors(ix->shape.layout), s));
    SBWT_CHECK_CUDA(cudaEventRecord(ev[2], s));
    SBWT_TRY(sbwt::run_presearch(ix, prm->k_presearch, s));
    SBWT_CHECK_CUDA(cudaEventRecord(ev[3], s));
    if (ix->shape.mode == SBWT_SEARCH_STREAM && ix->lines_ok) SBWT_TRY(sbwt::build_stream(ix, s));
    SBWT_CHECK_CUDA(cudaEventRecord(ev[4], s));
    SBWT_CHECK_CUDA(cudaDeviceSynchronize());
    for (int i = 0; i < 4; i++) SBWT_CHECK_CUDA(cudaEventElapsedTime(&ix->build_ms[i], ev[i], ev[i + 1]));
    if (!want_poppy) ix->build_ms[1] = 0.0f;
    if (!ix->stream_ok) ix->build_ms[3] = 0.0f;
    return 0;
}

int new_index(const sbwt_params *prm, sbwt_index **out, sbwt_index **ix_out) {
    if (!out) return set_error("out is NULL");
    *out = nullptr;
    sbwt_params def;
    sbwt_params_default(&def);
    if (!prm) prm = &def;
    SBWT_TRY(validate_params(prm));
    SBWT_TRY(use_device(prm->device));
    sbwt_index *ix = new (std::nothrow) sbwt_index();
    if (!ix) return set_error("out of host memory");
    ix->device = prm->device;
    ix->k = prm->k;
    cudaDeviceGetAttribute(&ix->num_sms, cudaDevAttrMultiProcessorCount, prm->device);
    if (ix->num_sms <= 0) ix->num_sms = 1;
    int l2 = 0;
    cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, prm->device);
    ix->l2_bytes = l2 > 0 ? (uint64_t)l2 : 0;
    int mp = 0, mw = 0;
    cudaDeviceGetAttribute(&mp, cudaDevAttrMaxPersistingL2CacheSize, prm->device);
    cudaDeviceGetAttribute(&mw, cudaDevAttrMaxAccessPolicyWindowSize, prm->device);
    ix->l2_max_persist = mp > 0 ? (size_t)mp : 0;
    ix->l2_max_window = mw > 0 ? (size_t)mw : 0;
    if (const char *e = std::getenv("SBWT_L2_PERSIST")) ix->shape.l2_persist = std::atoi(e) != 0;
    if (const char *e = std::getenv("SBWT_RUN_INDEX64")) ix->shape.index64 = std::atoi(e) != 0;
    *ix_out = ix;
    return 0;
}

// BitVector::create header checks (include/bit_vector.hpp:65-109).
int read_vector(const char *path, u64 &n_bits, std::vector<u64> &words) {
    FILE *f = std::fopen(path, "rb");
    if (!f) return set_error("The file %s can not be opened.", path);
    std::fseek(f, 0, SEEK_END);
    const long size = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    if (size < 8) {
        std::fclose(f);
        return set_error("The size of the file %s is too small to contain any data.", path);
    }
    unsigned char hdr[8];
    if (std::fread(hdr, 1, 8, f) != 8) {
        std::fclose(f);
        return set_error("The file %s can not be read.", path);
    }
    u64 n = 0;
    for (int i = 0; i < 8; i++) n |= (u64)hdr[i] << (8 * i);
    if (n == 0) {
        std::fclose(f);
        return set_error("The first 8 bytes in the file %s indicates that there is a bit vector of size 0 in the file.",
                         path);
    }
    const u64 nbytes = (n + 7) / 8;
    if ((u64)size - 8 < nbytes) {
        std::fclose(f);
        return set_error("The file %s holds %llu data bytes; its header announces %llu bits (%llu bytes).", path,
                         (unsigned long long)((u64)size - 8), (unsigned long long)n, (unsigned long long)nbytes);
    }
    words.assign((n + 63) / 64, 0ull);
    const size_t got = std::fread(words.data(), 1, nbytes, f);
    std::fclose(f);
    if (got != nbytes) return set_error("The file %s can not be read.", path);
    // byte swap (rank_data_structures.hpp:98,103-113): position p at bit 63 - p%64
    const int64_t nw = (int64_t)words.size();
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < nw; i++) words[i] = __builtin_bswap64(words[i]);
    n_bits = n;
    return 0;
}

}  // namespace
}  // namespace sbwt

using namespace sbwt;

extern "C" int sbwt_params_default(sbwt_params *p) {
    if (!p) return set_error("params is NULL");
    std::memset(p, 0, sizeof(*p));
    p->k = 30;                   // parameters.hpp:49
    p->k_presearch = 12;         // parameters.hpp:50
    p->bits_in_superblock = 1024;  // parameters.hpp:42
    p->rank_structure = SBWT_POPPY;
    p->with_shuffles = 0;
    p->threads_per_block = 0;
    p->device = 0;
    p->layout = SBWT_LAYOUT_LINES;
    p->kmers_per_thread = 0;
    p->threads_per_kmer = 0;
    p->search_mode = SBWT_SEARCH_STREAM;
    return 0;
}

extern "C" int sbwt_index_from_host(const uint64_t *const bits[4], uint64_t n_bits, const sbwt_params *params,
                                    sbwt_index **out) {
    clear_error();
    sbwt_params def;
    sbwt_params_default(&def);
    if (!params) params = &def;
    if (n_bits == 0) return set_error("the index has no columns");
    for (int c = 0; c < 4; c++)
        if (!bits || !bits[c]) return set_error("bit vector %d is NULL", c);
    sbwt_index *ix = nullptr;
    SBWT_TRY(new_index(params, out, &ix));
    ix->n = n_bits;
    const int rc = finish_index(ix, bits, params);
    if (rc) {
        sbwt_index_free(ix);
        return rc;
    }
    *out = ix;
    return 0;
}

extern "C" int sbwt_index_load(const char *file_a, const char *file_c, const char *file_g, const char *file_t,
                               const sbwt_params *params, sbwt_index **out) {
    clear_error();
    const char *files[4] = {file_a, file_c, file_g, file_t};
    std::vector<u64> w[4];
    u64 n[4] = {0, 0, 0, 0};
    int rc[4] = {0, 0, 0, 0};
    for (int c = 0; c < 4; c++) {
        if (!files[c]) return set_error("bit vector file %d is NULL", c);
    }
    // the four files are read in parallel, as the reference's OpenMP tasks (matrix_sbwt.hpp:70-110)
#pragma omp parallel for num_threads(4)
    for (int c = 0; c < 4; c++) rc[c] = read_vector(files[c], n[c], w[c]);
    for (int c = 0; c < 4; c++)
        if (rc[c]) return set_error("%s", "a bit vector file could not be read (see the file checks)");
    if (n[1] != n[0] || n[2] != n[0] || n[3] != n[0])  // matrix_sbwt.hpp:52-55
        return set_error("The bit vectors have different lengths (%llu, %llu, %llu, %llu).", (unsigned long long)n[0],
                         (unsigned long long)n[1], (unsigned long long)n[2], (unsigned long long)n[3]);
    const u64 *ptrs[4] = {w[0].data(), w[1].data(), w[2].data(), w[3].data()};
    return sbwt_index_from_host(ptrs, n[0], params, out);
}

extern "C" void sbwt_index_free(sbwt_index *ix) {
    if (!ix) return;
    cudaSetDevice(ix->device);
    sbwt::l2_setaside_release(ix);
    cudaFree(ix->d_bits);
    cudaFree(ix->d_lines);
    cudaFree(ix->d_wide);
    cudaFree(ix->d_L0);
    cudaFree(ix->d_L12);
    cudaFree(ix->d_pre);
    cudaFree(ix->d_pre32);
    cudaFree(ix->d_scan);
    cudaFree(ix->d_node);
    cudaFree(ix->d_sel);
    cudaFree(ix->d_back);
    for (int i = 0; i < sbwt_index::kPipeSlots; i++) {
        ix->ws[i].release();
        if (ix->pipe_stream[i]) cudaStreamDestroy(ix->pipe_stream[i]);
    }
    for (auto &e : ix->prof_ev)
        if (e) cudaEventDestroy(e);
    delete ix;
}

extern "C" int sbwt_index_info(const sbwt_index *ix, uint64_t *n_bits, uint64_t C[5], uint32_t *k, uint32_t *p) {
    clear_error();
    if (!ix) return set_error("index is NULL");
    if (n_bits) *n_bits = ix->n;
    if (C) std::memcpy(C, ix->C, sizeof(ix->C));
    if (k) *k = ix->k;
    if (p) *p = ix->p;
    return 0;
}

extern "C" int sbwt_presearch(sbwt_index *ix, uint32_t p) {
    clear_error();
    if (!ix) return set_error("index is NULL");
    SBWT_CHECK_CUDA(cudaSetDevice(ix->device));
    cudaEvent_t e0, e1;
    SBWT_CHECK_CUDA(cudaEventCreate(&e0));
    SBWT_CHECK_CUDA(cudaEventCreate(&e1));
    cudaEventRecord(e0, 0);
    const int rc = run_presearch(ix, p, 0);
    cudaEventRecord(e1, 0);
    if (rc == 0 && cudaEventSynchronize(e1) == cudaSuccess) cudaEventElapsedTime(&ix->build_ms[2], e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return rc;
}

extern "C" int sbwt_build_times(const sbwt_index *ix, float ms[4]) {
    clear_error();
    if (!ix || !ms) return set_error("NULL argument");
    std::memcpy(ms, ix->build_ms, sizeof(ix->build_ms));
    return 0;
}

extern "C" int sbwt_pipeline_bytes(const sbwt_index *ix, uint64_t *h2d, uint64_t *d2h) {
    clear_error();
    if (!ix || !h2d || !d2h) return set_error("NULL argument");
    *h2d = ix->pipe_h2d;
    *d2h = ix->pipe_d2h;
    return 0;
}

extern "C" int sbwt_presearch_export(const sbwt_index *ix, uint64_t *lefts, uint64_t *rights, uint64_t count) {
    clear_error();
    if (!ix || !lefts || !rights) return set_error("NULL argument");
    SBWT_CHECK_CUDA(cudaSetDevice(ix->device));
    return export_presearch(ix, lefts, rights, count);
}

extern "C" int sbwt_rank_export(sbwt_index *ix, uint32_t sb, int32_t kind, int c, uint64_t *L0, uint64_t l0_words,
                                uint64_t *L12, uint64_t l12_words) {
    clear_error();
    if (!ix || !L0 || !L12) return set_error("NULL argument");
    if (c < 0 || c > 3) return set_error("vector index must be 0..3");
    SBWT_CHECK_CUDA(cudaSetDevice(ix->device));
    if (!ix->poppy_ok || ix->sb != sb || ix->kind != kind) SBWT_TRY(build_poppy(ix, sb, kind, 0));
    if (l0_words != ix->l0w || l12_words != ix->l12w)
        return set_error("rank export: expected %llu L0 and %llu L12 words", (unsigned long long)ix->l0w,
                         (unsigned long long)ix->l12w);
    SBWT_CHECK_CUDA(cudaMemcpy(L0, ix->d_L0 + (u64)c * ix->l0w, ix->l0w * sizeof(u64), cudaMemcpyDeviceToHost));
    SBWT_CHECK_CUDA(cudaMemcpy(L12, ix->d_L12 + (u64)c * ix->l12w, ix->l12w * sizeof(u64), cudaMemcpyDeviceToHost));
    return 0;
}

extern "C" int sbwt_configure(sbwt_index *ix, int32_t layout, uint32_t sb, int32_t kind, int32_t shuffles, uint32_t kpt,
                              uint32_t tpk, uint32_t tpb) {
    clear_error();
    if (!ix) return set_error("index is NULL");
    SBWT_CHECK_CUDA(cudaSetDevice(ix->device));
    if (layout == SBWT_LAYOUT_POPPY) {
        if (!ix->poppy_ok || ix->sb != sb || ix->kind != kind) SBWT_TRY(build_poppy(ix, sb, kind, 0));
    } else if (layout == SBWT_LAYOUT_LINES || wide_sectors(layout)) {
        if (!ix->lines_ok) return set_error("the line layout is not available for an index of %llu columns",
                                            (unsigned long long)ix->n);
        if (wide_sectors(layout) && ix->wide_s != wide_sectors(layout)) SBWT_TRY(build_wide(ix, wide_sectors(layout), 0));
    } else {
        return set_error("unknown layout %d", layout);
    }
    if (tpb != SBWT_KEEP && tpb && (tpb % 32 || tpb > 256))
        return set_error("threads_per_block must be a multiple of 32 up to 256");
    if (kpt != SBWT_KEEP && !(kpt == 0 || kpt == 1 || kpt == 2 || kpt == 3 || kpt == 4 || kpt == 6 || kpt == 8))
        return set_error("kmers_per_thread must be 0 (queue-fed), 1, 2, 3, 4, 6 or 8");
    if (tpk != SBWT_KEEP && tpk && !(tpk == 1 || tpk == 2 || tpk == 4))
        return set_error("threads_per_kmer must be 1, 2 or 4");
    KernelShape &sh = ix->shape;
    sh.layout = layout;
    sh.sb = sb;
    sh.kind = kind;
    sh.shuffles = shuffles;
    if (kpt != SBWT_KEEP) sh.kpt = kpt;
    if (tpk != SBWT_KEEP && tpk) sh.tpk = tpk;
    if (tpb != SBWT_KEEP && tpb) sh.tpb = tpb;
    return 0;
}

extern "C" int sbwt_set_walk_options(sbwt_index *ix, uint32_t window, uint32_t blocks_per_sm, int32_t evict,
                                     int32_t l2_persist) {
    clear_error();
    if (!ix) return set_error("index is NULL");
    if (window != SBWT_KEEP && !(window == 64 || window == 128 || window == 256))
        return set_error("window must be 64, 128 or 256 k-mers");
    if (evict != (int32_t)SBWT_KEEP && (evict < 0 || evict > 2)) return set_error("evict must be 0, 1 or 2");
    SBWT_CHECK_CUDA(cudaSetDevice(ix->device));
    KernelShape &sh = ix->shape;
    if (window != SBWT_KEEP) sh.window = window;
    if (blocks_per_sm != SBWT_KEEP) sh.blocks_per_sm = blocks_per_sm;
    if (evict != (int32_t)SBWT_KEEP) sh.evict = evict;
    if (l2_persist != (int32_t)SBWT_KEEP) {
        sh.l2_persist = l2_persist != 0;
        if (!sh.l2_persist && ix->l2_setaside) l2_setaside_release(ix);
    }
    ix->gen++;
    return 0;
}

extern "C" int sbwt_set_search_mode(sbwt_index *ix, int32_t mode) {
    clear_error();
    if (!ix) return set_error("index is NULL");
    if (mode != SBWT_SEARCH_EVERY_KMER && mode != SBWT_SEARCH_SKIP_ABSENT && mode != SBWT_SEARCH_STREAM)
        return set_error("unknown search mode %d", mode);
    SBWT_CHECK_CUDA(cudaSetDevice(ix->device));
    if (mode == SBWT_SEARCH_STREAM && ix->lines_ok) SBWT_TRY(build_stream(ix, 0));
    ix->shape.mode = mode;
    return 0;
}

namespace sbwt {

// Option (KernelShape.l2_persist, environment SBWT_L2_PERSIST=1, tried by
// the autotuner): the search launch carries an access-policy window over the
// current layout's rank lines with the persisting property, and the index
// sizes the device's persisting L2 set-aside to hold them (a CUDA context
// limit, taken on the first such launch and released when the last index
// that took it is freed).  Layouts larger than the set-aside (poppy, or lines
// beyond it) get no window.  Measured on the large workload: 8.64 ms a
// launch against 8.33 ms without (the lines are not what misses L2; the L2
// hit rate stays at 20 %), and 11.4 ms with the set-aside carved out of L2
// but no window, so it is off by default.
namespace {
std::mutex g_l2_mutex;
constexpr int kL2Devices = 64;
int g_l2_users[kL2Devices] = {0};   // live indexes holding the set-aside
size_t g_l2_set[kL2Devices] = {0};  // its size: the largest any of them asked for
}  // namespace

bool l2_window(const sbwt_index *ix, cudaAccessPolicyWindow *w) {
    if (!ix->shape.l2_persist) return false;
    if (ix->l2_setaside == 0) l2_setaside_acquire(const_cast<sbwt_index *>(ix));  // first windowed launch
    if (ix->l2_setaside == 0) return false;
    const void *base = nullptr;
    size_t bytes = 0;
    if (ix->shape.layout == SBWT_LAYOUT_LINES && ix->lines_ok) {
        base = ix->d_lines, bytes = 4ull * ix->lpc * sizeof(ulonglong4);
    } else if (wide_sectors(ix->shape.layout) && ix->wide_s == wide_sectors(ix->shape.layout)) {
        base = ix->d_wide, bytes = 4ull * ix->wide_lpc * ix->wide_s * sizeof(ulonglong4);
    }
    if (!base || bytes > ix->l2_max_window || bytes > ix->l2_max_persist) return false;
    w->base_ptr = const_cast<void *>(base);
    w->num_bytes = bytes;
    w->hitRatio = bytes <= ix->l2_setaside ? 1.0f : (float)ix->l2_setaside / (float)bytes;
    w->hitProp = cudaAccessPropertyPersisting;
    w->missProp = cudaAccessPropertyStreaming;
    return true;
}

int l2_setaside_acquire(sbwt_index *ix) {
    if (!ix->lines_ok || ix->l2_max_persist == 0 || ix->device < 0 || ix->device >= kL2Devices) return 0;
    // the largest line layout this index may search: the 32-byte lines
    const size_t want = std::min<size_t>(4ull * ix->lpc * sizeof(ulonglong4), ix->l2_max_persist);
    std::lock_guard<std::mutex> lk(g_l2_mutex);
    const int d = ix->device;
    const size_t need = std::max(want, g_l2_set[d]);
    if (need != g_l2_set[d]) {
        const cudaError_t e = cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, need);
        if (e != cudaSuccess) {  // no set-aside (for example under MPS): search without the window
            cudaGetLastError();
            return 0;
        }
        g_l2_set[d] = need;
    }
    g_l2_users[d]++;
    ix->l2_setaside = need;
    return 0;
}

void l2_setaside_release(sbwt_index *ix) {
    if (ix->l2_setaside == 0 || ix->device < 0 || ix->device >= kL2Devices) return;
    std::lock_guard<std::mutex> lk(g_l2_mutex);
    const int d = ix->device;
    if (--g_l2_users[d] <= 0) {
        g_l2_users[d] = 0;
        cudaCtxResetPersistingL2Cache();
        cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, 0);
        g_l2_set[d] = 0;
    }
    ix->l2_setaside = 0;
}

void set_gather_policies(const sbwt_index *ix, SearchArgs &a) {
    const u64 half = ix->l2_bytes / 2;
    const u64 pre_bytes = ix->p ? (1ull << (2 * ix->p)) * (ix->pre64 ? 16ull : 8ull) : 0;
    const u64 back_bytes = ix->d_back ? ix->n * 8ull : 0;
    const int ev = ix->shape.evict;
    a.ef_pre = a.runs && ev != 1 && (ev == 2 || pre_bytes > half);
    a.ef_back = a.runs && ev != 1 && (ev == 2 || back_bytes > half);
}

SearchArgs base_args(const sbwt_index *ix, bool rows) {
    SearchArgs a;
    std::memset(&a, 0, sizeof(a));
    a.lines = ix->d_lines;
    a.lpc = ix->lpc;
    a.bits = ix->d_bits;
    a.L0 = ix->d_L0;
    a.L12 = ix->d_L12;
    a.wpv = ix->wpv;
    a.l0w = ix->l0w;
    a.l12w = ix->l12w;
    std::memcpy(a.C, ix->C, sizeof(a.C));
    a.pre = ix->d_pre;
    a.p = ix->p;
    a.k = ix->k;
    a.chunk = search_chunk(ix, rows);
    a.runs = rows && runs_form(ix);
    a.stream = a.runs && stream_form(ix);
    a.index64 = (u32)ix->shape.index64;
    a.pre32 = a.runs ? ix->d_pre32 : nullptr;
    if (a.stream) a.sv = stream_view(ix);
    set_gather_policies(ix, a);
    return a;
}

// Device-resident batch of rows on stream s using workspace w.
int enqueue_rows(sbwt_index *ix, Workspace &w, SearchArgs &a, const uint8_t *d_letters, u64 n_letters, const u64 *d_rows,
                 u64 n_rows, u64 *d_answers, uint32_t *d_member, u64 n_kmers, cudaStream_t s, bool prof);

int search_rows_device(sbwt_index *ix, Workspace &w, const uint8_t *d_letters, u64 n_letters, const u64 *d_rows,
                       u64 n_rows, u64 *d_answers, uint32_t *d_member, u64 n_kmers, cudaStream_t s) {
    if (n_rows == 0 || n_kmers == 0) return 0;
    const u64 n_words = (n_letters + 32 + 31) / 32;
    SearchArgs a = base_args(ix, true);
    if (!d_answers && !a.runs) {  // membership only: the per-k-mer kernels derive it from answers
        SBWT_TRY(grow(w.answers, w.answers_cap, n_kmers));
        d_answers = w.answers;
    }
    SBWT_TRY(grow(w.words, w.words_cap, n_words));
    SBWT_TRY(grow(w.kstart, w.kstart_cap, n_rows + 1));
    SBWT_TRY(grow(w.scan, w.scan_cap, scan_scratch_words(n_rows)));
    SBWT_TRY(grow(w.chunk_row, w.chunk_cap, (n_kmers + a.chunk - 1) / a.chunk));
    SBWT_TRY(grow(w.counter, w.counter_cap, 1));
    const bool prof = ix->prof_on;
    // CUDA graph: the whole chain is captured once and replayed while its
    // parameters stay the same (not on the legacy default stream, not while
    // profiling per phase)
    bool capturing = false;
    if (ix->use_graph && !prof && s != nullptr) {
        const KernelShape &sh = ix->shape;
        const uint64_t key[12] = {(uint64_t)d_letters, n_letters, (uint64_t)d_rows, n_rows, (uint64_t)d_answers,
                                  (uint64_t)d_member, n_kmers, (uint64_t)s, ix->gen,
                                  ((uint64_t)sh.layout << 48) | ((uint64_t)sh.mode << 40) | ((uint64_t)sh.kpt << 32) |
                                      ((uint64_t)sh.tpk << 16) | sh.tpb,
                                  (uint64_t)w.words ^ (uint64_t)w.kstart, (uint64_t)w.chunk_row ^ (uint64_t)w.counter};
        if (w.graph && std::memcmp(key, w.graph_key, sizeof key) == 0) {
            SBWT_CHECK_CUDA(cudaGraphLaunch(w.graph, s));
            return 0;
        }
        if (w.graph) cudaGraphExecDestroy(w.graph);
        w.graph = nullptr;
        std::memcpy(w.graph_key, key, sizeof key);
        SBWT_CHECK_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        capturing = true;
    }
    const int rc = enqueue_rows(ix, w, a, d_letters, n_letters, d_rows, n_rows, d_answers, d_member, n_kmers, s, prof);
    if (capturing) {
        cudaGraph_t g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(s, &g);
        if (rc) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        if (e != cudaSuccess) return set_error("graph capture failed: %s", cudaGetErrorString(e));
        const cudaError_t ei = cudaGraphInstantiate(&w.graph, g, 0);
        cudaGraphDestroy(g);
        if (ei != cudaSuccess) {
            w.graph = nullptr;
            return set_error("graph instantiation failed: %s", cudaGetErrorString(ei));
        }
        SBWT_CHECK_CUDA(cudaGraphLaunch(w.graph, s));
    }
    return rc;
}

int prepare_rows(sbwt_index *ix, Workspace &w, SearchArgs &a, const uint8_t *d_letters, u64 n_letters,
                 const u64 *d_rows, u64 n_rows, u64 n_kmers, cudaStream_t s) {
    (void)ix;
    const u64 n_words = (n_letters + 32 + 31) / 32;
    SBWT_TRY(grow(w.words, w.words_cap, n_words));
    SBWT_TRY(grow(w.kstart, w.kstart_cap, n_rows + 1));
    SBWT_TRY(grow(w.scan, w.scan_cap, scan_scratch_words(n_rows)));
    SBWT_TRY(grow(w.chunk_row, w.chunk_cap, (n_kmers + a.chunk - 1) / a.chunk));
    SBWT_TRY(grow(w.counter, w.counter_cap, 1));
    SBWT_TRY(launch_pack(d_letters, n_letters, w.words, s));
    SBWT_TRY(launch_kstart(d_rows, n_rows, ix->k, w.kstart, w.scan, s));
    SBWT_TRY(launch_chunk_rows(w.kstart, n_rows, n_kmers, a.chunk, w.chunk_row, s));
    a.words = w.words;
    a.positions = nullptr;
    a.row_starts = d_rows;
    a.kstart = w.kstart;
    a.chunk_row = w.chunk_row;
    a.n_rows = n_rows;
    a.max_pos = (n_words - 1) * 32 - 1;
    a.n_kmers = n_kmers;
    a.counter = w.counter;
    return 0;
}

// The kernels of one batch, in stream order.
int enqueue_rows(sbwt_index *ix, Workspace &w, SearchArgs &a, const uint8_t *d_letters, u64 n_letters, const u64 *d_rows,
                 u64 n_rows, u64 *d_answers, uint32_t *d_member, u64 n_kmers, cudaStream_t s, bool prof) {
    const u64 n_words = (n_letters + 32 + 31) / 32;
    if (prof) SBWT_CHECK_CUDA(cudaEventRecord(ix->prof_ev[0], s));
    SBWT_TRY(launch_pack(d_letters, n_letters, w.words, s));
    if (prof) SBWT_CHECK_CUDA(cudaEventRecord(ix->prof_ev[1], s));
    SBWT_TRY(launch_kstart(d_rows, n_rows, ix->k, w.kstart, w.scan, s));
    SBWT_TRY(launch_chunk_rows(w.kstart, n_rows, n_kmers, a.chunk, w.chunk_row, s));
    if (prof) SBWT_CHECK_CUDA(cudaEventRecord(ix->prof_ev[2], s));
    a.words = w.words;
    a.positions = nullptr;
    a.row_starts = d_rows;
    a.kstart = w.kstart;
    a.chunk_row = w.chunk_row;
    a.n_rows = n_rows;
    a.max_pos = (n_words - 1) * 32 - 1;
    a.answers = d_answers;  // NULL (run-walking kernel only): membership bitmap only
    a.n_kmers = n_kmers;
    a.counter = w.counter;
    a.member = a.runs ? d_member : nullptr;  // the run-walking kernel writes the bitmap itself
    const bool member_pass = d_member && !a.runs;
    uint32_t blocks = 0;
    SBWT_TRY(launch_search(ix, a, s, &blocks));
    if (prof) SBWT_CHECK_CUDA(cudaEventRecord(ix->prof_ev[3], s));
    if (member_pass) SBWT_TRY(launch_member_bits(d_answers, n_kmers, d_member, s));
    if (prof) {
        SBWT_CHECK_CUDA(cudaEventRecord(ix->prof_ev[4], s));
        ix->prof_launches = 1 + 3 + 1 + 1 + (member_pass ? 1 : 0);
        ix->prof_blocks = blocks;
        ix->prof_member = member_pass;
    }
    return 0;
}

}  // namespace sbwt

extern "C" int sbwt_search_packed(sbwt_index *ix, const uint64_t *d_kmer_string, uint64_t n_words,
                                  uint64_t *d_positions_in_results_out, uint64_t n_kmers, void *stream) {
    clear_error();
    if (!ix) return set_error("index is NULL");
    if (n_kmers == 0) return 0;
    if (!d_kmer_string || !d_positions_in_results_out) return set_error("NULL device pointer");
    if (n_words < 2) return set_error("the packed k-mer string needs at least 2 words (one of padding)");
    SBWT_CHECK_CUDA(cudaSetDevice(ix->device));
    cudaStream_t s = (cudaStream_t)stream;
    Workspace &w = ix->ws[0];
    SBWT_TRY(grow(w.counter, w.counter_cap, 1));
    const u64 *runs_dev = nullptr;
    if (runs_form(ix)) {
        // runs of consecutive positions go to the run-walking kernel (packed_runs.cu); the run
        // count stays on the device, and of the two launches below only the one it chose searches
        SearchArgs a = base_args(ix, true);
        SBWT_TRY(packed_runs(w, d_positions_in_results_out, n_kmers, a.chunk, s, &runs_dev));
        a.words = d_kmer_string;
        a.positions = nullptr;
        a.row_starts = w.rows;
        a.kstart = w.kstart;
        a.chunk_row = w.chunk_row;
        a.runs_dev = runs_dev;
        a.n_rows = n_kmers / kMinRunKmers;  // the most runs the walk takes (its index-width choice)
        a.max_pos = (n_words - 1) * 32 - 1;
        a.answers = d_positions_in_results_out;
        a.n_kmers = n_kmers;
        a.counter = w.counter;
        SBWT_TRY(launch_search(ix, a, s, nullptr));
    }
    SearchArgs a = base_args(ix, false);
    a.words = d_kmer_string;
    a.positions = d_positions_in_results_out;
    a.runs_dev = runs_dev;
    a.max_pos = (n_words - 1) * 32 - 1;
    a.answers = d_positions_in_results_out;
    a.n_kmers = n_kmers;
    a.counter = w.counter;
    return launch_search(ix, a, s, nullptr);
}

extern "C" int sbwt_pack(const uint8_t *d_letters, uint64_t n_letters, uint64_t *d_words, void *stream) {
    clear_error();
    if (!d_letters && n_letters) return set_error("NULL device pointer");
    if (!d_words) return set_error("NULL device pointer");
    return launch_pack(d_letters, n_letters, d_words, (cudaStream_t)stream);
}

extern "C" int sbwt_search_reads(sbwt_index *ix, const uint8_t *d_letters, uint64_t n_letters,
                                 const uint64_t *d_row_starts, uint64_t n_rows, uint64_t *d_answers,
                                 uint32_t *d_member_bits, uint64_t n_kmers, void *stream) {
    clear_error();
    if (!ix) return set_error("index is NULL");
    if (n_rows && (!d_letters || !d_row_starts)) return set_error("NULL device pointer");
    if (n_kmers && !d_answers && !d_member_bits) return set_error("NULL answers and membership pointers");
    SBWT_CHECK_CUDA(cudaSetDevice(ix->device));
    return search_rows_device(ix, ix->ws[0], d_letters, n_letters, d_row_starts, n_rows, d_answers, d_member_bits,
                              n_kmers, (cudaStream_t)stream);
}

extern "C" int sbwt_set_l2_fetch_granularity(sbwt_index *ix, uint32_t bytes) {
    clear_error();
    if (!ix) return set_error("index is NULL");
    if (bytes != 32 && bytes != 64 && bytes != 128) return set_error("the L2 fetch granularity must be 32, 64 or 128");
    SBWT_CHECK_CUDA(cudaSetDevice(ix->device));
    SBWT_CHECK_CUDA(cudaDeviceSetLimit(cudaLimitMaxL2FetchGranularity, bytes));
    return 0;
}

extern "C" int sbwt_use_graphs(sbwt_index *ix, int on) {
    clear_error();
    if (!ix) return set_error("index is NULL");
    ix->use_graph = on != 0;
    return 0;
}

extern "C" int sbwt_profile_enable(sbwt_index *ix, int on) {
    clear_error();
    if (!ix) return set_error("index is NULL");
    SBWT_CHECK_CUDA(cudaSetDevice(ix->device));
    if (on) {
        for (auto &e : ix->prof_ev)
            if (!e) SBWT_CHECK_CUDA(cudaEventCreate(&e));
    }
    ix->prof_on = on != 0;
    ix->prof_launches = 0;
    return 0;
}

extern "C" int sbwt_profile_read(sbwt_index *ix, sbwt_profile *out) {
    clear_error();
    if (!ix || !out) return set_error("NULL argument");
    if (!ix->prof_on || ix->prof_launches == 0) return set_error("no profiled call (sbwt_profile_enable first)");
    SBWT_CHECK_CUDA(cudaSetDevice(ix->device));
    SBWT_CHECK_CUDA(cudaEventSynchronize(ix->prof_ev[4]));
    float t[4];
    for (int i = 0; i < 4; i++) SBWT_CHECK_CUDA(cudaEventElapsedTime(&t[i], ix->prof_ev[i], ix->prof_ev[i + 1]));
    out->pack_ms = t[0];
    out->table_ms = t[1];
    out->search_ms = t[2];
    out->member_ms = ix->prof_member ? t[3] : 0.0f;
    out->launches = ix->prof_launches;
    out->search_blocks = ix->prof_blocks;
    return 0;
}

extern "C" uint64_t sbwt_count_kmers(const uint64_t *row_starts, uint64_t n_rows, uint32_t k) {
    uint64_t t = 0;
#pragma omp parallel for schedule(static) reduction(+ : t) if (n_rows > (1u << 16))
    for (int64_t r = 0; r < (int64_t)n_rows; r++) {
        const uint64_t len = row_starts[r + 1] - row_starts[r];
        if (len >= k) t += len - k + 1;
    }
    return t;
}
