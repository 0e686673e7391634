// prefilter.cu -- the learned-Bloom sandwich in front of the exact search
// (no reference counterpart).
//
// Training: candidates are sampled from the index itself (k-mers of random
// nodes, reconstructed by select walks) and as negatives (uniform random
// k-mers, and indexed k-mers with 1-3 substitutions); every candidate is
// labelled by the exact search.  The MLP (one-hot 4k -> 256 -> 256 -> 1,
// BF16, FP32 accumulation) is trained with binary cross-entropy and Adam by
// this project's own kernels (mlp.cu); one step is captured in a CUDA graph
// and replayed.
//
// Filtering: a k-mer whose logit is below tau is checked against a Bloom
// filter holding every indexed k-mer the model rejects; only if the filter
// also rejects it is its answer set to "absent" without a search.  An
// indexed k-mer is therefore never reported absent, and every answer equals
// the plain search's.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "internal.h"
#include "mlp.h"
#include "mlp_kernels.cuh"

using namespace sbwt;
using namespace sbwt::mlp;

struct sbwt_prefilter {
    int device = 0;
    uint32_t k = 31;
    MlpOffsets off;
    float *theta = nullptr;  // FP32 parameters
    bf16 *W1b = nullptr, *W2b = nullptr;
    uint32_t *bloom = nullptr;
    uint64_t bloom_mask = 0;
    uint32_t bloom_hashes = 3;
    float tau = 0.0f;
    int *d_err = nullptr;
    float *d_logits = nullptr;
    size_t logits_cap = 0;
    unsigned long long *d_skipped = nullptr;
    // prefiltered searches of reads: the reject bitmap of the batch and a
    // chunk of its k-mers as a list (the inference input)
    uint32_t *d_reject = nullptr;
    size_t reject_cap = 0;
    uint64_t *d_klist = nullptr;
    size_t klist_cap = 0;
    // host copy of the trained biases and output weights (inference parameters)
    sbwt::mlp::InferBias bias{};
    sbwt_prefilter_stats stats{};
};

namespace sbwt {
namespace mlp {
namespace {

// ------------------------------------------------------- training state

struct Train {
    uint32_t B = 0, k = 31;
    uint64_t n_train = 0;
    MlpOffsets off;
    const uint64_t *kmers = nullptr;
    const uint8_t *labels = nullptr;
    float *theta = nullptr, *grad = nullptr, *m = nullptr, *v = nullptr;
    bf16 *W1b = nullptr, *W2b = nullptr, *W2bT = nullptr;
    bf16 *X = nullptr, *XT = nullptr, *H1 = nullptr, *H1T = nullptr, *dZ2 = nullptr, *dZ2T = nullptr, *dZ1 = nullptr,
         *dZ1T = nullptr;
    float *Y = nullptr, *Z1 = nullptr, *Z2 = nullptr, *dH1 = nullptr;
    float *loss_sum = nullptr, *loss_hist = nullptr;
    unsigned long long *step = nullptr;
    int *err = nullptr;
    std::vector<void *> owned;

    template <class T>
    int alloc(T *&p, size_t count) {
        SBWT_CHECK_CUDA(cudaMalloc((void **)&p, std::max<size_t>(count, 1) * sizeof(T)));
        owned.push_back((void *)p);
        return 0;
    }
    int setup(uint32_t batch, uint32_t kk, uint32_t hist) {
        B = batch;
        k = kk;
        const uint32_t P = off.count;
        SBWT_TRY(alloc(theta, P));
        SBWT_TRY(alloc(grad, P));
        SBWT_TRY(alloc(m, P));
        SBWT_TRY(alloc(v, P));
        SBWT_TRY(alloc(W1b, 256 * 128));
        SBWT_TRY(alloc(W2b, 256 * 256));
        SBWT_TRY(alloc(W2bT, 256 * 256));
        SBWT_TRY(alloc(X, (size_t)B * kIn));
        SBWT_TRY(alloc(XT, (size_t)B * kIn));
        SBWT_TRY(alloc(H1, (size_t)B * kHid));
        SBWT_TRY(alloc(H1T, (size_t)B * kHid));
        SBWT_TRY(alloc(dZ2, (size_t)B * kHid));
        SBWT_TRY(alloc(dZ2T, (size_t)B * kHid));
        SBWT_TRY(alloc(dZ1, (size_t)B * kHid));
        SBWT_TRY(alloc(dZ1T, (size_t)B * kHid));
        SBWT_TRY(alloc(Y, B));
        SBWT_TRY(alloc(Z1, (size_t)B * kHid));
        SBWT_TRY(alloc(Z2, (size_t)B * kHid));
        SBWT_TRY(alloc(dH1, (size_t)B * kHid));
        SBWT_TRY(alloc(loss_sum, 1));
        SBWT_TRY(alloc(loss_hist, hist + 2));
        SBWT_TRY(alloc(step, 1));
        SBWT_TRY(alloc(err, 1));
        SBWT_CHECK_CUDA(cudaMemset(m, 0, P * sizeof(float)));
        SBWT_CHECK_CUDA(cudaMemset(v, 0, P * sizeof(float)));
        SBWT_CHECK_CUDA(cudaMemset(step, 0, sizeof(*step)));
        SBWT_CHECK_CUDA(cudaMemset(err, 0, sizeof(*err)));
        SBWT_CHECK_CUDA(cudaMemset(loss_hist, 0, (hist + 2) * sizeof(float)));
        return 0;
    }
    // the BF16 operand copies of W1 and W2 from theta
    int refresh_bf16(cudaStream_t s) {
        to_bf16_kernel<<<(256 * 128 + 255) / 256, 256, 0, s>>>(theta + off.W1, W1b, 256 * 128);
        to_bf16_kernel<<<(256 * 256 + 255) / 256, 256, 0, s>>>(theta + off.W2, W2b, 256 * 256);
        SBWT_CHECK_CUDA(cudaGetLastError());
        return 0;
    }
    ~Train() {
        for (void *p : owned) cudaFree(p);
    }
};

// One training step (forward, loss, backward, and optionally Adam).
int enqueue_step(Train &t, cudaStream_t s, bool adam, float lr, uint32_t hist_every) {
    const uint32_t B = t.B;
    const int splits = std::max<int>(1, (int)(B / 256));
    SBWT_CHECK_CUDA(cudaMemsetAsync(t.grad, 0, t.off.count * sizeof(float), s));
    SBWT_CHECK_CUDA(cudaMemsetAsync(t.loss_sum, 0, sizeof(float), s));
    onehot_batch_kernel<<<(B + 127) / 128, 128, 0, s>>>(t.kmers, t.labels, t.n_train, t.step, B, t.k, t.X, t.Y);
    SBWT_TRY(gemm_tn(t.X, t.W1b, t.Z1, B, kHid, kIn, 1, t.err, s));  // Z1 = X W1^T
    bias_relu_kernel<<<(unsigned)(((size_t)B * kHid + 255) / 256), 256, 0, s>>>(t.Z1, t.theta + t.off.b1, t.H1,
                                                                                (size_t)B * kHid);
    SBWT_TRY(gemm_tn(t.H1, t.W2b, t.Z2, B, kHid, kHid, 1, t.err, s));  // Z2 = H1 W2^T
    head_kernel<<<(B + 7) / 8, 256, 0, s>>>(t.Z2, t.theta, t.Y, B, t.dZ2, t.grad, t.loss_sum, t.off);
    SBWT_TRY(transpose(t.W2b, t.W2bT, kHid, kHid, s));
    SBWT_TRY(gemm_tn(t.dZ2, t.W2bT, t.dH1, B, kHid, kHid, 1, t.err, s));  // dH1 = dZ2 W2
    relu_grad_kernel<<<(B + 7) / 8, 256, 0, s>>>(t.dH1, t.H1, B, t.dZ1, t.grad, t.off);
    SBWT_TRY(transpose(t.dZ2, t.dZ2T, B, kHid, s));
    SBWT_TRY(transpose(t.H1, t.H1T, B, kHid, s));
    SBWT_TRY(gemm_tn(t.dZ2T, t.H1T, t.grad + t.off.W2, kHid, kHid, B, splits, t.err, s));  // dW2 = dZ2^T H1
    SBWT_TRY(transpose(t.dZ1, t.dZ1T, B, kHid, s));
    SBWT_TRY(transpose(t.X, t.XT, B, kIn, s));
    SBWT_TRY(gemm_tn(t.dZ1T, t.XT, t.grad + t.off.W1, kHid, kIn, B, splits, t.err, s));  // dW1 = dZ1^T X
    if (adam) {
        adam_kernel<<<(t.off.count + 255) / 256, 256, 0, s>>>(t.theta, t.grad, t.m, t.v, t.step, t.off.count, lr, t.k,
                                                             t.W1b, t.W2b, t.off);
        step_kernel<<<1, 1, 0, s>>>(t.step, t.loss_hist, t.loss_sum, hist_every);
    }
    SBWT_CHECK_CUDA(cudaGetLastError());
    return 0;
}

// PyTorch-style default initialisation: U(-1/sqrt(fan_in), 1/sqrt(fan_in))
// for weights and biases, from a seeded splitmix64 stream.
std::vector<float> init_theta(const MlpOffsets &off, uint32_t k, uint64_t seed) {
    std::vector<float> th(off.count, 0.0f);
    uint64_t st = seed;
    auto uni = [&](float bound) {
        st += 0x9E3779B97F4A7C15ull;
        const double u = (double)(mix64(st) >> 11) * (1.0 / 9007199254740992.0);
        return (float)((2.0 * u - 1.0) * bound);
    };
    const float bi = 1.0f / std::sqrt((float)(4 * k)), bh = 1.0f / 16.0f;
    for (uint32_t o = 0; o < 256; o++)
        for (uint32_t i = 0; i < 128; i++) th[off.W1 + o * 128 + i] = i < 4 * k ? uni(bi) : 0.0f;
    for (uint32_t o = 0; o < 256; o++) th[off.b1 + o] = uni(bi);
    for (uint32_t i = 0; i < 256 * 256; i++) th[off.W2 + i] = uni(bh);
    for (uint32_t o = 0; o < 256; o++) th[off.b2 + o] = uni(bh);
    for (uint32_t o = 0; o < 256; o++) th[off.w3 + o] = uni(bh);
    th[off.b3] = uni(bh);
    return th;
}

int check_err(const int *d_err, const char *what) {
    int e = 0;
    SBWT_CHECK_CUDA(cudaMemcpy(&e, d_err, sizeof(e), cudaMemcpyDeviceToHost));
    if (e) return set_error("%s: a tensor-core wait timed out (code %d)", what, e);
    return 0;
}

C5 c5_of(const sbwt_index *ix) {
    C5 c;
    for (int i = 0; i < 5; i++) c.c[i] = ix->C[i];
    return c;
}

// Exact answers of a k-mer list (kmer-list mode of the search kernel).
int search_list(sbwt_index *ix, const uint64_t *d_kmers, uint64_t n, uint64_t *d_answers, const float *logits,
                const sbwt_prefilter *pf, unsigned long long *skipped, cudaStream_t s);

}  // namespace
}  // namespace mlp
}  // namespace sbwt

namespace sbwt {
namespace mlp {
namespace {

int search_list(sbwt_index *ix, const uint64_t *d_kmers, uint64_t n, uint64_t *d_answers, const float *logits,
                const sbwt_prefilter *pf, unsigned long long *skipped, cudaStream_t s) {
    if (n == 0) return 0;
    Workspace &w = ix->ws[0];
    SBWT_TRY(grow(w.counter, w.counter_cap, 1));
    SearchArgs a = base_args(ix, false);
    a.kmer_list = d_kmers;
    a.answers = d_answers;
    a.n_kmers = n;
    a.counter = w.counter;
    if (logits && pf) {
        a.logits = logits;
        a.tau = pf->tau;
        a.bloom_bits = pf->bloom;
        a.bloom_mask = pf->bloom_mask;
        a.bloom_hashes = pf->bloom_hashes;
        a.skipped = skipped;
    }
    return launch_search(ix, a, s, nullptr);
}

}  // namespace
}  // namespace mlp
}  // namespace sbwt

extern "C" int sbwt_mlp_params_default(sbwt_mlp_params *p) {
    if (!p) return set_error("params is NULL");
    std::memset(p, 0, sizeof(*p));
    p->steps = 20000;
    p->batch = 8192;
    p->lr = 1e-3f;
    p->n_positive = 50000000ull;
    p->n_negative = 50000000ull;
    p->seed = 1234;
    p->tau = 0.0f;
    p->bloom_fpr = 0.01f;
    p->bloom_hashes = 3;
    return 0;
}

extern "C" int sbwt_prefilter_train(sbwt_index *ix, const sbwt_mlp_params *prm, sbwt_prefilter **out) {
    clear_error();
    if (!ix || !out) return set_error("NULL argument");
    *out = nullptr;
    sbwt_mlp_params def;
    sbwt_mlp_params_default(&def);
    if (!prm) prm = &def;
    if (!ix->lines_ok) return set_error("the prefilter needs the line layout (index of fewer than 3.7e9 columns)");
    if (prm->batch == 0 || prm->batch % 256) return set_error("batch must be a positive multiple of 256");
    if (prm->bloom_hashes < 1 || prm->bloom_hashes > 16) return set_error("bloom_hashes must be in [1, 16]");
    if (!(prm->bloom_fpr > 0.0f && prm->bloom_fpr < 1.0f)) return set_error("bloom_fpr must be in (0, 1)");
    if (ix->n >= (1ull << 32)) return set_error("the prefilter samples nodes with 32-bit indices");
    SBWT_CHECK_CUDA(cudaSetDevice(ix->device));
    const auto t0 = std::chrono::steady_clock::now();
    cudaStream_t s = nullptr;
    SBWT_CHECK_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    sbwt_prefilter *pf = new sbwt_prefilter();
    pf->device = ix->device;
    pf->k = ix->k;
    pf->tau = prm->tau;
    pf->bloom_hashes = prm->bloom_hashes;
    int rc = 0;
    uint64_t *d_train = nullptr, *d_ans = nullptr, *d_all = nullptr;
    uint8_t *d_labels = nullptr;
    unsigned long long *d_cnt = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    do {
        const uint64_t want = prm->n_positive + prm->n_negative;
        const uint64_t n_train = std::max<uint64_t>(want / prm->batch, 1) * prm->batch;
        if ((rc = (cudaMalloc(&d_train, n_train * 8) != cudaSuccess))) { rc = set_error("out of device memory (training set)"); break; }
        if (cudaMalloc(&d_ans, n_train * 8) != cudaSuccess || cudaMalloc(&d_labels, n_train) != cudaSuccess ||
            cudaMalloc(&d_cnt, 4 * sizeof(unsigned long long)) != cudaSuccess ||
            cudaMalloc(&pf->d_err, sizeof(int)) != cudaSuccess ||
            cudaMalloc(&pf->d_skipped, sizeof(unsigned long long)) != cudaSuccess) {
            rc = set_error("out of device memory (training set)");
            break;
        }
        cudaMemsetAsync(d_cnt, 0, 4 * sizeof(unsigned long long), s);
        cudaMemsetAsync(pf->d_err, 0, sizeof(int), s);
        const C5 c5 = c5_of(ix);
        sample_kernel<<<(unsigned)((n_train + 255) / 256), 256, 0, s>>>(
            ix->d_lines, ix->lpc, c5, (uint32_t)ix->n, ix->k, prm->n_positive, std::max<uint64_t>(prm->n_negative, 0),
            prm->seed, n_train, d_train);
        if ((rc = search_list(ix, d_train, n_train, d_ans, nullptr, nullptr, nullptr, s)) != 0) break;
        labels_kernel<<<(unsigned)((n_train + 255) / 256), 256, 0, s>>>(d_ans, n_train, d_labels, d_cnt);
        // model state
        Train t;
        t.n_train = n_train;
        t.kmers = d_train;
        t.labels = d_labels;
        const uint32_t hist_every = 100;
        if ((rc = t.setup(prm->batch, ix->k, prm->steps / hist_every + 1)) != 0) break;
        const std::vector<float> th0 = init_theta(t.off, ix->k, prm->seed ^ 0xA5A5A5A5ull);
        SBWT_CHECK_CUDA(cudaMemcpyAsync(t.theta, th0.data(), th0.size() * sizeof(float), cudaMemcpyHostToDevice, s));
        if ((rc = t.refresh_bf16(s)) != 0) break;
        // one step, captured once, replayed
        if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
            rc = set_error("training: graph capture failed to start");
            break;
        }
        rc = enqueue_step(t, s, true, prm->lr, hist_every);
        cudaError_t ce = cudaStreamEndCapture(s, &graph);
        if (rc) break;
        if (ce != cudaSuccess || cudaGraphInstantiate(&exec, graph, 0) != cudaSuccess) {
            rc = set_error("training: graph capture failed: %s", cudaGetErrorString(ce));
            break;
        }
        const auto tt = std::chrono::steady_clock::now();
        for (uint32_t i = 0; i < prm->steps && rc == 0; i++)
            if (cudaGraphLaunch(exec, s) != cudaSuccess) rc = set_error("training: graph launch failed");
        if (rc) break;
        SBWT_CHECK_CUDA(cudaStreamSynchronize(s));
        pf->stats.train_ms = (float)std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tt).count();
        if ((rc = check_err(t.err, "training")) != 0) break;
        SBWT_CHECK_CUDA(cudaMemcpy(&pf->stats.final_loss, t.loss_sum, sizeof(float), cudaMemcpyDeviceToHost));
        {
            float l0 = 0;
            SBWT_CHECK_CUDA(cudaMemcpy(&l0, t.loss_hist, sizeof(float), cudaMemcpyDeviceToHost));
            pf->stats.first_loss = l0;
        }
        // keep the trained parameters
        SBWT_CHECK_CUDA(cudaMalloc(&pf->theta, t.off.count * sizeof(float)));
        SBWT_CHECK_CUDA(cudaMalloc(&pf->W1b, 256 * 128 * sizeof(bf16)));
        SBWT_CHECK_CUDA(cudaMalloc(&pf->W2b, 256 * 256 * sizeof(bf16)));
        SBWT_CHECK_CUDA(cudaMemcpyAsync(pf->theta, t.theta, t.off.count * sizeof(float), cudaMemcpyDeviceToDevice, s));
        SBWT_CHECK_CUDA(cudaMemcpyAsync(pf->W1b, t.W1b, 256 * 128 * sizeof(bf16), cudaMemcpyDeviceToDevice, s));
        SBWT_CHECK_CUDA(cudaMemcpyAsync(pf->W2b, t.W2b, 256 * 256 * sizeof(bf16), cudaMemcpyDeviceToDevice, s));
        {
            std::vector<float> th(t.off.count);
            SBWT_CHECK_CUDA(cudaMemcpyAsync(th.data(), t.theta, t.off.count * sizeof(float), cudaMemcpyDeviceToHost, s));
            SBWT_CHECK_CUDA(cudaStreamSynchronize(s));
            bias_from_host(th.data(), t.off, pf->bias);
        }
        // accuracy on the training candidates (first min(n, 4M)) at tau
        {
            const uint64_t na = std::min<uint64_t>(n_train, 4u << 20);
            float *lg = nullptr;
            SBWT_CHECK_CUDA(cudaMalloc(&lg, na * sizeof(float)));
            rc = infer(d_train, na, ix->k, pf->W1b, pf->W2b, pf->bias, logits_only(lg), pf->d_err, ix->num_sms, s);
            if (rc == 0) {
                accuracy_kernel<<<(unsigned)((na + 255) / 256), 256, 0, s>>>(lg, d_labels, na, pf->tau, d_cnt + 1);
                unsigned long long cnt[2];
                cudaMemcpyAsync(cnt, d_cnt, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s);
                cudaStreamSynchronize(s);
                pf->stats.train_accuracy = (double)cnt[1] / (double)na;
                pf->stats.label_positive_fraction = (double)cnt[0] / (double)n_train;
            }
            cudaFree(lg);
            if (rc) break;
        }
        // Bloom filter over every indexed k-mer the model rejects
        const uint64_t nodes = ix->n - 1;
        if (cudaMalloc(&d_all, nodes * 8) != cudaSuccess) { rc = set_error("out of device memory (k-mer list)"); break; }
        float *lg = nullptr;
        SBWT_CHECK_CUDA(cudaMalloc(&lg, nodes * sizeof(float)));
        enumerate_kernel<<<(unsigned)((nodes + 255) / 256), 256, 0, s>>>(ix->d_lines, ix->lpc, c5, (uint32_t)ix->n,
                                                                         ix->k, d_all);
        rc = infer(d_all, nodes, ix->k, pf->W1b, pf->W2b, pf->bias, logits_only(lg), pf->d_err, ix->num_sms, s);
        if (rc == 0) {
            cudaMemsetAsync(d_cnt + 2, 0, sizeof(unsigned long long), s);
            bloom_build_kernel<<<(unsigned)((nodes + 255) / 256), 256, 0, s>>>(d_all, lg, nodes, pf->tau, ix->k,
                                                                                nullptr, 0, prm->bloom_hashes, d_cnt + 2);
            unsigned long long rej = 0;
            cudaMemcpyAsync(&rej, d_cnt + 2, sizeof(rej), cudaMemcpyDeviceToHost, s);
            cudaStreamSynchronize(s);
            // m bits for false-positive rate f with h hashes: m = -h n / ln(1 - f^(1/h))
            const double h = prm->bloom_hashes;
            const double mbits = std::max(1024.0, -h * (double)std::max<unsigned long long>(rej, 1) /
                                                      std::log(1.0 - std::pow((double)prm->bloom_fpr, 1.0 / h)));
            uint64_t m = 1024;
            while ((double)m < mbits) m <<= 1;
            if (cudaMalloc(&pf->bloom, m / 8) != cudaSuccess) rc = set_error("out of device memory (Bloom filter)");
            if (rc == 0) {
                cudaMemsetAsync(pf->bloom, 0, m / 8, s);
                pf->bloom_mask = m - 1;
                cudaMemsetAsync(d_cnt + 3, 0, sizeof(unsigned long long), s);
                bloom_build_kernel<<<(unsigned)((nodes + 255) / 256), 256, 0, s>>>(
                    d_all, lg, nodes, pf->tau, ix->k, pf->bloom, pf->bloom_mask, prm->bloom_hashes, d_cnt + 3);
                unsigned long long cnt[2];
                cudaMemcpyAsync(cnt, d_cnt + 2, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s);
                cudaStreamSynchronize(s);
                pf->stats.n_rejected_indexed = cnt[1];
                pf->stats.bloom_bits = m;
            }
        }
        cudaFree(lg);
        if (rc) break;
        rc = check_err(pf->d_err, "prefilter inference");
        if (rc) break;
        // indexed k-mers = nodes that are not dummies (counted only: d_labels holds the n_train
        // training labels, fewer than the nodes of a large index)
        {
            unsigned long long *cnt = d_cnt;
            cudaMemsetAsync(cnt, 0, sizeof(unsigned long long), s);
            labels_kernel<<<(unsigned)((nodes + 255) / 256), 256, 0, s>>>(d_all, nodes, nullptr, cnt);
            unsigned long long c = 0;
            cudaMemcpyAsync(&c, cnt, sizeof(c), cudaMemcpyDeviceToHost, s);
            cudaStreamSynchronize(s);
            pf->stats.n_indexed_kmers = c;
        }
        pf->stats.n_train = n_train;
        pf->stats.total_ms = (float)std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    } while (false);
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    cudaFree(d_train);
    cudaFree(d_ans);
    cudaFree(d_all);
    cudaFree(d_labels);
    cudaFree(d_cnt);
    cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
    if (rc) {
        sbwt_prefilter_free(pf);
        return rc;
    }
    *out = pf;
    return 0;
}

extern "C" void sbwt_prefilter_free(sbwt_prefilter *pf) {
    if (!pf) return;
    cudaSetDevice(pf->device);
    cudaFree(pf->theta);
    cudaFree(pf->W1b);
    cudaFree(pf->W2b);
    cudaFree(pf->bloom);
    cudaFree(pf->d_reject);
    cudaFree(pf->d_klist);
    cudaFree(pf->d_err);
    cudaFree(pf->d_logits);
    cudaFree(pf->d_skipped);
    delete pf;
}

extern "C" int sbwt_prefilter_stats_get(const sbwt_prefilter *pf, sbwt_prefilter_stats *out) {
    clear_error();
    if (!pf || !out) return set_error("NULL argument");
    *out = pf->stats;
    return 0;
}

extern "C" int sbwt_prefilter_params(const sbwt_prefilter *pf, float *theta, uint64_t count) {
    clear_error();
    if (!pf || !theta) return set_error("NULL argument");
    if (count != pf->off.count) return set_error("the parameter vector has %u floats", pf->off.count);
    SBWT_CHECK_CUDA(cudaSetDevice(pf->device));
    SBWT_CHECK_CUDA(cudaMemcpy(theta, pf->theta, count * sizeof(float), cudaMemcpyDeviceToHost));
    return 0;
}

extern "C" int sbwt_prefilter_logits(sbwt_prefilter *pf, const uint64_t *d_kmers, uint64_t n, float *d_logits,
                                     void *stream) {
    clear_error();
    if (!pf) return set_error("prefilter is NULL");
    if (n && (!d_kmers || !d_logits)) return set_error("NULL device pointer");
    SBWT_CHECK_CUDA(cudaSetDevice(pf->device));
    int dev_sms = 0;
    cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, pf->device);
    return infer(d_kmers, n, pf->k, pf->W1b, pf->W2b, pf->bias, logits_only(d_logits), pf->d_err, dev_sms,
                 (cudaStream_t)stream);
}

extern "C" int sbwt_search_kmers(sbwt_index *ix, const uint64_t *d_kmers, uint64_t n, uint64_t *d_answers,
                                 void *stream) {
    clear_error();
    if (!ix) return set_error("index is NULL");
    if (n && (!d_kmers || !d_answers)) return set_error("NULL device pointer");
    SBWT_CHECK_CUDA(cudaSetDevice(ix->device));
    return search_list(ix, d_kmers, n, d_answers, nullptr, nullptr, nullptr, (cudaStream_t)stream);
}

extern "C" int sbwt_search_kmers_filtered(sbwt_index *ix, sbwt_prefilter *pf, const uint64_t *d_kmers, uint64_t n,
                                          uint64_t *d_answers, uint64_t *n_skipped, void *stream) {
    clear_error();
    if (!ix || !pf) return set_error("NULL argument");
    if (pf->k != ix->k) return set_error("the prefilter was trained for k = %u", pf->k);
    if (n == 0) {
        if (n_skipped) *n_skipped = 0;
        return 0;
    }
    if (!d_kmers || !d_answers) return set_error("NULL device pointer");
    SBWT_CHECK_CUDA(cudaSetDevice(ix->device));
    cudaStream_t s = (cudaStream_t)stream;
    if (pf->logits_cap < n) {
        cudaFree(pf->d_logits);
        pf->d_logits = nullptr;
        pf->logits_cap = 0;
        SBWT_CHECK_CUDA(cudaMalloc(&pf->d_logits, n * sizeof(float)));
        pf->logits_cap = n;
    }
    SBWT_TRY(infer(d_kmers, n, pf->k, pf->W1b, pf->W2b, pf->bias, logits_only(pf->d_logits), pf->d_err,
                   ix->num_sms, s));
    SBWT_CHECK_CUDA(cudaMemsetAsync(pf->d_skipped, 0, sizeof(unsigned long long), s));
    SBWT_TRY(search_list(ix, d_kmers, n, d_answers, pf->d_logits, pf, pf->d_skipped, s));
    if (n_skipped) {
        unsigned long long c = 0;
        SBWT_CHECK_CUDA(cudaMemcpyAsync(&c, pf->d_skipped, sizeof(c), cudaMemcpyDeviceToHost, s));
        SBWT_CHECK_CUDA(cudaStreamSynchronize(s));
        *n_skipped = c;
        int e = 0;
        SBWT_CHECK_CUDA(cudaMemcpy(&e, pf->d_err, sizeof(e), cudaMemcpyDeviceToHost));
        if (e) return set_error("prefilter inference: a tensor-core wait timed out (code %d)", e);
    }
    return 0;
}

namespace {
// k-mers per inference pass of a prefiltered search of reads (the list is
// 8 bytes a k-mer); a multiple of the 128-k-mer tile.  Environment:
// SBWT_FILTER_CHUNK_KMERS sets another size (rounded up to 128).
uint64_t filter_chunk() {
    uint64_t c = 64ull << 20;
    if (const char *e = std::getenv("SBWT_FILTER_CHUNK_KMERS")) {
        const unsigned long long v = std::strtoull(e, nullptr, 10);
        if (v) c = (v + 127) / 128 * 128;
    }
    return c;
}
}  // namespace

extern "C" int sbwt_search_reads_filtered(sbwt_index *ix, sbwt_prefilter *pf, const uint8_t *d_letters,
                                          uint64_t n_letters, const uint64_t *d_row_starts, uint64_t n_rows,
                                          uint64_t *d_answers, uint32_t *d_member_bits, uint64_t n_kmers,
                                          uint64_t *n_skipped, void *stream) {
    clear_error();
    if (!ix || !pf) return set_error("NULL argument");
    if (pf->k != ix->k) return set_error("the prefilter was trained for k = %u", pf->k);
    if (n_skipped) *n_skipped = 0;
    if (n_rows == 0 || n_kmers == 0) return 0;
    if (!d_letters || !d_row_starts) return set_error("NULL device pointer");
    if (!d_answers && !d_member_bits) return set_error("NULL answers and membership pointers");
    SBWT_CHECK_CUDA(cudaSetDevice(ix->device));
    cudaStream_t s = (cudaStream_t)stream;
    Workspace &w = ix->ws[0];
    SearchArgs a = base_args(ix, true);
    if (!a.runs || ix->shape.layout != SBWT_LAYOUT_LINES)
        return set_error("the prefiltered search of reads needs the run walk on the line layout "
                         "(search mode stream or skip, one lane per k-mer, queue-fed)");
    SBWT_TRY(prepare_rows(ix, w, a, d_letters, n_letters, d_row_starts, n_rows, n_kmers, s));
    const uint64_t words = (n_kmers + 31) / 32;
    SBWT_TRY(grow(pf->d_reject, pf->reject_cap, words));
    const uint64_t chunk = filter_chunk();
    SBWT_TRY(grow(pf->d_klist, pf->klist_cap, std::min(n_kmers, chunk)));
    // the sandwich's decision for every k-mer of the batch: model at tau, then the backup Bloom filter
    const InferOut out{nullptr, nullptr, pf->tau, pf->bloom, pf->bloom_mask, pf->bloom_hashes};
    for (uint64_t j0 = 0; j0 < n_kmers; j0 += chunk) {
        const uint64_t cnt = std::min(chunk, n_kmers - j0);
        SBWT_TRY(launch_kmer_list(a, j0, cnt, pf->d_klist, s));
        InferOut o = out;
        o.reject = pf->d_reject + j0 / 32;
        SBWT_TRY(infer(pf->d_klist, cnt, pf->k, pf->W1b, pf->W2b, pf->bias, o, pf->d_err, ix->num_sms, s));
    }
    SBWT_CHECK_CUDA(cudaMemsetAsync(pf->d_skipped, 0, sizeof(unsigned long long), s));
    a.reject = pf->d_reject;
    a.skipped = pf->d_skipped;
    a.answers = d_answers;
    a.member = d_member_bits;
    SBWT_TRY(launch_search(ix, a, s, nullptr));
    if (n_skipped) {
        unsigned long long c = 0;
        SBWT_CHECK_CUDA(cudaMemcpyAsync(&c, pf->d_skipped, sizeof(c), cudaMemcpyDeviceToHost, s));
        SBWT_CHECK_CUDA(cudaStreamSynchronize(s));
        *n_skipped = c;
        int e = 0;
        SBWT_CHECK_CUDA(cudaMemcpy(&e, pf->d_err, sizeof(e), cudaMemcpyDeviceToHost));
        if (e) return set_error("prefilter inference: a tensor-core wait timed out (code %d)", e);
    }
    return 0;
}

extern "C" int sbwt_mlp_gradients(uint32_t k, const float *theta, const uint64_t *kmers, const uint8_t *labels,
                                  uint32_t n, float *loss, float *grad) {
    clear_error();
    if (!theta || !kmers || !labels || !grad) return set_error("NULL argument");
    if (n == 0 || n % 256) return set_error("n must be a positive multiple of 256");
    if (k < 3 || k > 32) return set_error("k must be in [3, 32]");
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) return set_error("no CUDA device is available");
    Train t;
    SBWT_TRY(t.setup(n, k, 1));
    uint64_t *d_k = nullptr;
    uint8_t *d_l = nullptr;
    SBWT_TRY(t.alloc(d_k, n));
    SBWT_TRY(t.alloc(d_l, n));
    t.kmers = d_k;
    t.labels = d_l;
    t.n_train = n;
    SBWT_CHECK_CUDA(cudaMemcpy(d_k, kmers, (size_t)n * 8, cudaMemcpyHostToDevice));
    SBWT_CHECK_CUDA(cudaMemcpy(d_l, labels, n, cudaMemcpyHostToDevice));
    SBWT_CHECK_CUDA(cudaMemcpy(t.theta, theta, t.off.count * sizeof(float), cudaMemcpyHostToDevice));
    SBWT_TRY(t.refresh_bf16(0));
    SBWT_TRY(enqueue_step(t, 0, false, 0.0f, 0));
    SBWT_CHECK_CUDA(cudaDeviceSynchronize());
    SBWT_TRY(check_err(t.err, "gradients"));
    SBWT_CHECK_CUDA(cudaMemcpy(grad, t.grad, t.off.count * sizeof(float), cudaMemcpyDeviceToHost));
    if (loss) SBWT_CHECK_CUDA(cudaMemcpy(loss, t.loss_sum, sizeof(float), cudaMemcpyDeviceToHost));
    return 0;
}

extern "C" int sbwt_mlp_logits(uint32_t k, const float *theta, const uint64_t *kmers, uint64_t n, float *logits) {
    clear_error();
    if (!theta || !kmers || !logits) return set_error("NULL argument");
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) return set_error("no CUDA device is available");
    MlpOffsets off;
    float *d_th = nullptr, *d_lg = nullptr;
    uint64_t *d_k = nullptr;
    bf16 *w1 = nullptr, *w2 = nullptr;
    int *err = nullptr;
    int rc = 0;
    if (cudaMalloc(&d_th, off.count * 4) || cudaMalloc(&d_lg, std::max<uint64_t>(n, 1) * 4) ||
        cudaMalloc(&d_k, std::max<uint64_t>(n, 1) * 8) || cudaMalloc(&w1, 256 * 128 * 2) || cudaMalloc(&w2, 256 * 256 * 2) ||
        cudaMalloc(&err, sizeof(int))) {
        rc = set_error("out of device memory");
    }
    if (rc == 0) {
        cudaMemset(err, 0, sizeof(int));
        cudaMemcpy(d_th, theta, off.count * 4, cudaMemcpyHostToDevice);
        cudaMemcpy(d_k, kmers, n * 8, cudaMemcpyHostToDevice);
        to_bf16_kernel<<<(256 * 128 + 255) / 256, 256>>>(d_th + off.W1, w1, 256 * 128);
        to_bf16_kernel<<<(256 * 256 + 255) / 256, 256>>>(d_th + off.W2, w2, 256 * 256);
        int sms = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0);
        InferBias hb;
        bias_from_host(theta, off, hb);
        rc = infer(d_k, n, k, w1, w2, hb, logits_only(d_lg), err, sms, 0);
        if (rc == 0) {
            cudaError_t e = cudaDeviceSynchronize();
            if (e != cudaSuccess) rc = set_error("inference failed: %s", cudaGetErrorString(e));
        }
        if (rc == 0) rc = check_err(err, "inference");
        if (rc == 0) cudaMemcpy(logits, d_lg, n * 4, cudaMemcpyDeviceToHost);
    }
    cudaFree(d_th); cudaFree(d_lg); cudaFree(d_k); cudaFree(w1); cudaFree(w2); cudaFree(err);
    return rc;
}
