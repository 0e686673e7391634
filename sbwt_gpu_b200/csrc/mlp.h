// mlp.h -- host-side declarations of the learned prefilter.
#pragma once
#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace sbwt {
namespace mlp {

// Offsets of each tensor in the flat FP32 parameter vector:
// W1 [256][128] (inputs past 4k are zero), b1 [256], W2 [256][256] ([out][in]),
// b2 [256], w3 [256], b3 [1].
struct MlpOffsets {
    uint32_t W1 = 0;
    uint32_t b1 = 256 * 128;
    uint32_t W2 = 256 * 128 + 256;
    uint32_t b2 = 256 * 128 + 256 + 256 * 256;
    uint32_t w3 = 256 * 128 + 256 + 256 * 256 + 256;
    uint32_t b3 = 256 * 128 + 256 + 256 * 256 + 256 + 256;
    uint32_t count = 256 * 128 + 256 + 256 * 256 + 256 + 256 + 1;
};

struct C5 {
    uint64_t c[5];
};

// Kernels of mlp.cu launched from prefilter.cu (see mlp.cu for each).
__global__ void onehot_batch_kernel(const uint64_t *kmers, const uint8_t *labels, uint64_t n_train,
                                    const unsigned long long *step, uint32_t batch, uint32_t k, __nv_bfloat16 *X,
                                    float *Y);
__global__ void bias_relu_kernel(const float *Z, const float *bias, __nv_bfloat16 *H, uint64_t count);
__global__ void head_kernel(const float *Z2, const float *theta, const float *Y, uint32_t batch, __nv_bfloat16 *dZ2,
                            float *grad, float *loss_sum, const MlpOffsets off);
__global__ void relu_grad_kernel(const float *dH1, const __nv_bfloat16 *H1, uint32_t batch, __nv_bfloat16 *dZ1,
                                 float *grad, const MlpOffsets off);
__global__ void adam_kernel(float *theta, const float *grad, float *m, float *v, const unsigned long long *step,
                            uint32_t count, float lr, uint32_t k, __nv_bfloat16 *W1b, __nv_bfloat16 *W2b,
                            const MlpOffsets off);
__global__ void step_kernel(unsigned long long *step, float *loss_hist, const float *loss_sum, uint32_t hist_every);
__global__ void to_bf16_kernel(const float *src, __nv_bfloat16 *dst, uint32_t count);
__global__ void sample_kernel(const ulonglong4 *lines, uint32_t lpc, C5 C5v, uint32_t n_nodes, uint32_t k,
                              uint64_t n_pos, uint64_t n_neg, uint64_t seed, uint64_t count, uint64_t *out);
__global__ void enumerate_kernel(const ulonglong4 *lines, uint32_t lpc, C5 C5v, uint32_t n_nodes, uint32_t k,
                                 uint64_t *out);
__global__ void labels_kernel(const uint64_t *answers, uint64_t n, uint8_t *labels, unsigned long long *positives);
__global__ void bloom_build_kernel(const uint64_t *kmers, const float *logits, uint64_t n, float tau, uint32_t k,
                                   uint32_t *bits, uint64_t mask, uint32_t hashes, unsigned long long *rejected);
__global__ void accuracy_kernel(const float *logits, const uint8_t *labels, uint64_t n, float tau,
                                unsigned long long *correct);

int gemm_tn(const __nv_bfloat16 *A, const __nv_bfloat16 *B, float *D, uint32_t M, uint32_t N, uint32_t K,
            uint32_t splits, int *err, cudaStream_t s);
// Outputs of an inference pass: the logits (NULL: not written) and/or the
// sandwich's reject bitmap (bit j%32 of word j/32 = k-mer j rejected by the
// model at tau and by the backup Bloom filter; NULL: not written).
struct InferOut {
    float *logits;
    uint32_t *reject;
    float tau;
    const uint32_t *bloom_bits;
    uint64_t bloom_mask;
    uint32_t bloom_hashes;
};
constexpr int kMaxDevicesAttr = 64;
inline InferOut logits_only(float *logits) { return InferOut{logits, nullptr, 0.0f, nullptr, 0, 0}; }

// The biases and the output weights of an inference launch, passed by value:
// they are the same for every thread of a warp, so in the parameter space
// they are read through the constant cache instead of the global-load queue.
struct alignas(16) InferBias {  // 16-byte aligned: the epilogues read it as float4
    float b1[256];
    float b2[256];
    float w3[256];
    float b3;
};
inline void bias_from_host(const float *theta, const MlpOffsets &off, InferBias &b) {
    for (int i = 0; i < 256; i++) {
        b.b1[i] = theta[off.b1 + i];
        b.b2[i] = theta[off.b2 + i];
        b.w3[i] = theta[off.w3 + i];
    }
    b.b3 = theta[off.b3];
}

int infer(const uint64_t *kmers, uint64_t n, uint32_t k, const __nv_bfloat16 *W1b, const __nv_bfloat16 *W2b,
          const InferBias &bias, const InferOut &out, int *err, int num_sms, cudaStream_t s);
int transpose(const __nv_bfloat16 *src, __nv_bfloat16 *dst, uint32_t R, uint32_t C, cudaStream_t s);

}  // namespace mlp
}  // namespace sbwt
