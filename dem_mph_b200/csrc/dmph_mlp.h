// Surrogate MLP: shapes, parameter block and GEMM arguments shared by the
// tensor-core kernels (dmph_mlp.cu) and their host driver (dmph_surrogate.cu).
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace dmph {

constexpr int kMlpLayers = 4;
constexpr int kMlpFeatures = 52;  // features computed per particle
constexpr int kMlpIn = 64;        // features padded to the K granularity of the weight-gradient GEMM
constexpr int kMlpHidden = 128;
constexpr int kMlpTargets = 6;    // velocity increment (3) and position residual (3)
constexpr int kMlpOut = 16;       // outputs padded to the smallest MMA N

enum MlpEpi { EPI_RELU = 0, EPI_OUT = 1, EPI_BWD_RELU = 2, EPI_WGRAD = 3 };

// D[M x N] = A[M x K] * B[N x K]^T; A and B row-major BF16 (K contiguous)
struct GemmArgs {
    const __nv_bfloat16 *A = nullptr;
    long long lda = 0;
    const __nv_bfloat16 *B = nullptr;
    long long ldb = 0;
    long long M = 0;
    int N = 0;
    long long K = 0;
    int epi = EPI_RELU;
    const float *bias = nullptr;
    __nv_bfloat16 *outB = nullptr;  // row-major BF16 result, leading dimension ldo
    long long ldo = 0;
    __nv_bfloat16 *outT = nullptr;  // transposed BF16 result, leading dimension ldT
    long long ldT = 0;
    float *outF = nullptr;          // FP32 result (EPI_OUT, ld ldo) or gradient (EPI_WGRAD)
    int transpose_out = 0;          // EPI_WGRAD: accumulate D^T
    const float *target = nullptr;  // EPI_OUT: targets [M x ldt]
    long long ldt = 0;
    int n_valid = 0;
    float grad_scale = 0.f;
    float *loss = nullptr;
    const __nv_bfloat16 *mask = nullptr;  // EPI_BWD_RELU: activation whose sign gates the gradient
    long long ldm = 0;
    int *err = nullptr;  // set to 1 when a bounded wait ran out
};

// FP32 master parameters (weights then biases of every layer in one array),
// Adam moments and gradient; BF16 weights [out][in] and transposed [in][out]
struct MlpParamsDev {
    float *w = nullptr, *m = nullptr, *v = nullptr, *grad = nullptr;
    int count = 0;
    int woff[kMlpLayers] = {0}, boff[kMlpLayers] = {0};
    int in[kMlpLayers] = {0}, out[kMlpLayers] = {0};
    __nv_bfloat16 *wb[kMlpLayers] = {nullptr}, *wt[kMlpLayers] = {nullptr};
};

void launch_gemm(const GemmArgs &g, int ksplit, cudaStream_t st);
// Y[n][kMlpOut] = MLP(X[n][kMlpIn]) in one fused kernel (TMA-fed feature
// tiles, weights resident in shared memory); X 16-byte aligned.  Nonzero
// when the launch could not be prepared (the tensor map); *err is set on
// the device when a bounded wait ran out.
int launch_mlp_forward(const MlpParamsDev &M, const __nv_bfloat16 *X, long long n, float *Y, int *err, int sms,
                       cudaStream_t st);
void launch_row_sums(const __nv_bfloat16 *T, long long ld, int rows, int cols, float *out, cudaStream_t st);
void launch_adam(const MlpParamsDev &M, float lr, int t, cudaStream_t st);
void launch_weights_to_bf16(const MlpParamsDev &M, cudaStream_t st);

}  // namespace dmph
