/*
 * hp2d_nn.h -- C ABI of the learned screening network's kernels (no counterpart in the
 * reference: HydroPol2D has no surrogate model).  A 4-level convolutional U-Net is trained
 * on peak-depth and arrival-time maps that the solver produces; these are its building
 * blocks, composed by the host (hydropol2d_b200/surrogate.py) into the forward pass, the
 * backward pass and the optimiser step.
 *
 * Layout: activations are NHWC BF16 (channels contiguous), stored as uint16_t bit patterns;
 * a 3x3 convolution is im2col (K = 9*C padded to a multiple of 64, K index = (ky*3+kx)*C+c)
 * followed by the tensor-core GEMM.  All calls are asynchronous on `stream` (a
 * cudaStream_t; NULL = legacy default stream) and take device pointers.
 */
#ifndef HP2D_NN_H
#define HP2D_NN_H

#include <stddef.h>
#include <stdint.h>

#include "hp2d.h"

#ifdef __cplusplus
extern "C" {
#endif

/* GEMM epilogues */
enum {
    HP2D_NN_EPI_F32 = 0,            /* C fp32 = A B^T */
    HP2D_NN_EPI_F32_ATOMIC = 1,     /* C fp32 += A B^T (required when split_k > 1) */
    HP2D_NN_EPI_BF16_BIAS_RELU = 2, /* C bf16 = max(A B^T + bias, 0) */
    HP2D_NN_EPI_BF16_BIAS = 3,      /* C bf16 = A B^T + bias */
    HP2D_NN_EPI_F32_BIAS = 4        /* C fp32 = A B^T + bias */
};

/* C[M x N] (epilogue) A[M x K] B[N x K]^T on the tcgen05 tensor cores: A and B BF16,
 * K-major (row pitch lda / ldb elements, multiples of 8, 16-byte aligned bases), K a
 * multiple of 64, FP32 accumulation; split_k slices of K accumulate atomically. */
hp2d_status hp2d_nn_gemm(int32_t M, int32_t N, int32_t K, const void* A, int32_t lda, const void* B,
                         int32_t ldb, void* C, int32_t ldc, const float* bias, int32_t epilogue,
                         int32_t split_k, void* stream);
/* 3x3, stride-1, zero-padded convolution as an implicit GEMM on the same tensor cores:
 * y[P, Co] (epilogue) = conv(x, w) with x [B,H,W,C] NHWC BF16 read through a 4-D tensor map
 * (no im2col buffer), w [Co, 9C] K-major BF16 (pitch ldw, K index (ky*3+kx)*C + c), P = B*H*W.
 * C a multiple of 32; W a multiple of 128 or a divisor of 128 with H*W a multiple of 128.
 * Epilogues F32, F32_BIAS, BF16_BIAS, BF16_BIAS_RELU. */
hp2d_status hp2d_nn_conv3x3(const uint16_t* x, int32_t B, int32_t H, int32_t W, int32_t C, const uint16_t* w,
                            int32_t ldw, int32_t Co, const float* bias, void* y, int32_t ldy, int32_t epilogue,
                            void* stream);
/* sticky error of the kernels (1 = a wait ran out); reading clears it; synchronises */
hp2d_status hp2d_nn_check(void);
const char* hp2d_nn_error(void);

/* im2col of a 3x3, stride-1, zero-padded convolution: x [B,H,W,C] -> cols [P, Kp]
 * (transpose = 0) or [Kp, P] (transpose = 1), P = B*H*W, zero columns k >= 9C. */
hp2d_status hp2d_nn_im2col3x3(const uint16_t* x, int32_t B, int32_t H, int32_t W, int32_t C, uint16_t* cols,
                              int32_t Kp, int32_t transpose, void* stream);
/* out[c, r] = in[r, c]: in [rows, cols] pitch ldi, out pitch ldo */
hp2d_status hp2d_nn_transpose(const uint16_t* in, int32_t rows, int32_t cols, int32_t ldi, uint16_t* out,
                              int32_t ldo, void* stream);
/* 2x2 max pooling (H, W even) and its backward (gradient to the first maximum; with
 * accumulate = 1 it is added to dx, rounded once to BF16) */
hp2d_status hp2d_nn_maxpool2(const uint16_t* x, int32_t B, int32_t H, int32_t W, int32_t C, uint16_t* y,
                             void* stream);
hp2d_status hp2d_nn_maxpool2_bwd(const uint16_t* x, const uint16_t* y, const uint16_t* dy, int32_t B, int32_t H,
                                 int32_t W, int32_t C, uint16_t* dx, int32_t accumulate, void* stream);
/* nearest-neighbour 2x upsampling [B,H,W,C] -> [B,2H,2W,C] and its backward (sum of 4) */
hp2d_status hp2d_nn_upsample2(const uint16_t* x, int32_t B, int32_t H, int32_t W, int32_t C, uint16_t* y,
                              void* stream);
hp2d_status hp2d_nn_upsample2_bwd(const uint16_t* dy, int32_t B, int32_t H, int32_t W, int32_t C, uint16_t* dx,
                                  void* stream);
/* channel slices: out[p, 0:n] = in[p, c0:c0+n] (pitches cin / cout); concat = two copies */
hp2d_status hp2d_nn_copy_channels(const uint16_t* in, int32_t cin, int32_t c0, int32_t n, int64_t P,
                                  uint16_t* out, int32_t cout, int32_t o0, void* stream);
/* dz = dy * (y > 0), in place on dy */
hp2d_status hp2d_nn_relu_bwd(const uint16_t* y, uint16_t* dy, int64_t n, void* stream);
/* out[c] += sum_p dz[p, c]  (dz [P, C] pitch ld) */
hp2d_status hp2d_nn_colsum(const uint16_t* dz, int64_t P, int32_t C, int32_t ld, float* out, void* stream);
/* masked squared error over channels 0..nch-1 of pred [P, ldp] (fp32) against target
 * [P, nch] with weights w [P, nch] (fp32): loss += sum w (pred - t)^2 * scale and
 * dpred [P, ldd] (bf16, other channels zero) = 2 w (pred - t) * scale */
hp2d_status hp2d_nn_mse(const float* pred, int32_t ldp, const float* target, const float* w, int64_t P,
                        int32_t nch, float scale, float* loss, uint16_t* dpred, int32_t ldd, void* stream);
/* Adam with decoupled weight decay on fp32 master weights; writes the bf16 copy */
hp2d_status hp2d_nn_adam(float* w, const float* g, float* m, float* v, uint16_t* w_bf16, int64_t n, float lr,
                         float beta1, float beta2, float eps, float weight_decay, int32_t step, void* stream);
/* weights of a 3x3 convolution [Co, Kp] (K = tap*Ci + ci) -> the backward-data weights
 * [Ci, Kp2] (K = tap*Co + co) of the flipped kernel, as BF16 */
hp2d_status hp2d_nn_flip3x3(const float* w, int32_t Co, int32_t Ci, int32_t Kp, uint16_t* wt, int32_t Kp2,
                            void* stream);
hp2d_status hp2d_nn_f32_to_bf16(const float* in, uint16_t* out, int64_t n, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* HP2D_NN_H */
