/*
 * langmuir_b200_cnn.h -- BF16 tensor-core kernels of the morphology surrogate.
 *
 * No reference counterpart: the reference screens ga2d morphologies with a
 * hand-fitted regression over image descriptors (LangmuirPython/ga2d/ga.py:83-141,
 * descriptors in ga_analyze.py:164-380).  These kernels train and run the CNN
 * that replaces it.  Network: four 3x3 convolutions of LGM_CNN_CHANNELS channels
 * (bias, ReLU; 2x2 average pooling after the first three), global average
 * pooling, and a two-layer fully connected head.
 *
 * Layouts: activations NHWC BF16 (x[b][y][x][c]); conv weights BF16
 * w[cout][k], k = (ky*3 + kx)*cin + c, with cin == 1 padded to k < 16 (zeros
 * for k >= 9); gradients and biases FP32.  Every product accumulates in FP32
 * (mma.sync m16n8k16 BF16).  All entry points are asynchronous on `stream`
 * (a cudaStream_t, NULL = legacy default) and take device pointers.
 */
#ifndef LANGMUIR_B200_CNN_H
#define LANGMUIR_B200_CNN_H

#include "langmuir_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

#define LGM_CNN_CHANNELS 32

/* act = relu?(conv3x3(x, w) + bias) at full resolution (act may be NULL) and
 * pooled = avgpool2x2(act) (may be NULL; not both).  cin is 1 or
 * LGM_CNN_CHANNELS; H % 8 == 0, W % 16 == 0.  With the weights from
 * lgm_cnn_flip_weights, bias NULL and relu 0 this is the input gradient. */
lgm_status lgm_cnn_conv3x3_fwd(int32_t cin, const void* x, const void* w, const float* bias,
                               void* act, void* pooled, int32_t B, int32_t H, int32_t W,
                               int32_t relu, void* stream);

/* lgm_cnn_conv3x3_fwd for cin = LGM_CNN_CHANNELS on the 5th-generation
 * tensor cores: tcgen05.mma (M128 N32 K16, BF16 in, FP32 accumulators in
 * tensor memory), the input patch staged three times shifted by one column so
 * that every tap's operand is a contiguous shared-memory block.  Same
 * arguments and results as lgm_cnn_conv3x3_fwd; all pointers 16-byte aligned.
 * A bounded wait that runs out sets a flag read by lgm_cnn_error. */
lgm_status lgm_cnn_conv3x3_fwd_tc(const void* x, const void* w, const float* bias, void* act,
                                  void* pooled, int32_t B, int32_t H, int32_t W, int32_t relu,
                                  void* stream);

/* Error bits raised on the device by the tensor-core kernels since the last
 * call (LGM_ERR_TIMEOUT if any), then cleared.  Synchronises the device. */
lgm_status lgm_cnn_error(uint32_t* flags);

/* dW[cout][k] += sum over pixels of dA[p][cout] * im2col(x)[p][k] and
 * db[cout] += sum_p dA[p][cout] (db may be NULL).  dW and db are FP32 and are
 * added to, not overwritten. */
lgm_status lgm_cnn_conv3x3_wgrad(int32_t cin, const void* x, const void* dA, float* dW, float* db,
                                 int32_t B, int32_t H, int32_t W, void* stream);

/* Input-gradient weights of a cin = LGM_CNN_CHANNELS layer:
 * wd[c][(ky*3 + kx)*COUT + o] = w[o][((2-ky)*3 + (2-kx))*cin + c]. */
lgm_status lgm_cnn_flip_weights(int32_t cin, const void* w, void* wd, void* stream);

/* C[m][n] = sum_k A(m,k) B(k,n) (+ bias[n]) (ReLU if relu), with
 * A(m,k) = A[m*sam + k*sak], B(k,n) = B[k*sbk + n*sbn] (BF16, element
 * strides), C FP32 with row stride N.  accumulate != 0 adds into C. */
lgm_status lgm_cnn_gemm(const void* A, int32_t sam, int32_t sak, const void* B, int32_t sbk,
                        int32_t sbn, float* C, const float* bias, int32_t M, int32_t N, int32_t K,
                        int32_t relu, int32_t accumulate, void* stream);

/* dA = (act > 0) * g, g = dP (same shape) or, pooled != 0, dP[b][y/2][x/2][c] / 4. */
lgm_status lgm_cnn_relu_pool_bwd(const void* act, const void* dP, void* dA, int32_t B, int32_t H,
                                 int32_t W, int32_t pooled, void* stream);

/* out[b][c] = mean over HW pixels of act[b][p][c] (FP32 and BF16 copies). */
lgm_status lgm_cnn_gap_fwd(const void* act, float* out32, void* out16, int32_t B, int32_t HW,
                           void* stream);

/* dA[b][p][c] = (act > 0) * dg[b][c] / HW. */
lgm_status lgm_cnn_gap_relu_bwd(const void* act, const float* dg, void* dA, int32_t B, int32_t HW,
                                void* stream);

/* out = bf16(in), zero where relu_mask[i] <= 0 (relu_mask may be NULL). */
lgm_status lgm_cnn_to_bf16(const float* in, void* out, int32_t n, const float* relu_mask,
                           void* stream);

#ifdef __cplusplus
}
#endif

#endif /* LANGMUIR_B200_CNN_H */
