/* cupyram_b200_mlp.h - C ABI of the learned surrogate's tensor-core kernels.
 *
 * No counterpart in the reference: clapeyre/cupyram has no learned model.
 * These entry points train and evaluate the small MLP ensemble that maps an
 * environment (sound-speed profile, depth, slope, bottom, frequency, source
 * depth) to a coarse transmission-loss field, falling back to the march for
 * the requests the ensemble disagrees on (cupyram_b200/surrogate.py).
 *
 * All pointers are device pointers; `stream` is a cudaStream_t (NULL: the
 * legacy default stream).  Matrices are row-major BF16 unless stated; every
 * call returns 0 or a CR_MLP_E* code and launches asynchronously.
 */
#ifndef CUPYRAM_B200_MLP_H
#define CUPYRAM_B200_MLP_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum cr_mlp_status {
    CR_MLP_OK = 0,
    CR_MLP_EBADSHAPE = 1, /* shape, stride or alignment outside what the kernel takes */
    CR_MLP_ECUDA = 2      /* launch failure */
};

/* Epilogues of cr_mlp_gemm (C = A B^T accumulated in FP32, then): */
enum cr_mlp_epi {
    CR_MLP_EPI_BIAS_RELU_BF16 = 0, /* out (bf16) = max(C + bias[col], 0)            */
    CR_MLP_EPI_BIAS_F32 = 1,       /* out (f32)  = C + bias[col]                     */
    CR_MLP_EPI_F32 = 2,            /* out (f32)  = C                                 */
    CR_MLP_EPI_RELU_MASK_BF16 = 3  /* out (bf16) = C where mask[row][col] > 0, else 0 */
};

/* C[M][N] = sum_k A[m][k] B[n][k]: A is M x K (row stride lda), B is N x K
 * (row stride ldb), both BF16 and K-contiguous.  M and N must be multiples of
 * 128, K of 32; lda and ldb multiples of 8 elements with 16-byte aligned
 * bases.  out has row stride ldo; mask (bf16, row stride ldm) is read by
 * CR_MLP_EPI_RELU_MASK_BF16 only, bias (f32, N values) by the bias epilogues. */
int cr_mlp_gemm(int epi, const void* A, const void* B, int M, int N, int K, int lda, int ldb, void* out, int ldo,
                const float* bias, const void* mask, int ldm, void* stream);

/* cr_mlp_gemm on the 5th-generation tensor cores (tcgen05.mma, FP32
 * accumulator in tensor memory).  Same operands, epilogues and alignment
 * rules; N must be a multiple of 256 and K of 64.  err: a device int that the kernel sets
 * to 1 if one of its (bounded) waits on the tensor cores gives up, in which
 * case out is incomplete. */
int cr_mlp_gemm_tc(int epi, const void* A, const void* B, int M, int N, int K, int lda, int ldb, void* out, int ldo,
                   const float* bias, const void* mask, int ldm, int* err, void* stream);

/* dst[c][r] = src[r][c] for a rows x cols BF16 matrix. */
int cr_mlp_transpose(const void* src, int lds, void* dst, int ldd, int rows, int cols, void* stream);

/* out[c] = sum over rows of src[r][c] (BF16 in, FP32 out). */
int cr_mlp_col_sum(const void* src, int ld, int rows, int cols, float* out, void* stream);

/* grad[i] = 2 (pred[i] - target[i]) * inv_count where valid[i], else 0
 * (pred f32, target and grad bf16, valid u8); *sse += sum of squared errors
 * over the valid entries (FP64, device). */
int cr_mlp_mse_grad(const float* pred, const void* target, const unsigned char* valid, long long n, float inv_count,
                    void* grad, double* sse, void* stream);

/* One bias-corrected Adam step on n FP32 parameters p with moments m, v
 * (weight_decay * p is added to the gradient); the updated parameters are
 * also written as BF16 to p_bf16 when it is not NULL.  step counts from 1. */
int cr_mlp_adam(float* p, const float* g, float* m, float* v, void* p_bf16, long long n, float lr, float beta1,
                float beta2, float eps, int step, float weight_decay, void* stream);

/* dst = BF16(src) for n values. */
int cr_mlp_to_bf16(const float* src, void* dst, long long n, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* CUPYRAM_B200_MLP_H */
