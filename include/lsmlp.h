/* lsmlp.h -- BF16 kernels of the learned SCF guess (liblsjk.so).
 *
 * No counterpart in the reference: its SCF starts from the SAD guess
 * (est/rhf.py:401-421, src/cpp/sad/sad.cpp). The learned guess predicts
 * per-atom-pair density blocks with a small multilayer perceptron; these
 * entry points are its training and inference kernels. Matrices are
 * row-major; "bf16" arrays hold bfloat16 values (2 bytes each), every product
 * is accumulated in FP32. All pointers are device pointers; `stream` is a
 * cudaStream_t (NULL = legacy default stream). Return 0 on success, 1 for a
 * bad argument, 2 for a CUDA error (message from lsmlp_last_error).
 */
#ifndef LSMLP_H
#define LSMLP_H

#ifdef __cplusplus
extern "C" {
#endif

const char* lsmlp_last_error(void);

/* C (+)= op(A) op(B): op(A) is M x K (A is K x M with lda if transA),
 * op(B) is K x N (B is N x K with ldb if transB); A, B bf16, C FP32. */
int lsmlp_gemm_bf16(const void* A, const void* B, float* C, int M, int N, int K, int lda, int ldb, int ldc,
                    int transA, int transB, int accumulate, void* stream);

/* Z[r][c] += bias[c]; H = bf16(act(Z)) when H is not NULL; act 1 = SiLU, 0 = identity. */
int lsmlp_bias_act(float* Z, const float* bias, void* H, int rows, int cols, int act, void* stream);

/* dZ = bf16(dH * act'(Z)) elementwise over n values. */
int lsmlp_act_grad(const float* dH, const float* Z, void* dZ, long n, int act, void* stream);

/* *loss += sum_i W_i (Y_i - T_i)^2 * inv_norm; dY = bf16(2 W (Y - T) inv_norm) when dY is not NULL. */
int lsmlp_mse(const float* Y, const float* T, const float* W, void* dY, long n, float inv_norm, float* loss,
              void* stream);

/* db[c] = sum_r dZ[r][c] (dZ bf16 rows x cols). */
int lsmlp_colsum(const void* dZ, float* db, int rows, int cols, void* stream);

/* One Adam step (step counts from 1) on FP32 weights W with gradient G and
 * moments M, V; writes bf16(W) to Wb when not NULL. */
int lsmlp_adam(float* W, const float* G, float* M, float* V, void* Wb, long n, float lr, float beta1, float beta2,
               float eps, int step, float weight_decay, void* stream);

/* Y = bf16(X) elementwise. */
int lsmlp_to_bf16(const float* X, void* Y, long n, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* LSMLP_H */
