// Kernels of the learned SCF guess: a small multilayer perceptron trained and
// evaluated in BF16 (weights, activations and back-propagated gradients
// stored as bfloat16, every product accumulated in FP32), with FP32 master
// weights updated by Adam. Entry points are declared in include/lsmlp.h; all
// take device pointers and enqueue on the given stream.
//
// The products run on the tensor cores (BF16 mma.sync with FP32 accumulation,
// 64 x 64 output tiles, 32-deep K slices staged through shared memory); the
// element-wise kernels are plain grid-stride loops.
#include <algorithm>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <string>
#include "../../include/lsmlp.h"

namespace {

thread_local std::string g_mlp_err;

int mlp_status(cudaError_t e)
{
    if (e == cudaSuccess) return 0;
    g_mlp_err = cudaGetErrorString(e);
    return 2;
}

constexpr int kTM = 64, kTN = 64, kTK = 32, kThreads = 128;
constexpr int kPad = 8;   // bf16 elements of padding per shared-memory row

// C[m][n] (+)= sum_k op(A)[m][k] op(B)[k][n]; op(A)[m][k] = ta ? A[k*lda+m] : A[m*lda+k],
// op(B)[k][n] = tb ? B[n*ldb+k] : B[k*ldb+n].
// BF16 tensor-core products with FP32 accumulation (mma.sync m16n8k16): a CTA
// of four warps owns a 64 x 64 tile of C, each warp a 32 x 32 quarter as 2 x 4
// fragments of 16 x 8; 32-deep K slices of op(A) (m-major rows) and op(B)
// (n-major rows, i.e. k contiguous for the column operand) are staged in
// shared memory as bf16, zero-filled past the matrix edges.
__global__ void __launch_bounds__(kThreads)
k_gemm_bf16(const __nv_bfloat16* __restrict__ A, const __nv_bfloat16* __restrict__ B, float* __restrict__ C,
            int M, int N, int K, int lda, int ldb, int ldc, int ta, int tb, int accumulate)
{
    __shared__ __align__(16) __nv_bfloat16 As[kTM][kTK + kPad];
    __shared__ __align__(16) __nv_bfloat16 Bs[kTN][kTK + kPad];
    const int m0 = blockIdx.y * kTM, n0 = blockIdx.x * kTN;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;   // the warp's quarter of the tile
    const int grp = lane >> 2, tig = lane & 3;
    const __nv_bfloat16 zero = __float2bfloat16_rn(0.0f);
    float acc[2][4][4] = {};
    for (int k0 = 0; k0 < K; k0 += kTK) {
        for (int idx = threadIdx.x; idx < kTM * kTK; idx += kThreads) {
            const int mm = idx / kTK, kk = idx % kTK;
            const int m = m0 + mm, k = k0 + kk;
            __nv_bfloat16 v = zero;
            if (m < M && k < K) v = ta ? A[(long) k * lda + m] : A[(long) m * lda + k];
            As[mm][kk] = v;
        }
        for (int idx = threadIdx.x; idx < kTN * kTK; idx += kThreads) {
            const int nn = idx / kTK, kk = idx % kTK;
            const int n = n0 + nn, k = k0 + kk;
            __nv_bfloat16 v = zero;
            if (n < N && k < K) v = tb ? B[(long) n * ldb + k] : B[(long) k * ldb + n];
            Bs[nn][kk] = v;
        }
        __syncthreads();
#pragma unroll
        for (int ks = 0; ks < kTK; ks += 16) {
            // fragments (PTX mma.m16n8k16 layouts): A rows grp / grp + 8, k pairs tig*2 (+8);
            // B column grp, k pairs tig*2 (+8)
            unsigned a[2][4], b[4][2];
#pragma unroll
            for (int mt = 0; mt < 2; ++mt) {
                const int r = wm + mt * 16 + grp, c = ks + tig * 2;
                a[mt][0] = *reinterpret_cast<const unsigned*>(&As[r][c]);
                a[mt][1] = *reinterpret_cast<const unsigned*>(&As[r + 8][c]);
                a[mt][2] = *reinterpret_cast<const unsigned*>(&As[r][c + 8]);
                a[mt][3] = *reinterpret_cast<const unsigned*>(&As[r + 8][c + 8]);
            }
#pragma unroll
            for (int nt = 0; nt < 4; ++nt) {
                const int r = wn + nt * 8 + grp, c = ks + tig * 2;
                b[nt][0] = *reinterpret_cast<const unsigned*>(&Bs[r][c]);
                b[nt][1] = *reinterpret_cast<const unsigned*>(&Bs[r][c + 8]);
            }
#pragma unroll
            for (int mt = 0; mt < 2; ++mt)
#pragma unroll
                for (int nt = 0; nt < 4; ++nt) {
                    float* d = acc[mt][nt];
                    asm volatile(
                        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
                        "{%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, {%0, %1, %2, %3};\n"
                        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
                        : "r"(a[mt][0]), "r"(a[mt][1]), "r"(a[mt][2]), "r"(a[mt][3]), "r"(b[nt][0]),
                          "r"(b[nt][1]));
                }
        }
        __syncthreads();
    }
    // accumulator layout: d0, d1 at row grp, columns tig*2, tig*2 + 1; d2, d3 at row grp + 8
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int nt = 0; nt < 4; ++nt)
#pragma unroll
            for (int h = 0; h < 2; ++h)
#pragma unroll
                for (int j = 0; j < 2; ++j) {
                    const int m = m0 + wm + mt * 16 + grp + 8 * h, n = n0 + wn + nt * 8 + tig * 2 + j;
                    if (m < M && n < N) {
                        float* c = C + (long) m * ldc + n;
                        const float v = acc[mt][nt][2 * h + j];
                        *c = accumulate ? *c + v : v;
                    }
                }
}

__device__ __forceinline__ float silu(float z) { return z / (1.0f + __expf(-z)); }
__device__ __forceinline__ float silu_grad(float z)
{
    const float s = 1.0f / (1.0f + __expf(-z));
    return s * (1.0f + z * (1.0f - s));
}

// Z[r][c] += bias[c]; H[r][c] = bf16(act(Z[r][c])) (act = SiLU, or identity).
__global__ void k_bias_act(float* __restrict__ Z, const float* __restrict__ bias, __nv_bfloat16* __restrict__ H,
                           int rows, int cols, int act)
{
    const long n = (long) rows * cols;
    for (long i = blockIdx.x * (long) blockDim.x + threadIdx.x; i < n; i += (long) gridDim.x * blockDim.x) {
        const float z = Z[i] + bias[i % cols];
        Z[i] = z;
        if (H) H[i] = __float2bfloat16_rn(act ? silu(z) : z);
    }
}

// dZ = bf16(dH * act'(Z)).
__global__ void k_act_grad(const float* __restrict__ dH, const float* __restrict__ Z, __nv_bfloat16* __restrict__ dZ,
                           long n, int act)
{
    for (long i = blockIdx.x * (long) blockDim.x + threadIdx.x; i < n; i += (long) gridDim.x * blockDim.x)
        dZ[i] = __float2bfloat16_rn(act ? dH[i] * silu_grad(Z[i]) : dH[i]);
}

// Masked mean squared error: loss += sum w (y - t)^2 / norm; dY = bf16(2 w (y - t) / norm).
__global__ void k_mse(const float* __restrict__ Y, const float* __restrict__ T, const float* __restrict__ W,
                      __nv_bfloat16* __restrict__ dY, long n, float inv_norm, float* __restrict__ loss)
{
    float s = 0.0f;
    for (long i = blockIdx.x * (long) blockDim.x + threadIdx.x; i < n; i += (long) gridDim.x * blockDim.x) {
        const float d = Y[i] - T[i];
        const float w = W[i];
        s += w * d * d;
        if (dY) dY[i] = __float2bfloat16_rn(2.0f * w * d * inv_norm);
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0 && loss) atomicAdd(loss, s * inv_norm);
}

// db[c] = sum_r bf16 dZ[r][c] (FP32 sums).
__global__ void k_colsum(const __nv_bfloat16* __restrict__ dZ, float* __restrict__ db, int rows, int cols)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= cols) return;
    float s = 0.0f;
    for (int r = 0; r < rows; ++r) s += __bfloat162float(dZ[(long) r * cols + c]);
    db[c] = s;
}

// Adam on FP32 master weights; Wb = bf16(W) for the next forward pass.
__global__ void k_adam(float* __restrict__ W, const float* __restrict__ G, float* __restrict__ Mo,
                       float* __restrict__ Vo, __nv_bfloat16* __restrict__ Wb, long n, float lr, float b1, float b2,
                       float eps, float c1, float c2, float wd)
{
    for (long i = blockIdx.x * (long) blockDim.x + threadIdx.x; i < n; i += (long) gridDim.x * blockDim.x) {
        const float g = G[i] + wd * W[i];
        const float m = b1 * Mo[i] + (1.0f - b1) * g;
        const float v = b2 * Vo[i] + (1.0f - b2) * g * g;
        Mo[i] = m;
        Vo[i] = v;
        const float w = W[i] - lr * (m * c1) / (sqrtf(v * c2) + eps);
        W[i] = w;
        if (Wb) Wb[i] = __float2bfloat16_rn(w);
    }
}

__global__ void k_to_bf16(const float* __restrict__ X, __nv_bfloat16* __restrict__ Y, long n)
{
    for (long i = blockIdx.x * (long) blockDim.x + threadIdx.x; i < n; i += (long) gridDim.x * blockDim.x)
        Y[i] = __float2bfloat16_rn(X[i]);
}

unsigned grid_for(long n) { return (unsigned) std::min<long>((n + 255) / 256, 148L * 8); }

} // namespace

extern "C" {

const char* lsmlp_last_error(void) { return g_mlp_err.c_str(); }

int lsmlp_gemm_bf16(const void* A, const void* B, float* C, int M, int N, int K, int lda, int ldb, int ldc,
                    int transA, int transB, int accumulate, void* stream)
{
    if (M < 0 || N < 0 || K < 0 || (M && N && (!A || !B || !C))) {
        g_mlp_err = "lsmlp_gemm_bf16: bad argument";
        return 1;
    }
    if (!M || !N) return 0;
    dim3 grid((N + kTN - 1) / kTN, (M + kTM - 1) / kTM);
    k_gemm_bf16<<<grid, kThreads, 0, (cudaStream_t) stream>>>(
        (const __nv_bfloat16*) A, (const __nv_bfloat16*) B, C, M, N, K, lda, ldb, ldc, transA, transB, accumulate);
    return mlp_status(cudaGetLastError());
}

int lsmlp_bias_act(float* Z, const float* bias, void* H, int rows, int cols, int act, void* stream)
{
    const long n = (long) rows * cols;
    if (!n) return 0;
    k_bias_act<<<grid_for(n), 256, 0, (cudaStream_t) stream>>>(Z, bias, (__nv_bfloat16*) H, rows, cols, act);
    return mlp_status(cudaGetLastError());
}

int lsmlp_act_grad(const float* dH, const float* Z, void* dZ, long n, int act, void* stream)
{
    if (!n) return 0;
    k_act_grad<<<grid_for(n), 256, 0, (cudaStream_t) stream>>>(dH, Z, (__nv_bfloat16*) dZ, n, act);
    return mlp_status(cudaGetLastError());
}

int lsmlp_mse(const float* Y, const float* T, const float* W, void* dY, long n, float inv_norm, float* loss,
              void* stream)
{
    if (!n) return 0;
    k_mse<<<grid_for(n), 256, 0, (cudaStream_t) stream>>>(Y, T, W, (__nv_bfloat16*) dY, n, inv_norm, loss);
    return mlp_status(cudaGetLastError());
}

int lsmlp_colsum(const void* dZ, float* db, int rows, int cols, void* stream)
{
    if (!cols) return 0;
    k_colsum<<<(cols + 127) / 128, 128, 0, (cudaStream_t) stream>>>((const __nv_bfloat16*) dZ, db, rows, cols);
    return mlp_status(cudaGetLastError());
}

int lsmlp_adam(float* W, const float* G, float* M, float* V, void* Wb, long n, float lr, float beta1, float beta2,
               float eps, int step, float weight_decay, void* stream)
{
    if (!n) return 0;
    if (step < 1) {
        g_mlp_err = "lsmlp_adam: step counts from 1";
        return 1;
    }
    const float c1 = 1.0f / (1.0f - powf(beta1, (float) step));
    const float c2 = 1.0f / (1.0f - powf(beta2, (float) step));
    k_adam<<<grid_for(n), 256, 0, (cudaStream_t) stream>>>(W, G, M, V, (__nv_bfloat16*) Wb, n, lr, beta1, beta2, eps,
                                                           c1, c2, weight_decay);
    return mlp_status(cudaGetLastError());
}

int lsmlp_to_bf16(const float* X, void* Y, long n, void* stream)
{
    if (!n) return 0;
    k_to_bf16<<<grid_for(n), 256, 0, (cudaStream_t) stream>>>(X, (__nv_bfloat16*) Y, n);
    return mlp_status(cudaGetLastError());
}

} // extern "C"
