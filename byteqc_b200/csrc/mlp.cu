// BF16 tensor-core kernels of the learned initial-density model (a
// 3-hidden-layer MLP): forward and backward of a dense layer and the Adam
// update.  Operands are BF16, accumulation FP32 (warp-level 16x16x16 tensor
// core fragments); master weights, biases, gradients and the loss stay FP32.
// Shapes: X (M x K), W (N x K) row-major, Y = act(X W^T + b) (M x N); M, N,
// K multiples of 16.
#include <cuda_bf16.h>
#include <mma.h>
#include "bqc.h"

using namespace nvcuda;

namespace {

constexpr int WARPS = 4;   // warps per block, one 16x16 output tile each

// Y = X W^T + b; optional ReLU; writes FP32 (pre-activation Z and/or
// activation) and a BF16 copy of the activation.
__global__ void linear_fwd_kernel(const __nv_bfloat16 *__restrict__ X,
                                  const __nv_bfloat16 *__restrict__ W,
                                  const float *__restrict__ b, float *Z, float *Yf,
                                  __nv_bfloat16 *Yb, int M, int N, int K, int relu) {
    __shared__ float tile[WARPS][16][16];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int n0 = (blockIdx.x * WARPS + warp) * 16, m0 = blockIdx.y * 16;
    if (n0 >= N) return;
    wmma::fragment<wmma::accumulator, 16, 16, 16, float> acc;
    wmma::fill_fragment(acc, 0.f);
    for (int k0 = 0; k0 < K; k0 += 16) {
        wmma::fragment<wmma::matrix_a, 16, 16, 16, __nv_bfloat16, wmma::row_major> a;
        wmma::fragment<wmma::matrix_b, 16, 16, 16, __nv_bfloat16, wmma::col_major> bw;
        wmma::load_matrix_sync(a, X + (size_t)m0 * K + k0, K);
        wmma::load_matrix_sync(bw, W + (size_t)n0 * K + k0, K);   // (W^T)[k][n] = W[n][k]
        wmma::mma_sync(acc, a, bw, acc);
    }
    wmma::store_matrix_sync(&tile[warp][0][0], acc, 16, wmma::mem_row_major);
    __syncwarp();
    for (int e = lane; e < 256; e += 32) {
        const int r = e >> 4, c = e & 15;
        const size_t o = (size_t)(m0 + r) * N + n0 + c;
        float z = tile[warp][r][c] + b[n0 + c];
        if (Z) Z[o] = z;
        float y = relu ? fmaxf(z, 0.f) : z;
        if (Yf) Yf[o] = y;
        if (Yb) Yb[o] = __float2bfloat16(y);
    }
}

// dZ = dY * (Z > 0) (or dY without ReLU), stored as BF16 for the GEMMs
__global__ void relu_bwd_kernel(const float *__restrict__ dY, const float *__restrict__ Z,
                                __nv_bfloat16 *dZ, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        float g = dY[i];
        if (Z != nullptr && Z[i] <= 0.f) g = 0.f;
        dZ[i] = __float2bfloat16(g);
    }
}

// dX = dZ W   (M x N) (N x K) -> (M x K)
__global__ void grad_x_kernel(const __nv_bfloat16 *__restrict__ dZ,
                              const __nv_bfloat16 *__restrict__ W, float *dX, int M, int N,
                              int K) {
    const int warp = threadIdx.x >> 5;
    const int k0 = (blockIdx.x * WARPS + warp) * 16, m0 = blockIdx.y * 16;
    if (k0 >= K) return;
    wmma::fragment<wmma::accumulator, 16, 16, 16, float> acc;
    wmma::fill_fragment(acc, 0.f);
    for (int n0 = 0; n0 < N; n0 += 16) {
        wmma::fragment<wmma::matrix_a, 16, 16, 16, __nv_bfloat16, wmma::row_major> a;
        wmma::fragment<wmma::matrix_b, 16, 16, 16, __nv_bfloat16, wmma::row_major> bw;
        wmma::load_matrix_sync(a, dZ + (size_t)m0 * N + n0, N);
        wmma::load_matrix_sync(bw, W + (size_t)n0 * K + k0, K);
        wmma::mma_sync(acc, a, bw, acc);
    }
    wmma::store_matrix_sync(dX + (size_t)m0 * K + k0, acc, K, wmma::mem_row_major);
}

// dW = dZ^T X  (N x M) (M x K) -> (N x K), summed over the batch
__global__ void grad_w_kernel(const __nv_bfloat16 *__restrict__ dZ,
                              const __nv_bfloat16 *__restrict__ X, float *dW, int M, int N,
                              int K) {
    const int warp = threadIdx.x >> 5;
    const int k0 = (blockIdx.x * WARPS + warp) * 16, n0 = blockIdx.y * 16;
    if (k0 >= K) return;
    wmma::fragment<wmma::accumulator, 16, 16, 16, float> acc;
    wmma::fill_fragment(acc, 0.f);
    for (int m0 = 0; m0 < M; m0 += 16) {
        // (dZ^T)[n][m] = dZ[m][n]: column-major view of dZ with leading dimension N
        wmma::fragment<wmma::matrix_a, 16, 16, 16, __nv_bfloat16, wmma::col_major> a;
        wmma::fragment<wmma::matrix_b, 16, 16, 16, __nv_bfloat16, wmma::row_major> bx;
        wmma::load_matrix_sync(a, dZ + (size_t)m0 * N + n0, N);
        wmma::load_matrix_sync(bx, X + (size_t)m0 * K + k0, K);
        wmma::mma_sync(acc, a, bx, acc);
    }
    wmma::store_matrix_sync(dW + (size_t)n0 * K + k0, acc, K, wmma::mem_row_major);
}

// db[n] = sum_m dZ[m][n] (FP32 from the FP32 gradient)
__global__ void grad_b_kernel(const float *__restrict__ dY, const float *__restrict__ Z,
                              float *db, int M, int N) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    float s = 0.f;
    for (int m = 0; m < M; m++) {
        float g = dY[(size_t)m * N + n];
        if (Z != nullptr && Z[(size_t)m * N + n] <= 0.f) g = 0.f;
        s += g;
    }
    db[n] = s;
}

__global__ void adam_kernel(float *w, const float *__restrict__ g, float *m, float *v,
                            __nv_bfloat16 *wb, int n, float lr, float b1, float b2, float eps,
                            float c1, float c2) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float gi = g[i];
        float mi = b1 * m[i] + (1.f - b1) * gi;
        float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
        w[i] = wi;
        if (wb) wb[i] = __float2bfloat16(wi);
    }
}

__global__ void to_bf16_kernel(const float *__restrict__ x, __nv_bfloat16 *y, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
        y[i] = __float2bfloat16(x[i]);
}

bool shapes_ok(int M, int N, int K) {
    return M > 0 && N > 0 && K > 0 && M % 16 == 0 && N % 16 == 0 && K % 16 == 0;
}

}  // namespace

extern "C" {

int BQCmlp_linear_fwd(const void *X, const void *W, const float *b, float *Z, float *Yf, void *Yb,
                      int M, int N, int K, int relu, cudaStream_t stream) {
    if (!shapes_ok(M, N, K)) return 3;
    bqc_count_launch(1);
    dim3 grid((N / 16 + WARPS - 1) / WARPS, M / 16);
    linear_fwd_kernel<<<grid, 32 * WARPS, 0, stream>>>(
        (const __nv_bfloat16 *)X, (const __nv_bfloat16 *)W, b, Z, Yf, (__nv_bfloat16 *)Yb, M, N,
        K, relu);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

int BQCmlp_linear_bwd(const float *dY, const float *Z, const void *X, const void *W, void *dZ_buf,
                      float *dX, float *dW, float *db, int M, int N, int K, cudaStream_t stream) {
    if (!shapes_ok(M, N, K)) return 3;
    bqc_count_launch(dX ? 4 : 3);
    size_t n = (size_t)M * N;
    relu_bwd_kernel<<<(unsigned)((n + 255) / 256 < 4096 ? (n + 255) / 256 : 4096), 256, 0, stream>>>(
        dY, Z, (__nv_bfloat16 *)dZ_buf, n);
    grad_b_kernel<<<(N + 127) / 128, 128, 0, stream>>>(dY, Z, db, M, N);
    dim3 gw((K / 16 + WARPS - 1) / WARPS, N / 16);
    grad_w_kernel<<<gw, 32 * WARPS, 0, stream>>>((const __nv_bfloat16 *)dZ_buf,
                                                  (const __nv_bfloat16 *)X, dW, M, N, K);
    if (dX) {
        dim3 gx((K / 16 + WARPS - 1) / WARPS, M / 16);
        grad_x_kernel<<<gx, 32 * WARPS, 0, stream>>>((const __nv_bfloat16 *)dZ_buf,
                                                      (const __nv_bfloat16 *)W, dX, M, N, K);
    }
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

int BQCmlp_adam(float *w, const float *g, float *m, float *v, void *w_bf16, int n, float lr,
                float b1, float b2, float eps, int step, cudaStream_t stream) {
    if (n <= 0 || step < 1) return 3;
    bqc_count_launch(1);
    float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
    int blocks = (n + 255) / 256 < 2048 ? (n + 255) / 256 : 2048;
    adam_kernel<<<blocks, 256, 0, stream>>>(w, g, m, v, (__nv_bfloat16 *)w_bf16, n, lr, b1, b2,
                                            eps, c1, c2);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

int BQCmlp_to_bf16(const float *x, void *y, size_t n, cudaStream_t stream) {
    bqc_count_launch(1);
    int blocks = (int)((n + 255) / 256 < 4096 ? (n + 255) / 256 : 4096);
    to_bf16_kernel<<<blocks > 0 ? blocks : 1, 256, 0, stream>>>(x, (__nv_bfloat16 *)y, n);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

}  // extern "C"
