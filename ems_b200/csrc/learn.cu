// learn.cu — kernels of the learned early stop (include/ems_learn.h), sm_100a.
//
// A small 1-D CNN (convolutions as im2col + GEMM, then two dense layers)
// trained and run on these kernels. The GEMM is a bf16 tensor-core kernel
// (mma.sync m16n8k16, f32 accumulation): 64×64 output tiles, four warps of
// 32×32, K in steps of 32 staged in shared memory. The matrices here are
// small (≤ 10^4 rows, ≤ 2·10^3 columns), so the kernel takes A and B with
// arbitrary element strides (a transposed operand is just other strides),
// which keeps the backward pass free of transpose copies.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/ems_learn.h"

namespace {

constexpr int GM = 64, GN = 64, GK = 32, GPAD = 8;

__device__ __forceinline__ uint16_t bf16_bits(float x) { return __bfloat16_as_ushort(__float2bfloat16_rn(x)); }

__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], const uint32_t (&b)[2]) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

__global__ void __launch_bounds__(128) k_gemm(const uint16_t* __restrict__ A, int64_t sa0, int64_t sa1,
                                              const uint16_t* __restrict__ B, int64_t sb0, int64_t sb1, float* C,
                                              int64_t ldc, int M, int N, int K, float alpha, float beta) {
    // As[m][k] (row-major A tile), Bs[n][k] (B tile stored column by column,
    // the layout of the MMA's "col" operand); rows padded against bank conflicts.
    __shared__ __align__(16) uint16_t As[GM][GK + GPAD];
    __shared__ __align__(16) uint16_t Bs[GN][GK + GPAD];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int g = lane >> 2, t = lane & 3;
    const int m0 = blockIdx.y * GM, n0 = blockIdx.x * GN;
    const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
    float acc[2][4][4];
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b)
#pragma unroll
            for (int c = 0; c < 4; ++c) acc[a][b][c] = 0.0f;
    for (int k0 = 0; k0 < K; k0 += GK) {
        for (int e = tid; e < GM * GK; e += 128) {
            const int r = e / GK, c = e - r * GK;
            const int i = m0 + r, k = k0 + c;
            As[r][c] = (i < M && k < K) ? A[i * sa0 + k * sa1] : (uint16_t)0;
        }
        for (int e = tid; e < GN * GK; e += 128) {
            const int r = e / GK, c = e - r * GK;  // r: column n, c: k
            const int j = n0 + r, k = k0 + c;
            Bs[r][c] = (j < N && k < K) ? B[k * sb0 + j * sb1] : (uint16_t)0;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < GK; kk += 16) {
            uint32_t af[2][4], bf[4][2];
#pragma unroll
            for (int mi = 0; mi < 2; ++mi) {
                const int r = wm + mi * 16 + g;
                af[mi][0] = *reinterpret_cast<const uint32_t*>(&As[r][kk + t * 2]);
                af[mi][1] = *reinterpret_cast<const uint32_t*>(&As[r + 8][kk + t * 2]);
                af[mi][2] = *reinterpret_cast<const uint32_t*>(&As[r][kk + 8 + t * 2]);
                af[mi][3] = *reinterpret_cast<const uint32_t*>(&As[r + 8][kk + 8 + t * 2]);
            }
#pragma unroll
            for (int ni = 0; ni < 4; ++ni) {
                const int n = wn + ni * 8 + g;
                bf[ni][0] = *reinterpret_cast<const uint32_t*>(&Bs[n][kk + t * 2]);
                bf[ni][1] = *reinterpret_cast<const uint32_t*>(&Bs[n][kk + 8 + t * 2]);
            }
#pragma unroll
            for (int mi = 0; mi < 2; ++mi)
#pragma unroll
                for (int ni = 0; ni < 4; ++ni) mma_bf16(acc[mi][ni], af[mi], bf[ni]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int mi = 0; mi < 2; ++mi)
#pragma unroll
        for (int ni = 0; ni < 4; ++ni)
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                const int i = m0 + wm + mi * 16 + g + (c >= 2 ? 8 : 0);
                const int j = n0 + wn + ni * 8 + t * 2 + (c & 1);
                if (i < M && j < N) {
                    float* p = C + i * ldc + j;
                    *p = beta != 0.0f ? alpha * acc[mi][ni][c] + beta * *p : alpha * acc[mi][ni][c];
                }
            }
}

__global__ void k_to_bf16(const float* src, uint16_t* dst, size_t n) {
    const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q < n) dst[q] = bf16_bits(src[q]);
}

__global__ void k_im2col(const float* x, uint16_t* col, int B, int T, int C, int k, int s, int To) {
    const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const size_t F = (size_t)k * C, total = (size_t)B * To * F;
    if (q >= total) return;
    const size_t r = q / F, f = q - r * F;
    const int b = (int)(r / To), to = (int)(r - (size_t)b * To);
    const int tap = (int)(f / C), ch = (int)(f - (size_t)tap * C);
    col[q] = bf16_bits(x[((size_t)b * T + (size_t)to * s + tap) * C + ch]);
}

__global__ void k_col2im(const float* dcol, float* dx, int B, int T, int C, int k, int s, int To) {
    const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= (size_t)B * T * C) return;
    const int ch = (int)(q % C);
    const size_t bt = q / C;
    const int t = (int)(bt % T), b = (int)(bt / T);
    const size_t F = (size_t)k * C;
    float acc = 0.0f;
    // t_out from high to low: taps in increasing order.
    int hi = t / s;
    if (hi > To - 1) hi = To - 1;
    for (int to = hi; to >= 0; --to) {
        const int tap = t - to * s;
        if (tap >= k) break;
        acc += dcol[((size_t)b * To + to) * F + (size_t)tap * C + ch];
    }
    dx[q] = acc;
}

__device__ __forceinline__ float sigmoid(float y) { return 1.0f / (1.0f + expf(-y)); }

__global__ void k_bias_act(float* y, const float* bias, float* a, int rows, int cols, int act) {
    const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= (size_t)rows * cols) return;
    const float v = y[q] + bias[q % cols];
    y[q] = v;
    a[q] = act ? v * sigmoid(v) : v;
}

__global__ void k_act_grad(const float* y, const float* da, float* dy, int rows, int cols, int act) {
    const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= (size_t)rows * cols) return;
    if (!act) {
        dy[q] = da[q];
        return;
    }
    const float s = sigmoid(y[q]);
    dy[q] = da[q] * (s + y[q] * s * (1.0f - s));
}

// One block per column: strided partial sums in a fixed order, then a tree.
__global__ void __launch_bounds__(256) k_bias_grad(const float* dy, float* db, int rows, int cols) {
    __shared__ float sh[256];
    const int j = blockIdx.x;
    float s = 0.0f;
    for (int r = threadIdx.x; r < rows; r += 256) s += dy[(size_t)r * cols + j];
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) db[j] = sh[0];
}

__global__ void k_mse_grad(const float* out, const float* target, float* grad, size_t n) {
    const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q < n) grad[q] = 2.0f * (out[q] - target[q]) / (float)n;
}

__global__ void __launch_bounds__(1024) k_mse_loss(const float* out, const float* target, float* loss, size_t n) {
    __shared__ float sh[1024];
    float s = 0.0f;
    for (size_t q = threadIdx.x; q < n; q += 1024) {
        const float d = out[q] - target[q];
        s += d * d;
    }
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int w = 512; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) loss[0] = sh[0] / (float)n;
}

__global__ void k_adam(float* p, uint16_t* pb, const float* g, float* m, float* v, size_t n, float lr, float b1,
                       float b2, float eps, float c1, float c2) {
    const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    const float gq = g[q];
    const float mq = b1 * m[q] + (1.0f - b1) * gq;
    const float vq = b2 * v[q] + (1.0f - b2) * gq * gq;
    m[q] = mq;
    v[q] = vq;
    const float pq = p[q] - lr * (mq / c1) / (sqrtf(vq / c2) + eps);
    p[q] = pq;
    pb[q] = bf16_bits(pq);
}

inline unsigned blocks(size_t n, unsigned t) { return (unsigned)((n + t - 1) / t); }
inline int launched() { return cudaGetLastError() == cudaSuccess ? 0 : 2; }

}  // namespace

extern "C" {

int ems_learn_gemm_bf16(const uint16_t* A, int64_t sa0, int64_t sa1, const uint16_t* B, int64_t sb0, int64_t sb1,
                        float* C, int64_t ldc, int M, int N, int K, float alpha, float beta, void* stream) {
    if (!A || !B || !C || M <= 0 || N <= 0 || K <= 0) return 1;
    // Element offsets are formed in 64 bits; one grid dimension per tile axis.
    if ((M + GM - 1) / GM > 65535) return 1;
    dim3 grid((N + GN - 1) / GN, (M + GM - 1) / GM);
    k_gemm<<<grid, 128, 0, (cudaStream_t)stream>>>(A, sa0, sa1, B, sb0, sb1, C, ldc, M, N, K, alpha, beta);
    return launched();
}

int ems_learn_to_bf16(const float* src, uint16_t* dst, size_t n, void* stream) {
    if (!n) return 0;
    if (!src || !dst) return 1;
    k_to_bf16<<<blocks(n, 256), 256, 0, (cudaStream_t)stream>>>(src, dst, n);
    return launched();
}

int ems_learn_im2col(const float* x, uint16_t* col, int B, int T, int C, int k, int s, void* stream) {
    if (!x || !col || B <= 0 || C <= 0 || k <= 0 || s <= 0 || T < k) return 1;
    const int To = (T - k) / s + 1;
    const size_t n = (size_t)B * To * k * C;
    k_im2col<<<blocks(n, 256), 256, 0, (cudaStream_t)stream>>>(x, col, B, T, C, k, s, To);
    return launched();
}

int ems_learn_col2im(const float* dcol, float* dx, int B, int T, int C, int k, int s, void* stream) {
    if (!dcol || !dx || B <= 0 || C <= 0 || k <= 0 || s <= 0 || T < k) return 1;
    const int To = (T - k) / s + 1;
    const size_t n = (size_t)B * T * C;
    k_col2im<<<blocks(n, 256), 256, 0, (cudaStream_t)stream>>>(dcol, dx, B, T, C, k, s, To);
    return launched();
}

int ems_learn_bias_act(float* y, const float* bias, float* a, int rows, int cols, int act, void* stream) {
    if (!y || !bias || !a || rows <= 0 || cols <= 0) return 1;
    k_bias_act<<<blocks((size_t)rows * cols, 256), 256, 0, (cudaStream_t)stream>>>(y, bias, a, rows, cols, act);
    return launched();
}

int ems_learn_act_grad(const float* y, const float* da, float* dy, int rows, int cols, int act, void* stream) {
    if (!y || !da || !dy || rows <= 0 || cols <= 0) return 1;
    k_act_grad<<<blocks((size_t)rows * cols, 256), 256, 0, (cudaStream_t)stream>>>(y, da, dy, rows, cols, act);
    return launched();
}

int ems_learn_bias_grad(const float* dy, float* db, int rows, int cols, void* stream) {
    if (!dy || !db || rows <= 0 || cols <= 0) return 1;
    k_bias_grad<<<cols, 256, 0, (cudaStream_t)stream>>>(dy, db, rows, cols);
    return launched();
}

int ems_learn_mse(const float* out, const float* target, float* grad, float* loss, size_t n, void* stream) {
    if (!out || !target || !grad || !loss || !n) return 1;
    k_mse_grad<<<blocks(n, 256), 256, 0, (cudaStream_t)stream>>>(out, target, grad, n);
    k_mse_loss<<<1, 1024, 0, (cudaStream_t)stream>>>(out, target, loss, n);
    return launched();
}

int ems_learn_adam(float* p, uint16_t* p_bf16, const float* g, float* m, float* v, size_t n, float lr, float b1,
                   float b2, float eps, int t, void* stream) {
    if (!p || !p_bf16 || !g || !m || !v || !n || t < 1) return 1;
    const float c1 = 1.0f - powf(b1, (float)t), c2 = 1.0f - powf(b2, (float)t);
    k_adam<<<blocks(n, 256), 256, 0, (cudaStream_t)stream>>>(p, p_bf16, g, m, v, n, lr, b1, b2, eps, c1, c2);
    return launched();
}

}  // extern "C"
