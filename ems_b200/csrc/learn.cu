// learn.cu — kernels of the learned early stop (include/ems_learn.h), sm_100a.
//
// A small 1-D CNN (convolutions as im2col + GEMM, then two dense layers)
// trained and run on these kernels. The GEMM runs on the tcgen05 tensor
// cores (bf16 operands from shared memory, f32 accumulator in tensor
// memory). The matrices here are small (≤ 10^5 rows, ≤ 2·10^3 columns), so
// the kernel takes A and B with arbitrary element strides (a transposed
// operand is just other strides), which keeps the backward pass free of
// transpose copies.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/ems_learn.h"

namespace {

// The GEMM C = alpha·A·B + beta·C on the fifth-generation tensor cores:
// one CTA of four warps per 128×128 tile of C, the f32 accumulator in
// tensor memory (128 lanes × 128 columns), K in chunks of 64. The four
// warps stage each chunk of A (128×64) and B (64×128) in shared memory in
// the no-swizzle K-major core-matrix layout: 8 rows × 8 bf16 (16 bytes per
// row) per core matrix, [k/8][row][8], so that the core matrices of one row
// group lie 128 bytes apart (stride offset) and the two K halves of one
// K=16 step M·16 bytes apart (leading offset). One elected thread issues
// four tcgen05.mma (M 128, N 128, K 16, bf16 in, f32 out) and commits them
// to an mbarrier; the CTA waits on it (bounded) before reusing the buffers.
// Operands are read with arbitrary element strides (a transposed operand
// is other strides), zero outside the matrix.
constexpr int TM = 128, TN = 128, TK = 64;
constexpr uint32_t kTmemCols = 128;
constexpr uint32_t kTileBytesA = TM * TK * 2, kTileBytesB = TN * TK * 2;
// A, B, the barrier, the tensor-memory address; padded so at most three
// CTAs share an SM (3 × 128 tensor-memory columns of the 512).
constexpr uint32_t kGemmSmem = 64 * 1024;
constexpr uint64_t kGemmWaitNs = 1000000000ull;

__device__ int g_learn_fail = 0;

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t now_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Waits for phase `parity`; false after kGemmWaitNs.
__device__ __forceinline__ bool bar_wait(uint64_t* bar, uint32_t parity) {
    uint32_t done = 0;
    const uint64_t t0 = now_ns();
    for (uint32_t it = 0;; ++it) {
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(smem_addr(bar)), "r"(parity)
            : "memory");
        if (done) return true;
        if ((it & 63u) == 63u && now_ns() - t0 > kGemmWaitNs) return false;
    }
}

// Shared-memory matrix descriptor, no swizzle: start, leading and stride
// byte offsets in 16-byte units, version 1 (bits 46-47).
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: f32 accumulator (bits 4-5 = 1), A
// and B bf16 (bits 7-9, 10-12 = 1), both K-major, N/8 at bit 17, M/16 at 24.
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(TN >> 3) << 17) |
                            ((uint32_t)(TM >> 4) << 24);

__global__ void __launch_bounds__(128) k_gemm_tc(const uint16_t* __restrict__ A, int64_t sa0, int64_t sa1,
                                                 const uint16_t* __restrict__ B, int64_t sb0, int64_t sb1, float* C,
                                                 int64_t ldc, int M, int N, int K, float alpha, float beta) {
    extern __shared__ __align__(1024) unsigned char smem[];
    uint16_t* As = reinterpret_cast<uint16_t*>(smem);
    uint16_t* Bs = reinterpret_cast<uint16_t*>(smem + kTileBytesA);
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + kTileBytesA + kTileBytesB);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem + kTileBytesA + kTileBytesB + 8);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.y * TM, n0 = blockIdx.x * TN;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tmem_slot)),
                     "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;
    bool ok = true;
    const int chunks = (K + TK - 1) / TK;
    for (int ch = 0; ch < chunks; ++ch) {
        const int k0 = ch * TK;
        // Stage the chunk: element (r, c) of a 128×64 tile at [c/8][r][c%8].
        for (int e = tid; e < TM * TK; e += 128) {
            const int r = e / TK, c = e - r * TK;
            const int i = m0 + r, k = k0 + c;
            As[((c >> 3) * TM + r) * 8 + (c & 7)] = (i < M && k < K) ? A[i * sa0 + k * sa1] : (uint16_t)0;
        }
        for (int e = tid; e < TN * TK; e += 128) {
            const int r = e / TK, c = e - r * TK;  // r: column n of C, c: k
            const int j = n0 + r, k = k0 + c;
            Bs[((c >> 3) * TN + r) * 8 + (c & 7)] = (j < N && k < K) ? B[k * sb0 + j * sb1] : (uint16_t)0;
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t a0 = smem_addr(As), b0 = smem_addr(Bs);
#pragma unroll
            for (int s = 0; s < TK / 16; ++s) {
                const uint64_t da = smem_desc(a0 + s * 2 * TM * 16, TM * 16, 128);
                const uint64_t db = smem_desc(b0 + s * 2 * TN * 16, TN * 16, 128);
                const uint32_t acc = (ch > 0 || s > 0) ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
                    "l"(da), "l"(db), "r"(kIdesc), "r"(acc)
                    : "memory");
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smem_addr(bar))
                         : "memory");
        }
        if (!bar_wait(bar, (uint32_t)(ch & 1))) ok = false;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    }
    // The epilogue's tensor-memory loads are warp-collective: every thread
    // takes the same branch.
    ok = __syncthreads_and(ok) != 0;
    if (!ok && tid == 0) atomicExch(&g_learn_fail, 1);
    if (ok) {
        // Warp w reads tensor-memory lanes 32w..32w+31: row 32w + lane of the tile.
        const int i = m0 + warp * 32 + lane;
        for (int cb = 0; cb < TN; cb += 16) {
            uint32_t v[16];
            const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)cb;
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, "
                "[%16];"
                : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                  "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
                  "=r"(v[15])
                : "r"(taddr)
                : "memory");
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (i < M) {
#pragma unroll
                for (int q = 0; q < 16; ++q) {
                    const int j = n0 + cb + q;
                    if (j < N) {
                        float* p = C + i * ldc + j;
                        const float x = __uint_as_float(v[q]);
                        *p = beta != 0.0f ? alpha * x + beta * *p : alpha * x;
                    }
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
    }
}

__device__ __forceinline__ uint16_t bf16_bits(float x) { return __bfloat16_as_ushort(__float2bfloat16_rn(x)); }

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
    if ((M + TM - 1) / TM > 65535) return 1;
    static bool attr = false;
    if (!attr) {
        if (cudaFuncSetAttribute(k_gemm_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGemmSmem) != cudaSuccess)
            return 2;
        attr = true;
    }
    dim3 grid((N + TN - 1) / TN, (M + TM - 1) / TM);
    k_gemm_tc<<<grid, 128, kGemmSmem, (cudaStream_t)stream>>>(A, sa0, sa1, B, sb0, sb1, C, ldc, M, N, K, alpha, beta);
    return launched();
}

int ems_learn_check(void) {
    int v = 0;
    if (cudaMemcpyFromSymbol(&v, g_learn_fail, sizeof(int)) != cudaSuccess) return 2;
    if (v) {
        const int zero = 0;
        cudaMemcpyToSymbol(g_learn_fail, &zero, sizeof(int));
        return 4;
    }
    return 0;
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
