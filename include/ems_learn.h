/* ems_learn.h — kernels of the learned early stop (libems_learn.so, sm_100a).
 *
 * No counterpart in the reference. The reference ends a run by its energy
 * criterion (src/engine/run.rs:231-262) or by the Settle spectral-tail rule
 * (src/engine/run.rs:309-382); this library adds a small 1-D convolutional
 * network that reads the first K samples of a port's voltage and current and
 * predicts the rest of the ring-down, so a run can stop early. The training
 * (forward, backward, Adam) and inference run on these kernels; the host
 * composes them (ems_b200/learn.py). All pointers are device pointers; every
 * call is asynchronous in `stream` (a cudaStream_t, NULL: legacy default).
 *
 * Layouts: activations channels-last, x[b][t][c], f32; weights of a layer
 * with fan-in F and C outputs as W[C][F] (a convolution's F = k * c_in in
 * (tap, channel) order), f32 masters with bf16 copies for the GEMMs;
 * bf16 values are uint16_t bit patterns (round to nearest even). */
#ifndef EMS_LEARN_H
#define EMS_LEARN_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* C[i][j] = alpha * sum_k A(i,k) B(k,j) + beta * C[i][j] with
 * A(i,k) = A[i*sa0 + k*sa1], B(k,j) = B[k*sb0 + j*sb1] (bf16), C f32 with
 * row stride ldc: tcgen05 tensor-core MMA (bf16 operands staged in shared
 * memory, f32 accumulator in tensor memory), 128x128 tiles of C.
 * beta = 0 ignores C's old contents. Returns 0, 1 for invalid sizes or 2
 * for a launch error; a bounded wait inside the kernel that ran out is
 * reported by ems_learn_check. */
int ems_learn_gemm_bf16(const uint16_t* A, int64_t sa0, int64_t sa1, const uint16_t* B, int64_t sb0, int64_t sb1,
                        float* C, int64_t ldc, int M, int N, int K, float alpha, float beta, void* stream);

/* 0, or 4 (and clears the flag) if a GEMM's bounded wait for its tensor-core
 * work ran out since the last call; 2 if the flag cannot be read. */
int ems_learn_check(void);

/* dst[q] = bf16(src[q]) for q < n. */
int ems_learn_to_bf16(const float* src, uint16_t* dst, size_t n, void* stream);

/* Columns of a valid 1-D convolution (kernel k, stride s) of x[b][T][c]:
 * col[(b*T_out + t)][(tap*c + ch)] = bf16(x[b][t*s + tap][ch]),
 * T_out = (T - k)/s + 1. */
int ems_learn_im2col(const float* x, uint16_t* col, int B, int T, int C, int k, int s, void* stream);

/* The adjoint of im2col: dx[b][t][ch] = sum over (t_out, tap) with
 * t_out*s + tap = t of dcol[(b*T_out + t_out)][(tap*C + ch)] (a gather, in
 * a fixed order). */
int ems_learn_col2im(const float* dcol, float* dx, int B, int T, int C, int k, int s, void* stream);

/* y[r][j] += bias[j]; a[r][j] = act(y[r][j]) (act 0: identity, 1: SiLU). */
int ems_learn_bias_act(float* y, const float* bias, float* a, int rows, int cols, int act, void* stream);

/* dy[r][j] = da[r][j] * act'(y[r][j]) (y the pre-activation). */
int ems_learn_act_grad(const float* y, const float* da, float* dy, int rows, int cols, int act, void* stream);

/* db[j] = sum_r dy[r][j] (rows in order, per column). */
int ems_learn_bias_grad(const float* dy, float* db, int rows, int cols, void* stream);

/* Mean squared error of out against target (n values): loss[0] and
 * grad = 2 (out - target) / n. */
int ems_learn_mse(const float* out, const float* target, float* grad, float* loss, size_t n, void* stream);

/* One Adam step on n parameters (f32 masters), with their bf16 copies
 * refreshed: m = b1 m + (1-b1) g; v = b2 v + (1-b2) g^2;
 * p -= lr * (m / (1 - b1^t)) / (sqrt(v / (1 - b2^t)) + eps). */
int ems_learn_adam(float* p, uint16_t* p_bf16, const float* g, float* m, float* v, size_t n, float lr, float b1,
                   float b2, float eps, int t, void* stream);

#ifdef __cplusplus
}
#endif

#endif
