// noalloc.cu — the energy invariant of a field state, computed without any
// device allocation (include/ems_gpu.h, ems_energy_noalloc).
//
// Some hosts cannot call cudaMalloc when they need this number: a solver
// embedded in a framework that owns all device memory through its own pool,
// or a real-time loop that must not allocate after start-up. This entry
// point takes the caller's device arrays and writes the result to a
// caller-provided device double; its only working memory is a file-scope
// __device__ array of kMaxBlocks partial sums (16 KiB) that every GPU which
// loads the library holds until the process exits.
#include <cuda_runtime.h>

#include <cfloat>
#include <cstdint>
#include <mutex>

#include "../../include/ems_gpu.h"
#include "arith.cuh"

namespace {

// Partial sums of one call: one per block of the first pass. The grid never
// exceeds kMaxBlocks blocks; a grid-stride loop covers any node count.
constexpr unsigned kMaxBlocks = 2048;
constexpr unsigned kThreads = 256;
// Nodes are indexed with 32-bit integers: at most this many per array.
constexpr uint64_t kMaxNodes = 0x7fffffffull;

static __device__ __align__(256) double scratch[kMaxBlocks];

struct Arrays {
    const float* u[3];
    const float* i[3];
    const float* c[12];
};

// One node's share of W^n in units of dt/4: Σ_a (1 + ca)/cb·u_a² and, for
// each dual edge the H update changes, (1 + da)/db·i_old·i_new, with i_new
// the H update's value (not stored) — the expressions of the engine's H
// kernel (src/engine/kernel.rs:132-244).
__device__ __forceinline__ double node_energy(const Arrays& A, uint32_t nx, uint32_t ny, uint32_t nz, uint32_t n) {
    const uint32_t k = n % nz, r = n / nz, j = r % ny, i = r / ny;
    const uint32_t sj = nz, si = ny * nz;
    const float ux = A.u[0][n], uy = A.u[1][n], uz = A.u[2][n];
    double w = 0.0;
    w = __dadd_rn(w, emsk::weight(A.c[0][n], __dmul_rn((double)ux, (double)ux), A.c[3][n]));
    w = __dadd_rn(w, emsk::weight(A.c[1][n], __dmul_rn((double)uy, (double)uy), A.c[4][n]));
    w = __dadd_rn(w, emsk::weight(A.c[2][n], __dmul_rn((double)uz, (double)uz), A.c[5][n]));
    if (j + 1 < ny && k + 1 < nz) {
        const float old = A.i[0][n], da = A.c[6][n], db = A.c[9][n];
        const float nw = emsk::h_upd(da, old, db, A.u[2][n + sj], uz, A.u[1][n + 1], uy);
        w = __dadd_rn(w, emsk::weight(da, __dmul_rn((double)old, (double)nw), db));
    }
    if (i + 1 < nx && k + 1 < nz) {
        const float old = A.i[1][n], da = A.c[7][n], db = A.c[10][n];
        const float nw = emsk::h_upd(da, old, db, A.u[0][n + 1], ux, A.u[2][n + si], uz);
        w = __dadd_rn(w, emsk::weight(da, __dmul_rn((double)old, (double)nw), db));
    }
    if (i + 1 < nx && j + 1 < ny) {
        const float old = A.i[2][n], da = A.c[8][n], db = A.c[11][n];
        const float nw = emsk::h_upd(da, old, db, A.u[1][n + si], uy, A.u[0][n + sj], ux);
        w = __dadd_rn(w, emsk::weight(da, __dmul_rn((double)old, (double)nw), db));
    }
    return w;
}

__global__ void __launch_bounds__(kThreads) k_energy_partials(const __grid_constant__ Arrays A, uint32_t nx, uint32_t ny,
                                                              uint32_t nz, double* partials) {
    const uint32_t total = nx * ny * nz;
    double w = 0.0;
    for (uint32_t n = blockIdx.x * kThreads + threadIdx.x; n < total; n += gridDim.x * kThreads)
        w = __dadd_rn(w, node_energy(A, nx, ny, nz, n));
    const double s = emsk::block_sum<kThreads>(w);
    if (threadIdx.x == 0) partials[blockIdx.x] = s;
}

__global__ void __launch_bounds__(1024) k_energy_total(const double* partials, unsigned blocks, double scale,
                                                       double* out) {
    double s = 0.0;
    for (unsigned q = threadIdx.x; q < blocks; q += blockDim.x) s = __dadd_rn(s, partials[q]);
    const double t = emsk::block_sum<1024>(s);
    if (threadIdx.x == 0) out[0] = __dmul_rn(scale, t);
}

// The device address of `scratch` on each device, found once per device
// (cudaGetSymbolAddress with that device current), for device ordinals
// 0..kMaxDevices-1. An address stays cached after a cudaDeviceReset of its
// device, when it no longer holds.
constexpr int kMaxDevices = 64;
std::mutex g_mu;
double* g_scratch[kMaxDevices] = {};

ems_status scratch_on(int device, double** out) {
    if (device < 0 || device >= kMaxDevices) return EMS_ERR_INVALID;
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch[device]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, scratch) != cudaSuccess) return EMS_ERR_CUDA;
        g_scratch[device] = (double*)p;
    }
    *out = g_scratch[device];
    return EMS_OK;
}

}  // namespace

extern "C" ems_status ems_energy_noalloc(const uint64_t nodes[3], double dt, const float* const u[3],
                                         const float* const i[3], const float* const coeff[12], double* energy,
                                         void* stream) {
    if (!nodes || !u || !i || !coeff || !energy || !(dt > 0.0)) return EMS_ERR_INVALID;
    if (nodes[0] < 2 || nodes[1] < 2 || nodes[2] < 2) return EMS_ERR_INVALID;
    // The product is checked factor by factor, so it cannot wrap: beyond
    // kMaxNodes the kernel's 32-bit node indexing would not hold.
    if (nodes[0] > kMaxNodes || nodes[1] > kMaxNodes / nodes[0]) return EMS_ERR_INVALID;
    if (nodes[2] > kMaxNodes / (nodes[0] * nodes[1])) return EMS_ERR_INVALID;
    const uint64_t n = nodes[0] * nodes[1] * nodes[2];
    Arrays A;
    for (int a = 0; a < 3; ++a) {
        if (!u[a] || !i[a]) return EMS_ERR_INVALID;
        A.u[a] = u[a];
        A.i[a] = i[a];
    }
    for (int l = 0; l < 12; ++l) {
        if (!coeff[l]) return EMS_ERR_INVALID;
        A.c[l] = coeff[l];
    }
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess) return EMS_ERR_CUDA;
    double* part = nullptr;
    ems_status st = scratch_on(device, &part);
    if (st) return st;
    cudaStream_t s = (cudaStream_t)stream;
    const uint64_t want = (n + kThreads - 1) / kThreads;
    const unsigned blocks = (unsigned)(want < kMaxBlocks ? want : kMaxBlocks);
    // Every partial the second pass reads is written by the first: nothing
    // in the scratch array has to start at zero.
    k_energy_partials<<<blocks, kThreads, 0, s>>>(A, (uint32_t)nodes[0], (uint32_t)nodes[1], (uint32_t)nodes[2], part);
    k_energy_total<<<1, 1024, 0, s>>>(part, blocks, 0.25 * dt, energy);
    return cudaGetLastError() == cudaSuccess ? EMS_OK : EMS_ERR_CUDA;
}
