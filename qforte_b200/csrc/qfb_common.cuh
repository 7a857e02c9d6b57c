// Shared plumbing of libqfb.so: status codes, the calling thread's stream and
// last-error message, stream-ordered device allocation, launch accounting, and
// the complex128 / bit helpers every kernel uses.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <cstdio>
#include <string>

#include "../../include/qfb.h"

namespace qfb {

// ---- host side ----------------------------------------------------------

extern thread_local std::string t_last_error;
extern thread_local cudaStream_t t_stream;
extern std::atomic<uint64_t> g_launches;

int fail(int code, const char *fmt, ...);
int cuda_fail(cudaError_t e, const char *what);

// Stream-ordered allocation from the device's default pool; the pool keeps
// freed blocks for reuse, so state copies inside a gradient loop cost no
// cudaMalloc and no device synchronisation.
int dev_alloc(void **p, size_t bytes);
void dev_free(void *p);

#define QFB_CUDA(call)                                                       \
    do {                                                                     \
        cudaError_t _e = (call);                                             \
        if (_e != cudaSuccess) return ::qfb::cuda_fail(_e, #call);           \
    } while (0)

#define QFB_LAUNCHED()                                                       \
    do {                                                                     \
        ::qfb::g_launches.fetch_add(1, std::memory_order_relaxed);           \
        cudaError_t _e = cudaGetLastError();                                 \
        if (_e != cudaSuccess) return ::qfb::cuda_fail(_e, "kernel launch"); \
    } while (0)

// Number of SMs of the current device (148 on B200).
int sm_count();

// Grid size for a grid-stride loop over `work` items of `per_block` each:
// capped at `waves` resident waves of 148 SMs.
inline unsigned grid_for(uint64_t work, unsigned per_block, unsigned waves = 8) {
    uint64_t g = (work + per_block - 1) / per_block;
    uint64_t cap = (uint64_t)sm_count() * waves;
    if (g > cap) g = cap;
    if (g < 1) g = 1;
    return (unsigned)g;
}

}  // namespace qfb

struct qfb_state_s {
    int nqubit;
    int nbatch;
    uint64_t nbasis;  // 2^nqubit amplitudes per slot
    double2 *d;       // [nbatch][nbasis]
};

// ---- device side ----------------------------------------------------------

__device__ __forceinline__ double2 c_mul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 c_add(double2 a, double2 b) {
    return make_double2(a.x + b.x, a.y + b.y);
}
// complex64 amplitudes (the throughput-only variant of the gate kernels)
__device__ __forceinline__ float2 c_mul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 c_add(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }

// An amplitude type's scalar, its constructor and the conversion of a
// complex128 matrix entry to it (identities for complex128).
template <class A>
struct AmpT;
template <>
struct AmpT<double2> {
    using S = double;
    __device__ __forceinline__ static double2 make(double re, double im) { return make_double2(re, im); }
    __device__ __forceinline__ static double2 cvt(double2 v) { return v; }
    __device__ __forceinline__ static double2 wide(double2 v) { return v; }
};
template <>
struct AmpT<float2> {
    using S = float;
    __device__ __forceinline__ static float2 make(float re, float im) { return make_float2(re, im); }
    __device__ __forceinline__ static float2 cvt(double2 v) {
        return make_float2((float)v.x, (float)v.y);
    }
    __device__ __forceinline__ static double2 wide(float2 v) { return make_double2(v.x, v.y); }
};
// conj(a) * b
__device__ __forceinline__ double2 c_cjmul(double2 a, double2 b) {
    return make_double2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ double2 c_scale(double2 a, double s) {
    return make_double2(a.x * s, a.y * s);
}
// i^q * v  (q mod 4): exact, no rounding.
__device__ __forceinline__ double2 c_ipow(double2 v, int q) {
    double2 r = (q & 1) ? make_double2(-v.y, v.x) : v;
    return (q & 2) ? make_double2(-r.x, -r.y) : r;
}
__device__ __forceinline__ int parity64(uint64_t v) { return __popcll(v) & 1; }

// Insert a 0 bit at position `pos` of `p`.
__device__ __forceinline__ uint64_t insert0(uint64_t p, int pos) {
    const uint64_t lo = p & ((1ull << pos) - 1ull);
    return ((p >> pos) << (pos + 1)) | lo;
}

__device__ __forceinline__ double2 warp_sum(double2 v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        v.x += __shfl_down_sync(0xffffffffu, v.x, o);
        v.y += __shfl_down_sync(0xffffffffu, v.y, o);
    }
    return v;
}

// Sum over the block (any blockDim multiple of 32, <= 1024); result valid in
// thread 0.  Fixed reduction tree, so results are run-to-run identical.
__device__ __forceinline__ double2 block_sum(double2 v) {
    __shared__ double2 s_warp[32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    v = warp_sum(v);
    if (lane == 0) s_warp[wid] = v;
    __syncthreads();
    const int nw = blockDim.x >> 5;
    v = (threadIdx.x < nw) ? s_warp[threadIdx.x] : make_double2(0.0, 0.0);
    if (wid == 0) v = warp_sum(v);
    __syncthreads();
    return v;
}
