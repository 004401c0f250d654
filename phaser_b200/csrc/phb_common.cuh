// Shared device helpers of the phaser_b200 kernels (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cmath>

#include "../../include/phaser_b200.h"

namespace phb {

// ------------------------------------------------------------------ complex
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b)
__device__ __forceinline__ float2 cmulc(float2 a, float2 b) {
    return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
__device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
// complex add / subtract / real scale as one packed FP32 instruction each (sm_100
// FADD2 / FMUL2: two round-to-nearest float32 operations, the same results as two scalar
// ones; the compiler does not pair scalar float2 arithmetic by itself)
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) {
    unsigned long long ra = *reinterpret_cast<unsigned long long *>(&a), rb = *reinterpret_cast<unsigned long long *>(&b),
                       rd;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(rd) : "l"(ra), "l"(rb));
    return *reinterpret_cast<float2 *>(&rd);
}
__device__ __forceinline__ float2 cscale(float2 a, float s) { return __fmul2_rn(a, make_float2(s, s)); }
__device__ __forceinline__ float cabs2(float2 a) { return a.x * a.x + a.y * a.y; }

// numpy.maximum(x, 0) semantics: NaN propagates (CUDA's fmaxf would drop it).
__device__ __forceinline__ float np_max0(float x) { return (x != x) ? x : (x > 0.f ? x : 0.f); }

__device__ __forceinline__ bool finite2(float2 a) { return isfinite(a.x) && isfinite(a.y); }

// ------------------------------------------------------ bounds-checking build
// Compiled with -DPHB_BOUNDS_CHECK=1 (libphaser_b200_bounds.so), every kernel that
// dereferences a caller-supplied position index (a row of `group`) checks it against
// n_pos first: an index outside [0, n_pos) is recorded (bit 2 of the workspace error
// word, PHB_STATUS_BOUNDS | group index in the step's status) and the position is
// skipped instead of read or written out of bounds.  The default build has no checks.
#ifndef PHB_BOUNDS_CHECK
#define PHB_BOUNDS_CHECK 0
#endif
__device__ __forceinline__ bool pos_ok(long long p, long long n_pos) {
#if PHB_BOUNDS_CHECK
    return p >= 0 && p < n_pos;
#else
    (void)p;
    (void)n_pos;
    return true;
#endif
}
__device__ __forceinline__ void report_bounds(int32_t *err_word, int32_t *status, int32_t group_index) {
    if (err_word) atomicOr(err_word, 2);
    if (status) atomicCAS(status, -1, PHB_STATUS_BOUNDS | group_index);
}

// ------------------------------------------------------ exact cutout indices
// (pos - corner) / sampling - (n - 1)/2, float64 with no contraction, then
// round-half-to-even: the same IEEE operations, in the same order, as
// phaser/utils/object.py:291-301 followed by numpy.round (object.py:493-495).
struct CutoutIndex {
    long long y0, x0;   // integer cutout start
    float sy, sx;       // sub-pixel shift in length units (float32, as fourier_shift_filter casts)
};

__device__ __host__ __forceinline__ double exact_index(float pos, double corner, double samp, long long n) {
#ifdef __CUDA_ARCH__
    double half = -fmax(0.0, (double)n - 1.0) / 2.0;          // exact for integer n
    double v = __ddiv_rn(__dsub_rn((double)pos, corner), samp);
    return __dadd_rn(v, half);
#else
    double half = -std::fmax(0.0, (double)n - 1.0) / 2.0;
    volatile double d = (double)pos - corner;
    volatile double q = d / samp;
    return q + half;
#endif
}

__device__ __forceinline__ CutoutIndex cutout_index(const float *scan, long long p, double cy, double cx,
                                                    double sy, double sx, long long ny, long long nx) {
    CutoutIndex r;
    double iy = exact_index(scan[2 * p + 0], cy, sy, ny);
    double ix = exact_index(scan[2 * p + 1], cx, sx, nx);
    double ry = rint(iy), rx = rint(ix);   // rint: round half to even
    r.y0 = (long long)ry;
    r.x0 = (long long)rx;
    r.sy = (float)__dmul_rn(__dsub_rn(iy, ry), sy);
    r.sx = (float)__dmul_rn(__dsub_rn(ix, rx), sx);
    return r;
}

// ------------------------------------------------------------ reductions
template <int NT>
__device__ __forceinline__ void block_sum_doubles(double *vals, int K, double *smem /* >= NT/32*K */) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int k = 0; k < K; ++k) {
        double v = vals[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) smem[warp * K + k] = v;
    }
    __syncthreads();
    if (warp == 0) {
        for (int k = 0; k < K; ++k) {
            double v = (lane < NT / 32) ? smem[lane * K + k] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            vals[k] = v;
        }
    }
    __syncthreads();
    // result valid in warp 0; broadcast
    if (threadIdx.x == 0)
        for (int k = 0; k < K; ++k) smem[k] = vals[k];
    __syncthreads();
    for (int k = 0; k < K; ++k) vals[k] = smem[k];
    __syncthreads();
}

template <int NT>
__device__ __forceinline__ float block_max_float(float v, float *smem) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    if (lane == 0) smem[warp] = v;
    __syncthreads();
    if (warp == 0) {
        float w = (lane < NT / 32) ? smem[lane] : -INFINITY;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) w = fmaxf(w, __shfl_xor_sync(0xffffffffu, w, o));
        if (lane == 0) smem[0] = w;
    }
    __syncthreads();
    float r = smem[0];
    __syncthreads();
    return r;
}

// Warp-level float64 sum; lane 0 adds it to *dst.  Call from uniform code (all 32 lanes).
__device__ __forceinline__ void warp_atomic_sum(double *dst, double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(dst, v);
}

// Bulk prefetch of a contiguous, 16-byte aligned global range into L2 (sm_90+);
// `bytes` a multiple of 16.  Issued by one thread; it does not block.
__device__ __forceinline__ void prefetch_l2(const void *ptr, uint32_t bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(ptr), "r"(bytes) : "memory");
}

// Vector fp32 atomics (sm_90+): one red per complex value.
__device__ __forceinline__ void atomic_add_c(float2 *addr, float2 v) {
    atomicAdd(addr, v);
}

}  // namespace phb
