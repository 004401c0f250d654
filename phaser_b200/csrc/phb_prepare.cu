// State preparation in front of the engines (phaser/execute.py:334-402):
// resampling of probe, patterns, pattern mask and object onto the engine's
// grids, and reslicing of the object along z.
//
// Resampling restates scipy.ndimage.affine_transform with order 1 and mode
// 'grid-constant' for the diagonal matrices the preparation uses
// (phaser/utils/num.py:713-750, phaser/utils/object.py:430-467): output pixel
// (i, j) is the bilinear interpolation of the input, extended by a constant
// beyond its edges, at (m_y i + o_y, m_x j + o_x).  Coordinates and weights are
// float64 (as scipy computes them); the reciprocal-space form reads the input
// through fftshift and writes the output through ifftshift
// (Sampling.resample_recip), both folded into the index arithmetic.  One thread
// per output element; the input rows a warp touches are contiguous, so the
// kernel streams at HBM rate (4 gathered reads, mostly from L1/L2, and one
// write per element).
//
// Reslicing restates resample_slices (phaser/utils/object.py:56-157): per
// pixel, log(obj) / thickness is interpolated linearly at the new slice
// centres (edge values outside), multiplied by the new thickness and
// exponentiated.  The per-slice interpolation table (two source slices and
// their weights) is computed on the host and passed by value.
#include "phb_common.cuh"
#include "phb_runtime.h"

namespace phb {

template <typename T>
struct Cval;
template <>
struct Cval<float2> {
    float2 v;
};
template <>
struct Cval<float> {
    float v;
};

__device__ __forceinline__ float2 axpy(double w, float2 v, float2 acc) {
    return make_float2(acc.x + (float)w * v.x, acc.y + (float)w * v.y);
}
__device__ __forceinline__ float axpy(double w, float v, float acc) { return acc + (float)w * v; }
__device__ __forceinline__ float2 zero_of(float2) { return make_float2(0.f, 0.f); }
__device__ __forceinline__ float zero_of(float) { return 0.f; }

// source row of coordinate y in an axis of n samples, through fftshift when recip
__device__ __forceinline__ int64_t src_index(int64_t y, int64_t n, int recip) {
    if (!recip) return y;
    int64_t s = (y - n / 2) % n;
    return s < 0 ? s + n : s;
}

template <typename T>
__global__ void __launch_bounds__(256) k_resample(const T *in, int64_t batch, int H, int W, T *out, int Ho, int Wo,
                                                  double my, double mx, double oy, double ox, Cval<T> cval,
                                                  int recip) {
    const int64_t n = batch * Ho * Wo;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t b = e / ((int64_t)Ho * Wo);
        const int i = (int)((e / Wo) % Ho), j = (int)(e % Wo);
        // output index -> resampled-grid index (ifftshift of the result when recip)
        const int ri = recip ? (i + Ho / 2) % Ho : i, rj = recip ? (j + Wo / 2) % Wo : j;
        const double cy = my * ri + oy, cx = mx * rj + ox;
        const double fy = floor(cy), fx = floor(cx);
        const int64_t y0 = (int64_t)fy, x0 = (int64_t)fx;
        const double ty = cy - fy, tx = cx - fx;
        const T *src = in + b * H * W;
        T acc = zero_of(cval.v);
#pragma unroll
        for (int dy = 0; dy < 2; ++dy) {
            const int64_t y = y0 + dy;
            const double wy = dy ? ty : 1.0 - ty;
            const bool iny = y >= 0 && y < H;
            const int64_t sy = iny ? src_index(y, H, recip) : 0;
#pragma unroll
            for (int dx = 0; dx < 2; ++dx) {
                const int64_t x = x0 + dx;
                const double w = wy * (dx ? tx : 1.0 - tx);
                const bool in_ = iny && x >= 0 && x < W;
                const T v = in_ ? src[sy * W + src_index(x, W, recip)] : cval.v;
                acc = axpy(w, v, acc);
            }
        }
        out[e] = acc;
    }
}

constexpr int MAX_SLICES = 128;

// z interpolation table: output slice i = exp(new_t[i] * (wa[i] L(ja[i]) + wb[i] L(jb[i])))
// with L(k) = log(obj[k - 1]) / old_t[k - 1] for 1 <= k <= S_old and the padding
// slice for k = 0 and k = S_old + 1
struct ZTable {
    int ja[MAX_SLICES], jb[MAX_SLICES];
    float wa[MAX_SLICES], wb[MAX_SLICES], new_t[MAX_SLICES], inv_old_t[MAX_SLICES];
};

__device__ __forceinline__ float2 clog(float2 z) { return make_float2(logf(hypotf(z.x, z.y)), atan2f(z.y, z.x)); }

__global__ void __launch_bounds__(256) k_reslice(const float2 *obj, int S_old, int64_t HW, float2 *out, int S_new,
                                                 int pad_mode, const ZTable tab) {
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < HW; p += (int64_t)gridDim.x * blockDim.x) {
        float2 pad_lo = make_float2(0.f, 0.f), pad_hi = pad_lo;   // vacuum
        if (pad_mode == 1) {                                       // edge slices
            pad_lo = cscale(clog(obj[p]), tab.inv_old_t[0]);
            pad_hi = cscale(clog(obj[(int64_t)(S_old - 1) * HW + p]), tab.inv_old_t[S_old - 1]);
        } else if (pad_mode == 2) {                                // mean over slices, NaNs skipped
            float2 s = make_float2(0.f, 0.f);
            int cr = 0, ci = 0;
            float sr = 0.f, si = 0.f;
            for (int k = 0; k < S_old; ++k) {
                const float2 l = cscale(clog(obj[(int64_t)k * HW + p]), tab.inv_old_t[k]);
                if (l.x == l.x) sr += l.x, ++cr;
                if (l.y == l.y) si += l.y, ++ci;
            }
            s.x = cr ? sr / cr : __int_as_float(0x7fc00000);
            s.y = ci ? si / ci : __int_as_float(0x7fc00000);
            pad_lo = pad_hi = s;
        }
        for (int i = 0; i < S_new; ++i) {
            float2 v = make_float2(0.f, 0.f);
            const int js[2] = {tab.ja[i], tab.jb[i]};
            const float ws[2] = {tab.wa[i], tab.wb[i]};
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                if (ws[q] == 0.f) continue;
                const int k = js[q];
                const float2 l = k == 0 ? pad_lo
                                        : k == S_old + 1 ? pad_hi
                                                         : cscale(clog(obj[(int64_t)(k - 1) * HW + p]),
                                                                  tab.inv_old_t[k - 1]);
                v = make_float2(v.x + ws[q] * l.x, v.y + ws[q] * l.y);
            }
            v = cscale(v, tab.new_t[i]);
            float sn, cs;
            sincosf(v.y, &sn, &cs);
            const float a = expf(v.x);
            out[(int64_t)i * HW + p] = make_float2(a * cs, a * sn);
        }
    }
}

}  // namespace phb

using namespace phb;

static inline unsigned grid_for(int64_t n) {
    int64_t g = (n + 255) / 256;
    if (g > 148 * 32) g = 148 * 32;
    return (unsigned)(g < 1 ? 1 : g);
}

extern "C" {

int phb_resample_c64(const void *in, int64_t batch, int32_t H, int32_t W, void *out, int32_t Ho, int32_t Wo,
                     double my, double mx, double oy, double ox, float cval_re, float cval_im, int32_t recip,
                     void *stream) {
    if (!in || !out || batch < 1 || H < 1 || W < 1 || Ho < 1 || Wo < 1) return PHB_ERR_INVALID_ARG;
    Cval<float2> c{make_float2(cval_re, cval_im)};
    k_resample<float2><<<grid_for(batch * Ho * Wo), 256, 0, (cudaStream_t)stream>>>(
        (const float2 *)in, batch, H, W, (float2 *)out, Ho, Wo, my, mx, oy, ox, c, recip ? 1 : 0);
    return check_launch();
}

int phb_resample_f32(const float *in, int64_t batch, int32_t H, int32_t W, float *out, int32_t Ho, int32_t Wo,
                     double my, double mx, double oy, double ox, float cval, int32_t recip, void *stream) {
    if (!in || !out || batch < 1 || H < 1 || W < 1 || Ho < 1 || Wo < 1) return PHB_ERR_INVALID_ARG;
    Cval<float> c{cval};
    k_resample<float><<<grid_for(batch * Ho * Wo), 256, 0, (cudaStream_t)stream>>>(
        in, batch, H, W, out, Ho, Wo, my, mx, oy, ox, c, recip ? 1 : 0);
    return check_launch();
}

int phb_resample_slices_c64(const void *obj, int32_t S_old, int64_t HW, const float *old_t, void *out,
                            int32_t S_new, const float *new_t, const int32_t *ja, const int32_t *jb,
                            const float *wa, const float *wb, int32_t pad_mode, void *stream) {
    if (!obj || !out || !old_t || !new_t || !ja || !jb || !wa || !wb || HW < 1) return PHB_ERR_INVALID_ARG;
    if (S_old < 1 || S_old > MAX_SLICES || S_new < 1 || S_new > MAX_SLICES || pad_mode < 0 || pad_mode > 2)
        return PHB_ERR_INVALID_ARG;
    ZTable tab;
    for (int k = 0; k < S_old; ++k) {
        if (!(old_t[k] > 0.f)) return PHB_ERR_INVALID_ARG;
        tab.inv_old_t[k] = 1.f / old_t[k];
    }
    for (int i = 0; i < S_new; ++i) {
        if (ja[i] < 0 || ja[i] > S_old + 1 || jb[i] < 0 || jb[i] > S_old + 1) return PHB_ERR_INVALID_ARG;
        tab.ja[i] = ja[i], tab.jb[i] = jb[i], tab.wa[i] = wa[i], tab.wb[i] = wb[i], tab.new_t[i] = new_t[i];
    }
    k_reslice<<<grid_for(HW), 256, 0, (cudaStream_t)stream>>>((const float2 *)obj, S_old, HW, (float2 *)out, S_new,
                                                              pad_mode, tab);
    return check_launch();
}

}  // extern "C"
