// Standalone numerics entry points: cutout indices, gather / scatter-add /
// set of object cutouts, and the batched centred orthonormal 2D FFT.
//
// These are the sm_100a forms of phaser/utils/object.py (ObjectCutout) and
// phaser/utils/num.py (fft2 / ifft2).  The fused engine in phb_engine.cu does
// the same work inside its own kernel; these calls serve the array-level API
// and the parity tests.
#include "phb_fft.cuh"
#include "phb_runtime.h"

namespace phb {

// ------------------------------------------------------------------ starts
__global__ void k_cutout_starts(const float *scan, const int64_t *group, int64_t B, double cy, double cx,
                                double sy, double sx, int64_t ny, int64_t nx, int64_t *starts, float *subpx) {
    int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= B) return;
    int64_t p = group ? group[b] : b;
    CutoutIndex ci = cutout_index(scan, p, cy, cx, sy, sx, ny, nx);
    starts[2 * b] = ci.y0;
    starts[2 * b + 1] = ci.x0;
    if (subpx) {
        subpx[2 * b] = ci.sy;
        subpx[2 * b + 1] = ci.sx;
    }
}

// ------------------------------------------------------------ gather / add
// One thread per output element; rows of a cutout are contiguous, so a warp
// reads/writes contiguous spans of the object row.
template <typename T>
__global__ void k_cutout_get(const T *obj, int64_t S, int64_t H, int64_t W, const int64_t *starts,
                             int64_t B, int64_t cy, int64_t cx, T fill, T *out) {
    const int64_t total = B * S * cy * cx;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (int64_t)gridDim.x * blockDim.x) {
        int64_t j = i % cx, t = i / cx;
        int64_t r = t % cy;
        t /= cy;
        int64_t s = t % S, b = t / S;
        int64_t y = r + starts[2 * b], x = j + starts[2 * b + 1];
        out[i] = (y >= 0 && y < H && x >= 0 && x < W) ? obj[(s * H + y) * W + x] : fill;
    }
}

template <int OP>   // 0 = add, 1 = set
__global__ void k_cutout_put_c64(float2 *obj, int64_t S, int64_t H, int64_t W, const int64_t *starts,
                                 int64_t B, int64_t cy, int64_t cx, const float2 *views) {
    const int64_t total = B * S * cy * cx;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (int64_t)gridDim.x * blockDim.x) {
        int64_t j = i % cx, t = i / cx;
        int64_t r = t % cy;
        t /= cy;
        int64_t s = t % S, b = t / S;
        int64_t y = r + starts[2 * b], x = j + starts[2 * b + 1];
        if (y < 0 || y >= H || x < 0 || x >= W) continue;
        float2 *dst = obj + (s * H + y) * W + x;
        if (OP == 0) atomic_add_c(dst, views[i]);
        else *dst = views[i];
    }
}

__global__ void k_cutout_add_f32(float *obj, int64_t S, int64_t H, int64_t W, const int64_t *starts,
                                 int64_t B, int64_t cy, int64_t cx, const float *views) {
    const int64_t total = B * S * cy * cx;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (int64_t)gridDim.x * blockDim.x) {
        int64_t j = i % cx, t = i / cx;
        int64_t r = t % cy;
        t /= cy;
        int64_t s = t % S, b = t / S;
        int64_t y = r + starts[2 * b], x = j + starts[2 * b + 1];
        if (y < 0 || y >= H || x < 0 || x >= W) continue;
        atomicAdd(obj + (s * H + y) * W + x, views[i]);
    }
}

// --------------------------------------------------------------- batched FFT
// One CTA per N x N tile (N = 256: one cluster of 4 CTAs).  fft2: out = (-1)^(ky+kx)
// DFT(in) / N  (== the ifftshift-then-FFT convention for even N); ifft2: out =
// IDFT((-1)^(ky+kx) in) / N.
template <int N>
__global__ void __launch_bounds__(FFT_THREADS, 1) k_fft2_centred(const float2 *in, float2 *out, int inverse) {
    using I = Idx<N>;
    constexpr int U = I::U, E = I::E;
    extern __shared__ float4 smem_raw[];
    float2 *xb = reinterpret_cast<float2 *>(smem_raw);
    float2 *twid = xb + Lay<N>::BUF;
    fft_init_twiddles<N>(twid);
    const size_t tile = blockIdx.x / TileCfg<N>::CTAS;
    const float2 *src = in + tile * N * N;
    float2 *dst = out + tile * N * N;
    float2 v[U][E];
    const float scale = 1.0f / (float)N;
    if (!inverse) {
#pragma unroll
        for (int u = 0; u < U; ++u)
#pragma unroll
            for (int q = 0; q < E; ++q) v[u][q] = src[I::row(u, q) * N + I::col(u, q)];
        __syncthreads();
        fft2_r2k<N>(v, xb, twid);
#pragma unroll
        for (int u = 0; u < U; ++u)
#pragma unroll
            for (int e = 0; e < E; ++e) {
                int ky = I::ky(u, e), kx = I::kx(u, e);
                float s = ((ky + kx) & 1) ? -scale : scale;
                dst[ky * N + kx] = cscale(v[u][e], s);
            }
    } else {
#pragma unroll
        for (int u = 0; u < U; ++u)
#pragma unroll
            for (int e = 0; e < E; ++e) {
                int ky = I::ky(u, e), kx = I::kx(u, e);
                float s = ((ky + kx) & 1) ? -scale : scale;
                v[u][e] = cscale(src[ky * N + kx], s);
            }
        __syncthreads();
        ifft2_k2r<N>(v, xb, twid);
#pragma unroll
        for (int u = 0; u < U; ++u)
#pragma unroll
            for (int q = 0; q < E; ++q) dst[I::row(u, q) * N + I::col(u, q)] = v[u][q];
    }
}

template <int N>
static int launch_fft2(const float2 *in, float2 *out, int64_t batch, int inverse, cudaStream_t st) {
    const size_t smem = (size_t)Lay<N>::BUF * sizeof(float2) + TileCfg<N>::TW * sizeof(float2);
    static bool configured = false;
    if (!configured) {
        if (cudaFuncSetAttribute(k_fft2_centred<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
            return PHB_ERR_CUDA;
        configured = true;
    }
    // in-place is safe: each CTA reads its part of the tile into registers before the
    // first exchange, and writes after the last one
    constexpr unsigned C = TileCfg<N>::CTAS;
    return launch_clustered(k_fft2_centred<N>, (unsigned)batch * C, FFT_THREADS, C, smem, st, in, out, inverse);
}

// ------------------------------------------------------------- constraints
// obj *= min(|obj|, amp) / |obj|  (phaser/engines/common/regularizers.py:36-42; 0/0 -> NaN as in numpy)
__global__ void k_clamp_amplitude(float2 *a, int64_t n, float amp) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        float2 v = a[i];
        const float mag = sqrtf(v.x * v.x + v.y * v.y);
        const float s = fminf(mag, amp) / mag;
        a[i] = make_float2(v.x * s, v.y * s);
    }
}

// a = ifft2(fft2(a) * mask), mask (N, N) in the zero-frequency-in-corner layout
// (LimitProbeSupport, phaser/engines/common/regularizers.py:45-64; ObjLowPass-style filters).
template <int N>
__global__ void __launch_bounds__(FFT_THREADS, 1) k_fourier_mask(float2 *a, const float *mask) {
    using I = Idx<N>;
    constexpr int U = I::U, E = I::E;
    extern __shared__ float4 smem_raw[];
    float2 *xb = reinterpret_cast<float2 *>(smem_raw);
    float2 *twid = xb + Lay<N>::BUF;
    fft_init_twiddles<N>(twid);
    float2 *t = a + (size_t)(blockIdx.x / TileCfg<N>::CTAS) * N * N;
    float2 v[U][E];
#pragma unroll
    for (int u = 0; u < U; ++u)
#pragma unroll
        for (int q = 0; q < E; ++q) v[u][q] = t[I::row(u, q) * N + I::col(u, q)];
    __syncthreads();
    fft2_r2k<N>(v, xb, twid);
    const float sc = 1.0f / (float)(N * N);
#pragma unroll
    for (int u = 0; u < U; ++u)
#pragma unroll
        for (int e = 0; e < E; ++e) v[u][e] = cscale(v[u][e], sc * __ldg(mask + I::ky(u, e) * N + I::kx(u, e)));
    ifft2_k2r<N>(v, xb, twid);
#pragma unroll
    for (int u = 0; u < U; ++u)
#pragma unroll
        for (int q = 0; q < E; ++q) t[I::row(u, q) * N + I::col(u, q)] = v[u][q];
}

template <int N>
static int launch_fourier_mask(float2 *a, const float *mask, int64_t batch, cudaStream_t st) {
    const size_t smem = (size_t)Lay<N>::BUF * sizeof(float2) + TileCfg<N>::TW * sizeof(float2);
    static bool configured = false;
    if (!configured) {
        if (cudaFuncSetAttribute(k_fourier_mask<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
            return record_cuda(cudaGetLastError());
        configured = true;
    }
    constexpr unsigned C = TileCfg<N>::CTAS;
    return launch_clustered(k_fourier_mask<N>, (unsigned)batch * C, FFT_THREADS, C, smem, st, a, mask);
}

}  // namespace phb

using namespace phb;

static inline int grid_for(int64_t total, int threads = 256) {
    int64_t g = (total + threads - 1) / threads;
    if (g > 148 * 64) g = 148 * 64;
    return (int)(g < 1 ? 1 : g);
}

extern "C" {

int phb_cutout_starts(const float *scan, const int64_t *group, int64_t B, double corner_y, double corner_x,
                      double samp_y, double samp_x, int64_t cut_y, int64_t cut_x, int64_t *starts, float *subpx,
                      void *stream) {
    if (!scan || !starts || B < 0 || cut_y < 0 || cut_x < 0) return PHB_ERR_INVALID_ARG;
    if (!(samp_y > 0) || !(samp_x > 0)) return PHB_ERR_INVALID_ARG;
    if (B == 0) return PHB_OK;
    k_cutout_starts<<<(unsigned)((B + 127) / 128), 128, 0, (cudaStream_t)stream>>>(
        scan, group, B, corner_y, corner_x, samp_y, samp_x, cut_y, cut_x, starts, subpx);
    return check_launch();
}

int phb_cutout_get_c64(const void *obj, int64_t S, int64_t H, int64_t W, const int64_t *starts, int64_t B,
                       int64_t cut_y, int64_t cut_x, float fill_re, float fill_im, void *out, void *stream) {
    if (!obj || !starts || !out || S <= 0 || H <= 0 || W <= 0 || B < 0 || cut_y <= 0 || cut_x <= 0)
        return PHB_ERR_INVALID_ARG;
    if (B == 0) return PHB_OK;
    const int64_t total = B * S * cut_y * cut_x;
    k_cutout_get<float2><<<grid_for(total), 256, 0, (cudaStream_t)stream>>>(
        (const float2 *)obj, S, H, W, starts, B, cut_y, cut_x, make_float2(fill_re, fill_im), (float2 *)out);
    return check_launch();
}

int phb_cutout_get_f32(const float *obj, int64_t S, int64_t H, int64_t W, const int64_t *starts, int64_t B,
                       int64_t cut_y, int64_t cut_x, float fill, float *out, void *stream) {
    if (!obj || !starts || !out || S <= 0 || H <= 0 || W <= 0 || B < 0 || cut_y <= 0 || cut_x <= 0)
        return PHB_ERR_INVALID_ARG;
    if (B == 0) return PHB_OK;
    const int64_t total = B * S * cut_y * cut_x;
    k_cutout_get<float><<<grid_for(total), 256, 0, (cudaStream_t)stream>>>(obj, S, H, W, starts, B, cut_y, cut_x,
                                                                            fill, out);
    return check_launch();
}

int phb_cutout_add_c64(void *obj, int64_t S, int64_t H, int64_t W, const int64_t *starts, int64_t B,
                       int64_t cut_y, int64_t cut_x, const void *views, void *stream) {
    if (!obj || !starts || !views || S <= 0 || H <= 0 || W <= 0 || B < 0 || cut_y <= 0 || cut_x <= 0)
        return PHB_ERR_INVALID_ARG;
    if (B == 0) return PHB_OK;
    const int64_t total = B * S * cut_y * cut_x;
    k_cutout_put_c64<0><<<grid_for(total), 256, 0, (cudaStream_t)stream>>>(
        (float2 *)obj, S, H, W, starts, B, cut_y, cut_x, (const float2 *)views);
    return check_launch();
}

int phb_cutout_set_c64(void *obj, int64_t S, int64_t H, int64_t W, const int64_t *starts, int64_t B,
                       int64_t cut_y, int64_t cut_x, const void *views, void *stream) {
    if (!obj || !starts || !views || S <= 0 || H <= 0 || W <= 0 || B < 0 || cut_y <= 0 || cut_x <= 0)
        return PHB_ERR_INVALID_ARG;
    if (B == 0) return PHB_OK;
    const int64_t total = B * S * cut_y * cut_x;
    k_cutout_put_c64<1><<<grid_for(total), 256, 0, (cudaStream_t)stream>>>(
        (float2 *)obj, S, H, W, starts, B, cut_y, cut_x, (const float2 *)views);
    return check_launch();
}

int phb_cutout_add_f32(float *obj, int64_t S, int64_t H, int64_t W, const int64_t *starts, int64_t B,
                       int64_t cut_y, int64_t cut_x, const float *views, void *stream) {
    if (!obj || !starts || !views || S <= 0 || H <= 0 || W <= 0 || B < 0 || cut_y <= 0 || cut_x <= 0)
        return PHB_ERR_INVALID_ARG;
    if (B == 0) return PHB_OK;
    const int64_t total = B * S * cut_y * cut_x;
    k_cutout_add_f32<<<grid_for(total), 256, 0, (cudaStream_t)stream>>>(obj, S, H, W, starts, B, cut_y, cut_x, views);
    return check_launch();
}

int phb_fft2_c64(const void *in, void *out, int64_t batch, int64_t N, int inverse, void *stream) {
    if (!in || !out || batch < 0) return PHB_ERR_INVALID_ARG;
    if (batch == 0) return PHB_OK;
    if (batch > 0x7fffffff) return PHB_ERR_INVALID_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    if (batch > 0x7fffffff / 4) return PHB_ERR_INVALID_ARG;
    if (N == 256) return launch_fft2<256>((const float2 *)in, (float2 *)out, batch, inverse, st);
    if (N == 128) return launch_fft2<128>((const float2 *)in, (float2 *)out, batch, inverse, st);
    if (N == 64) return launch_fft2<64>((const float2 *)in, (float2 *)out, batch, inverse, st);
    return PHB_ERR_UNSUPPORTED;
}

int phb_clamp_amplitude_c64(void *arr, int64_t n, float amplitude, void *stream) {
    if (!arr || n < 0) return PHB_ERR_INVALID_ARG;
    if (n == 0) return PHB_OK;
    k_clamp_amplitude<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>((float2 *)arr, n, amplitude);
    return check_launch();
}

int phb_fourier_mask_c64(void *arr, int64_t batch, int64_t N, const float *mask, void *stream) {
    if (!arr || !mask || batch < 0) return PHB_ERR_INVALID_ARG;
    if (batch == 0) return PHB_OK;
    cudaStream_t st = (cudaStream_t)stream;
    if (N == 256) return launch_fourier_mask<256>((float2 *)arr, mask, batch, st);
    if (N == 128) return launch_fourier_mask<128>((float2 *)arr, mask, batch, st);
    if (N == 64) return launch_fourier_mask<64>((float2 *)arr, mask, batch, st);
    return PHB_ERR_UNSUPPORTED;
}

}  // extern "C"
