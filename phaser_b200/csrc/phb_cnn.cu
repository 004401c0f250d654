// Learned warm start: a small convolutional network that maps a diffraction
// pattern to the object patch under the probe.  It has no counterpart in the
// reference; the iterative solvers refine its stitched prediction.
//
// Layers are 3x3 convolutions (padding 1, stride 1 or 2) on NCHW float32
// activations with bfloat16 weights and float32 accumulation, ReLU, and a
// nearest-neighbour 2x upsampling.  Everything here is off the multislice hot
// path (a few hundred MFLOP per pattern), so the kernels are direct
// shared-memory-tiled convolutions on the FP32 pipe.
#include <cuda_bf16.h>

#include "phb_common.cuh"
#include "phb_runtime.h"

namespace phb {

constexpr int CT = 16;    // output tile side (pixels) of the forward / data-gradient kernels
constexpr int CIB = 8;    // input channels staged per step

// ------------------------------------------------------------------ forward
// out[n][co][y][x] = bias[co] + sum_{ci,ky,kx} w[co][ci][ky][kx] in[n][ci][S y + ky - 1][S x + kx - 1]
template <int COB, int S>
__global__ void __launch_bounds__(256) k_conv_fwd(const float *in, const __nv_bfloat16 *w, const float *bias,
                                                  float *out, int Ci, int Hi, int Wi, int Co, int Ho, int Wo,
                                                  int relu) {
    constexpr int PH = (CT - 1) * S + 3;
    // Row stride of the staged input: a warp reads two tile rows (16 threads each); at
    // stride 1 a row stride of 48 words puts the second half-warp 16 banks after the
    // first, so the two never share a bank.
    constexpr int PW = S == 1 ? 48 : PH;
    __shared__ float patch[CIB][PH][PW];
    // weights [ci][tap][co], read as float4 broadcasts (4 output channels per load)
    __shared__ __align__(16) float ws[CIB][9][COB];
    const int tiles_x = (Wo + CT - 1) / CT;
    const int ty0 = (blockIdx.x / tiles_x) * CT, tx0 = (blockIdx.x % tiles_x) * CT;
    const int co0 = blockIdx.y * COB, n = blockIdx.z;
    const int ty = threadIdx.x / CT, tx = threadIdx.x % CT;
    const int y = ty0 + ty, x = tx0 + tx;
    const int iy0 = ty0 * S - 1, ix0 = tx0 * S - 1;
    float acc[COB];
#pragma unroll
    for (int c = 0; c < COB; ++c) acc[c] = 0.f;
    const float *inn = in + (size_t)n * Ci * Hi * Wi;
    for (int ci0 = 0; ci0 < Ci; ci0 += CIB) {
        for (int e = threadIdx.x; e < CIB * PH * PH; e += blockDim.x) {
            const int c = e / (PH * PH), r = (e / PH) % PH, q = e % PH;
            const int iy = iy0 + r, ix = ix0 + q, ci = ci0 + c;
            patch[c][r][q] = (ci < Ci && iy >= 0 && iy < Hi && ix >= 0 && ix < Wi)
                                 ? inn[((size_t)ci * Hi + iy) * Wi + ix] : 0.f;
        }
        for (int e = threadIdx.x; e < CIB * 9 * COB; e += blockDim.x) {
            const int c = e / (9 * COB), t = (e / COB) % 9, o = e % COB;
            const int ci = ci0 + c, co = co0 + o;
            ws[c][t][o] = (ci < Ci && co < Co) ? __bfloat162float(w[((size_t)co * Ci + ci) * 9 + t]) : 0.f;
        }
        __syncthreads();
#pragma unroll
        for (int c = 0; c < CIB; ++c)
#pragma unroll
            for (int t = 0; t < 9; ++t) {
                const float v = patch[c][ty * S + t / 3][tx * S + t % 3];
                if constexpr (COB % 4 == 0) {
                    const float4 *w4 = reinterpret_cast<const float4 *>(&ws[c][t][0]);
#pragma unroll
                    for (int o = 0; o < COB / 4; ++o) {
                        const float4 q = w4[o];
                        acc[4 * o + 0] = fmaf(v, q.x, acc[4 * o + 0]);
                        acc[4 * o + 1] = fmaf(v, q.y, acc[4 * o + 1]);
                        acc[4 * o + 2] = fmaf(v, q.z, acc[4 * o + 2]);
                        acc[4 * o + 3] = fmaf(v, q.w, acc[4 * o + 3]);
                    }
                } else {
#pragma unroll
                    for (int o = 0; o < COB; ++o) acc[o] = fmaf(v, ws[c][t][o], acc[o]);
                }
            }
        __syncthreads();
    }
    if (y < Ho && x < Wo) {
#pragma unroll
        for (int o = 0; o < COB; ++o) {
            const int co = co0 + o;
            if (co >= Co) break;
            float r = acc[o] + bias[co];
            if (relu) r = fmaxf(r, 0.f);
            out[(((size_t)n * Co + co) * Ho + y) * Wo + x] = r;
        }
    }
}

// --------------------------------------------------------- data gradient
// din[n][ci][Y][X] = sum_{co,ky,kx: S y + ky - 1 = Y, S x + kx - 1 = X} w[co][ci][ky][kx] dout[n][co][y][x]
template <int CIO, int S>
__global__ void __launch_bounds__(256) k_conv_bwd_data(const float *dout, const __nv_bfloat16 *w, float *din,
                                                       int Ci, int Hi, int Wi, int Co, int Ho, int Wo) {
    constexpr int COB2 = 8;
    __shared__ __align__(16) float ws[COB2][9][CIO];   // read as float4 broadcasts
    const int tiles_x = (Wi + CT - 1) / CT;
    const int Y = (blockIdx.x / tiles_x) * CT + threadIdx.x / CT, X = (blockIdx.x % tiles_x) * CT + threadIdx.x % CT;
    const int ci0 = blockIdx.y * CIO, n = blockIdx.z;
    float acc[CIO];
#pragma unroll
    for (int c = 0; c < CIO; ++c) acc[c] = 0.f;
    const float *dn = dout + (size_t)n * Co * Ho * Wo;
    for (int co0 = 0; co0 < Co; co0 += COB2) {
        for (int e = threadIdx.x; e < COB2 * 9 * CIO; e += blockDim.x) {
            const int o = e / (9 * CIO), t = (e / CIO) % 9, c = e % CIO;
            const int co = co0 + o, ci = ci0 + c;
            ws[o][t][c] = (co < Co && ci < Ci) ? __bfloat162float(w[((size_t)co * Ci + ci) * 9 + t]) : 0.f;
        }
        __syncthreads();
        if (Y < Hi && X < Wi) {
#pragma unroll
            for (int t = 0; t < 9; ++t) {
                const int ky = t / 3, kx = t % 3;
                const int sy = Y + 1 - ky, sx = X + 1 - kx;
                if (sy < 0 || sx < 0 || sy % S || sx % S) continue;
                const int yy = sy / S, xx = sx / S;
                if (yy >= Ho || xx >= Wo) continue;
#pragma unroll
                for (int o = 0; o < COB2; ++o) {
                    const int co = co0 + o;
                    if (co >= Co) break;
                    const float g = dn[((size_t)co * Ho + yy) * Wo + xx];
                    if constexpr (CIO % 4 == 0) {
                        const float4 *w4 = reinterpret_cast<const float4 *>(&ws[o][t][0]);
#pragma unroll
                        for (int c = 0; c < CIO / 4; ++c) {
                            const float4 q = w4[c];
                            acc[4 * c + 0] = fmaf(g, q.x, acc[4 * c + 0]);
                            acc[4 * c + 1] = fmaf(g, q.y, acc[4 * c + 1]);
                            acc[4 * c + 2] = fmaf(g, q.z, acc[4 * c + 2]);
                            acc[4 * c + 3] = fmaf(g, q.w, acc[4 * c + 3]);
                        }
                    } else {
#pragma unroll
                        for (int c = 0; c < CIO; ++c) acc[c] = fmaf(g, ws[o][t][c], acc[c]);
                    }
                }
            }
        }
        __syncthreads();
    }
    if (Y < Hi && X < Wi) {
#pragma unroll
        for (int c = 0; c < CIO; ++c) {
            const int ci = ci0 + c;
            if (ci >= Ci) break;
            din[(((size_t)n * Ci + ci) * Hi + Y) * Wi + X] = acc[c];
        }
    }
}

// ------------------------------------------------------- weight gradient
// dw[co][ci][t] += sum_{n,y,x} dout[n][co][y][x] in[n][ci][S y + ky - 1][S x + kx - 1]; db[co] += sum dout
// One CTA per (8 output channels, input channel, batch chunk); block-reduced, one atomic per weight.
template <int S>
__global__ void __launch_bounds__(256) k_conv_bwd_w(const float *in, const float *dout, float *dw, float *db,
                                                    int Nb, int Ci, int Hi, int Wi, int Co, int Ho, int Wo,
                                                    int n_per_block) {
    constexpr int COB2 = 8;
    __shared__ float red[8][COB2 * 9 + COB2];
    const int co0 = blockIdx.x * COB2, ci = blockIdx.y;
    const int n0 = blockIdx.z * n_per_block, n1 = min(Nb, n0 + n_per_block);
    float acc[COB2 * 9 + COB2];
#pragma unroll
    for (int i = 0; i < COB2 * 9 + COB2; ++i) acc[i] = 0.f;
    const int P = Ho * Wo;
    for (int n = n0; n < n1; ++n) {
        const float *inn = in + ((size_t)n * Ci + ci) * Hi * Wi;
        const float *dn = dout + (size_t)n * Co * P;
        for (int p = threadIdx.x; p < P; p += blockDim.x) {
            const int y = p / Wo, x = p % Wo;
            float v[9];
#pragma unroll
            for (int t = 0; t < 9; ++t) {
                const int iy = S * y + t / 3 - 1, ix = S * x + t % 3 - 1;
                v[t] = (iy >= 0 && iy < Hi && ix >= 0 && ix < Wi) ? inn[(size_t)iy * Wi + ix] : 0.f;
            }
#pragma unroll
            for (int o = 0; o < COB2; ++o) {
                const int co = co0 + o;
                const float g = co < Co ? dn[(size_t)co * P + p] : 0.f;
#pragma unroll
                for (int t = 0; t < 9; ++t) acc[o * 9 + t] = fmaf(g, v[t], acc[o * 9 + t]);
                acc[COB2 * 9 + o] += g;
            }
        }
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int i = 0; i < COB2 * 9 + COB2; ++i) {
        float s = acc[i];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) red[wid][i] = s;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < COB2 * 9 + COB2; i += blockDim.x) {
        float s = 0.f;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) s += red[k][i];
        if (i < COB2 * 9) {
            const int o = i / 9, t = i % 9, co = co0 + o;
            if (co < Co) atomicAdd(&dw[((size_t)co * Ci + ci) * 9 + t], s);
        } else if (ci == 0) {
            const int co = co0 + (i - COB2 * 9);
            if (co < Co) atomicAdd(&db[co], s);
        }
    }
}

// ----------------------------------------------------------- elementwise
__global__ void k_relu_bwd(float *g, const float *y, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        if (!(y[i] > 0.f)) g[i] = 0.f;
}

__global__ void k_upsample2(const float *in, float *out, int64_t planes, int H, int W) {
    const int64_t total = planes * 4 * H * W;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t pl = i / (4 * H * W);
        const int r = (int)(i / (2 * W) % (2 * H)), c = (int)(i % (2 * W));
        out[i] = in[(pl * H + r / 2) * W + c / 2];
    }
}

__global__ void k_upsample2_bwd(const float *gout, float *gin, int64_t planes, int H, int W) {
    const int64_t total = planes * H * W;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t pl = i / (H * W);
        const int r = (int)(i / W % H), c = (int)(i % W);
        const float *g = gout + (pl * 2 * H + 2 * r) * (2 * W) + 2 * c;
        gin[i] = g[0] + g[1] + g[2 * W] + g[2 * W + 1];
    }
}

// mean squared error over n values: *loss += sum (p - t)^2 / n, grad = 2 (p - t) / n
__global__ void k_mse(const float *pred, const float *target, float *grad, int64_t n, double *loss) {
    double acc = 0.0;
    const float inv = 1.0f / (float)n;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float d = pred[i] - target[i];
        acc += (double)d * (double)d;
        if (grad) grad[i] = 2.f * d * inv;
    }
    if (loss) warp_atomic_sum(loss, acc / (double)n);
}

__global__ void k_to_bf16(const float *x, __nv_bfloat16 *y, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        y[i] = __float2bfloat16_rn(x[i]);
}

// ------------------------------------------------------- data preparation
// Network input of pattern b: log(1 + max(I, 0)) with the zero frequency moved to
// the centre, binned by `bin` x `bin`, divided by its maximum.  One CTA per pattern.
__global__ void __launch_bounds__(256) k_pattern_features(const float *pat, const int64_t *index, int N, int crop,
                                                          int bin, int flip, float *out) {
    const int b = blockIdx.x, F = crop / bin, c0 = N / 2 - crop / 2;
    const float *p = pat + (size_t)(index ? index[b] : b) * N * N;
    float *o = out + (size_t)b * F * F;
    __shared__ float smax[32];
    float mx = 0.f;
    for (int i = threadIdx.x; i < F * F; i += blockDim.x) {
        const int fy = i / F, fx = i % F;
        float s = 0.f;
        for (int dy = 0; dy < bin; ++dy)
            for (int dx = 0; dx < bin; ++dx) {
                // spatial frequency of this detector pixel (zero at the crop's centre), mirrored
                // through zero when flip is set; stored patterns hold zero frequency at [0, 0]
                int ky = c0 + fy * bin + dy - N / 2, kx = c0 + fx * bin + dx - N / 2;
                if (flip) ky = -ky, kx = -kx;
                s += fmaxf(p[((ky + N) % N) * N + (kx + N) % N], 0.f);
            }
        const float v = log1pf(s);
        o[i] = v;
        mx = fmaxf(mx, v);
    }
    mx = block_max_float<256>(mx, smax);
    const float inv = mx > 0.f ? 1.f / mx : 0.f;
    for (int i = threadIdx.x; i < F * F; i += blockDim.x) o[i] *= inv;
}

// Training target of position b: the centred P x P patch of the projected
// object under the cutout (same exact cutout start as the solvers), as
// (Re - 1, Im) planes.  One CTA per position.
__global__ void __launch_bounds__(256) k_patch_targets(const float2 *proj, int64_t H, int64_t W, const float *scan,
                                                       const int64_t *index, double cy, double cx, double sy,
                                                       double sx, int N, int P, float *out) {
    const int b = blockIdx.x;
    const int64_t pos = index ? index[b] : b;
    const CutoutIndex ci = cutout_index(scan, pos, cy, cx, sy, sx, N, N);
    const int off = (N - P) / 2;
    float *o = out + (size_t)b * 2 * P * P;
    for (int i = threadIdx.x; i < P * P; i += blockDim.x) {
        const int64_t y = ci.y0 + off + i / P, x = ci.x0 + off + i % P;
        const float2 v = (y >= 0 && y < H && x >= 0 && x < W) ? proj[y * W + x] : make_float2(1.f, 0.f);
        o[i] = v.x - 1.f;
        o[P * P + i] = v.y;
    }
}

// Stitch predicted patches (B, 2, P, P) = (Re - 1, Im) into sum / weight grids, each
// patch pixel weighted by window[P * P] (1 when window is NULL).
__global__ void __launch_bounds__(256) k_stitch(const float *pred, const float *scan, const int64_t *index,
                                                double cy, double cx, double sy, double sx, int N, int P,
                                                const float *window, float2 *acc, float *wgt, int64_t H,
                                                int64_t W) {
    const int b = blockIdx.x;
    const int64_t pos = index ? index[b] : b;
    const CutoutIndex ci = cutout_index(scan, pos, cy, cx, sy, sx, N, N);
    const int off = (N - P) / 2;
    const float *p = pred + (size_t)b * 2 * P * P;
    for (int i = threadIdx.x; i < P * P; i += blockDim.x) {
        const int64_t y = ci.y0 + off + i / P, x = ci.x0 + off + i % P;
        if (y < 0 || y >= H || x < 0 || x >= W) continue;
        const float w = window ? window[i] : 1.f;
        atomic_add_c(acc + y * W + x, make_float2(w * (p[i] + 1.f), w * p[P * P + i]));
        atomicAdd(wgt + y * W + x, w);
    }
}

// obj = acc / wgt where covered, 1 elsewhere
__global__ void k_stitch_finish(const float2 *acc, const float *wgt, float2 *obj, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        obj[i] = wgt[i] > 0.f ? cscale(acc[i], 1.f / wgt[i]) : make_float2(1.f, 0.f);
}

// product of the object's slices (the projected transmission)
__global__ void k_project(const float2 *obj, int64_t S, int64_t HW, float2 *out) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < HW; i += (int64_t)gridDim.x * blockDim.x) {
        float2 v = obj[i];
        for (int64_t s = 1; s < S; ++s) v = cmul(v, obj[s * HW + i]);
        out[i] = v;
    }
}

}  // namespace phb

using namespace phb;

static inline unsigned ew_grid(int64_t n) {
    int64_t g = (n + 255) / 256;
    if (g > 148 * 16) g = 148 * 16;
    return (unsigned)(g < 1 ? 1 : g);
}

template <int COB, int S>
static void launch_fwd(const float *in, const __nv_bfloat16 *w, const float *b, float *out, int Nb, int Ci, int Hi,
                       int Wi, int Co, int Ho, int Wo, int relu, cudaStream_t st) {
    dim3 grid((unsigned)(((Ho + CT - 1) / CT) * ((Wo + CT - 1) / CT)), (unsigned)((Co + COB - 1) / COB), (unsigned)Nb);
    k_conv_fwd<COB, S><<<grid, 256, 0, st>>>(in, w, b, out, Ci, Hi, Wi, Co, Ho, Wo, relu);
}

template <int CIO, int S>
static void launch_bwd_data(const float *dout, const __nv_bfloat16 *w, float *din, int Nb, int Ci, int Hi, int Wi,
                            int Co, int Ho, int Wo, cudaStream_t st) {
    dim3 grid((unsigned)(((Hi + CT - 1) / CT) * ((Wi + CT - 1) / CT)), (unsigned)((Ci + CIO - 1) / CIO), (unsigned)Nb);
    k_conv_bwd_data<CIO, S><<<grid, 256, 0, st>>>(dout, w, din, Ci, Hi, Wi, Co, Ho, Wo);
}

extern "C" {

int phb_conv3x3_fwd(const float *in, const void *w_bf16, const float *bias, float *out, int32_t Nb, int32_t Ci,
                    int32_t Hi, int32_t Wi, int32_t Co, int32_t stride, int32_t relu, void *stream) {
    if (!in || !w_bf16 || !bias || !out || Nb < 1 || Ci < 1 || Co < 1 || Hi < 1 || Wi < 1) return PHB_ERR_INVALID_ARG;
    if (stride != 1 && stride != 2) return PHB_ERR_UNSUPPORTED;
    if (Nb > 65535 || (stride == 2 && ((Hi | Wi) & 1))) return PHB_ERR_UNSUPPORTED;
    const int Ho = Hi / stride, Wo = Wi / stride;
    const __nv_bfloat16 *w = (const __nv_bfloat16 *)w_bf16;
    cudaStream_t st = (cudaStream_t)stream;
    if (Co <= 2) {
        if (stride == 1) launch_fwd<2, 1>(in, w, bias, out, Nb, Ci, Hi, Wi, Co, Ho, Wo, relu, st);
        else launch_fwd<2, 2>(in, w, bias, out, Nb, Ci, Hi, Wi, Co, Ho, Wo, relu, st);
    } else {
        if (stride == 1) launch_fwd<16, 1>(in, w, bias, out, Nb, Ci, Hi, Wi, Co, Ho, Wo, relu, st);
        else launch_fwd<16, 2>(in, w, bias, out, Nb, Ci, Hi, Wi, Co, Ho, Wo, relu, st);
    }
    return check_launch();
}

int phb_conv3x3_bwd_data(const float *dout, const void *w_bf16, float *din, int32_t Nb, int32_t Ci, int32_t Hi,
                         int32_t Wi, int32_t Co, int32_t stride, void *stream) {
    if (!dout || !w_bf16 || !din || Nb < 1 || Ci < 1 || Co < 1 || Hi < 1 || Wi < 1) return PHB_ERR_INVALID_ARG;
    if (stride != 1 && stride != 2) return PHB_ERR_UNSUPPORTED;
    if (Nb > 65535 || (stride == 2 && ((Hi | Wi) & 1))) return PHB_ERR_UNSUPPORTED;
    const int Ho = Hi / stride, Wo = Wi / stride;
    const __nv_bfloat16 *w = (const __nv_bfloat16 *)w_bf16;
    cudaStream_t st = (cudaStream_t)stream;
    if (stride == 1) launch_bwd_data<16, 1>(dout, w, din, Nb, Ci, Hi, Wi, Co, Ho, Wo, st);
    else launch_bwd_data<16, 2>(dout, w, din, Nb, Ci, Hi, Wi, Co, Ho, Wo, st);
    return check_launch();
}

int phb_conv3x3_bwd_weight(const float *in, const float *dout, float *dw, float *db, int32_t Nb, int32_t Ci,
                           int32_t Hi, int32_t Wi, int32_t Co, int32_t stride, void *stream) {
    if (!in || !dout || !dw || !db || Nb < 1 || Ci < 1 || Co < 1 || Hi < 1 || Wi < 1) return PHB_ERR_INVALID_ARG;
    if (stride != 1 && stride != 2) return PHB_ERR_UNSUPPORTED;
    if (Ci > 65535 || (stride == 2 && ((Hi | Wi) & 1))) return PHB_ERR_UNSUPPORTED;
    const int Ho = Hi / stride, Wo = Wi / stride;
    const int per = 8;
    dim3 grid((unsigned)((Co + 7) / 8), (unsigned)Ci, (unsigned)((Nb + per - 1) / per));
    cudaStream_t st = (cudaStream_t)stream;
    if (stride == 1) k_conv_bwd_w<1><<<grid, 256, 0, st>>>(in, dout, dw, db, Nb, Ci, Hi, Wi, Co, Ho, Wo, per);
    else k_conv_bwd_w<2><<<grid, 256, 0, st>>>(in, dout, dw, db, Nb, Ci, Hi, Wi, Co, Ho, Wo, per);
    return check_launch();
}

int phb_relu_bwd(float *grad, const float *y, int64_t n, void *stream) {
    if (!grad || !y || n < 0) return PHB_ERR_INVALID_ARG;
    if (n == 0) return PHB_OK;
    k_relu_bwd<<<ew_grid(n), 256, 0, (cudaStream_t)stream>>>(grad, y, n);
    return check_launch();
}

int phb_upsample2(const float *in, float *out, int64_t planes, int32_t H, int32_t W, void *stream) {
    if (!in || !out || planes < 1 || H < 1 || W < 1) return PHB_ERR_INVALID_ARG;
    k_upsample2<<<ew_grid(planes * 4 * H * W), 256, 0, (cudaStream_t)stream>>>(in, out, planes, H, W);
    return check_launch();
}

int phb_upsample2_bwd(const float *gout, float *gin, int64_t planes, int32_t H, int32_t W, void *stream) {
    if (!gout || !gin || planes < 1 || H < 1 || W < 1) return PHB_ERR_INVALID_ARG;
    k_upsample2_bwd<<<ew_grid(planes * H * W), 256, 0, (cudaStream_t)stream>>>(gout, gin, planes, H, W);
    return check_launch();
}

int phb_mse(const float *pred, const float *target, float *grad, int64_t n, double *loss, void *stream) {
    if (!pred || !target || n < 1 || (!grad && !loss)) return PHB_ERR_INVALID_ARG;
    k_mse<<<ew_grid(n), 256, 0, (cudaStream_t)stream>>>(pred, target, grad, n, loss);
    return check_launch();
}

int phb_to_bf16(const float *x, void *y, int64_t n, void *stream) {
    if (!x || !y || n < 0) return PHB_ERR_INVALID_ARG;
    if (n == 0) return PHB_OK;
    k_to_bf16<<<ew_grid(n), 256, 0, (cudaStream_t)stream>>>(x, (__nv_bfloat16 *)y, n);
    return check_launch();
}

int phb_pattern_features(const float *patterns, const int64_t *index, int32_t B, int32_t N, int32_t crop,
                         int32_t bin, int32_t flip, float *out, void *stream) {
    if (!patterns || !out || B < 1 || N < 2 || N % 2 || crop < 2 || crop > N || crop % 2 || bin < 1 || crop % bin)
        return PHB_ERR_INVALID_ARG;
    k_pattern_features<<<B, 256, 0, (cudaStream_t)stream>>>(patterns, index, N, crop, bin, flip ? 1 : 0, out);
    return check_launch();
}

int phb_patch_targets(const void *proj, int64_t H, int64_t W, const float *scan, const int64_t *index, int32_t B,
                      double corner_y, double corner_x, double samp_y, double samp_x, int32_t N, int32_t P,
                      float *out, void *stream) {
    if (!proj || !scan || !out || B < 1 || P < 1 || P > N || H < 1 || W < 1) return PHB_ERR_INVALID_ARG;
    k_patch_targets<<<B, 256, 0, (cudaStream_t)stream>>>((const float2 *)proj, H, W, scan, index, corner_y, corner_x,
                                                         samp_y, samp_x, N, P, out);
    return check_launch();
}

int phb_stitch_patches(const float *pred, const float *scan, const int64_t *index, int32_t B, double corner_y,
                       double corner_x, double samp_y, double samp_x, int32_t N, int32_t P, const float *window,
                       void *acc, float *wgt, int64_t H, int64_t W, void *stream) {
    if (!pred || !scan || !acc || !wgt || B < 1 || P < 1 || P > N || H < 1 || W < 1) return PHB_ERR_INVALID_ARG;
    k_stitch<<<B, 256, 0, (cudaStream_t)stream>>>(pred, scan, index, corner_y, corner_x, samp_y, samp_x, N, P,
                                                  window, (float2 *)acc, wgt, H, W);
    return check_launch();
}

int phb_stitch_finish(const void *acc, const float *wgt, void *obj, int64_t n, void *stream) {
    if (!acc || !wgt || !obj || n < 1) return PHB_ERR_INVALID_ARG;
    k_stitch_finish<<<ew_grid(n), 256, 0, (cudaStream_t)stream>>>((const float2 *)acc, wgt, (float2 *)obj, n);
    return check_launch();
}

int phb_project_slices(const void *obj, int64_t S, int64_t HW, void *out, void *stream) {
    if (!obj || !out || S < 1 || HW < 1) return PHB_ERR_INVALID_ARG;
    k_project<<<ew_grid(HW), 256, 0, (cudaStream_t)stream>>>((const float2 *)obj, S, HW, (float2 *)out);
    return check_launch();
}

}  // extern "C"
