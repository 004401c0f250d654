// Object constraints and gradient-engine cost regularisers (sm_100a).
//
// Constraints of phaser/engines/common/regularizers.py applied between
// mini-batches or iterations:
//   layers             RegularizeLayers  (regularizers.py:86-132): log-domain
//                      Gaussian smoothing along z, 'nearest' edges, blended
//   obj_low_pass       ObjLowPass        (regularizers.py:135-161)
//   obj_gaussian       ObjGaussian       (regularizers.py:164-192)
//                      both O <- ifft2(filter * fft2(O)) on the whole object
//   remove_phase_ramp  RemovePhaseRamp   (regularizers.py:67-83, utils/image.py:30-55)
// and the cost regularisers of the gradient engine (regularizers.py:195-385),
// whose values join the group loss and whose gradients join the object gradient.
#include "phb_common.cuh"
#include "phb_runtime.h"

namespace phb {

// ------------------------------------------------------------------ layers
// One thread per object pixel (h, w): the S complex logs are kept in shared
// memory, smoothed along z with the normalised taps, exponentiated and blended:
// O <- weight * exp(conv(log O)) + (1 - weight) * O.  scipy.ndimage.convolve1d
// with mode 'nearest' clamps the index at both ends; the taps are symmetric.
__global__ void k_layers(float2 *obj, int64_t S, int64_t HW, const float *taps, int n, float weight) {
    extern __shared__ float2 lg[];   // [S][blockDim.x]
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool ok = p < HW;
    const int r = (n - 1) / 2;
    if (ok) {
        for (int64_t s = 0; s < S; ++s) {
            const float2 o = obj[s * HW + p];
            lg[s * blockDim.x + threadIdx.x] = make_float2(logf(hypotf(o.x, o.y)), atan2f(o.y, o.x));
        }
        for (int64_t s = 0; s < S; ++s) {
            float2 acc = make_float2(0.f, 0.f);
            for (int j = 0; j < n; ++j) {
                int64_t q = s + r - j;
                q = q < 0 ? 0 : (q >= S ? S - 1 : q);
                const float2 l = lg[q * blockDim.x + threadIdx.x];
                acc.x = fmaf(taps[j], l.x, acc.x);
                acc.y = fmaf(taps[j], l.y, acc.y);
            }
            float sn, cs;
            sincosf(acc.y, &sn, &cs);
            const float m = expf(acc.x);
            float2 *dst = obj + s * HW + p;
            const float2 o = *dst;
            *dst = make_float2(weight * m * cs + (1.f - weight) * o.x, weight * m * sn + (1.f - weight) * o.y);
        }
    }
}

// ------------------------------------------------------- DFT along the last axis
// out[b][k][r] = scale * sum_c in[b][r][c] * exp(sign 2 pi i c k / C) (* filt[k][r])
// A 64 x 64 output tile per CTA, 16-wide chunks of c staged in shared memory with
// their twiddles (exact integer phase (c k) mod C, sincospi in float64).  Two
// passes give a 2D DFT of arbitrary size in natural order; the centring shifts of
// phaser's fft2/ifft2 cancel in ifft2(filter * fft2(x)).
constexpr int DT = 64, DC = 16;

__global__ void __launch_bounds__(256) k_dft_t(const float2 *in, float2 *out, int64_t R, int64_t C, int sign,
                                               float scale, const float *filt) {
    __shared__ float2 As[DC][DT];
    __shared__ float2 Ts[DC][DT];
    const int64_t b = blockIdx.z;
    const int64_t r0 = (int64_t)blockIdx.y * DT, k0 = (int64_t)blockIdx.x * DT;
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const float2 *src = in + b * R * C;
    float2 acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = make_float2(0.f, 0.f);
    for (int64_t c0 = 0; c0 < C; c0 += DC) {
        for (int e = threadIdx.x; e < DC * DT; e += blockDim.x) {
            const int cc = e % DC, rr = e / DC;     // 16 consecutive c of one row per 16 threads
            const int64_t r = r0 + rr, c = c0 + cc;
            As[cc][rr] = (r < R && c < C) ? src[r * C + c] : make_float2(0.f, 0.f);
            const int kk = e % DT, cc2 = e / DT;
            const int64_t k = k0 + kk, c2 = c0 + cc2;
            float2 tw = make_float2(0.f, 0.f);
            if (k < C && c2 < C) {
                const int64_t m = (c2 * k) % C;
                double sv, cv;
                sincospi(2.0 * (double)m / (double)C, &sv, &cv);
                tw = make_float2((float)cv, (float)(sign * sv));
            }
            Ts[cc2][kk] = tw;
        }
        __syncthreads();
#pragma unroll 4
        for (int c = 0; c < DC; ++c) {
            float2 a[4], t[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) a[j] = As[c][tx + 16 * j];
#pragma unroll
            for (int i = 0; i < 4; ++i) t[i] = Ts[c][ty + 16 * i];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    acc[i][j].x = fmaf(a[j].x, t[i].x, fmaf(-a[j].y, t[i].y, acc[i][j].x));
                    acc[i][j].y = fmaf(a[j].x, t[i].y, fmaf(a[j].y, t[i].x, acc[i][j].y));
                }
        }
        __syncthreads();
    }
    float2 *dst = out + b * R * C;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int64_t k = k0 + ty + 16 * i;
        if (k >= C) continue;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int64_t r = r0 + tx + 16 * j;
            if (r >= R) continue;
            float s = scale;
            if (filt) s *= filt[k * R + r];
            dst[k * R + r] = cscale(acc[i][j], s);
        }
    }
}

// --------------------------------------------------------- linear phase ramp
// Least-squares plane phi ~ p0 + p1 x + p2 y over a rectangular region, per
// slice (utils/image.py:30-55 with the region mask of object.py:380-384), then
// O <- |O| exp(i (phi - plane)).  Sums in float64.
__global__ void k_ramp_sums(const float2 *obj, int64_t H, int64_t W, int64_t y0, int64_t y1, int64_t x0, int64_t x1,
                            double *sums /* [S][3] */) {
    const int64_t s = blockIdx.y;
    const int64_t nx = x1 - x0, n = (y1 - y0) * nx;
    double a = 0.0, bx = 0.0, by = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t y = y0 + i / nx, x = x0 + i % nx;
        const float2 o = obj[(s * H + y) * W + x];
        const double ph = (double)atan2f(o.y, o.x);
        a += ph;
        bx += ph * (double)x;
        by += ph * (double)y;
    }
    warp_atomic_sum(&sums[3 * s + 0], a);
    warp_atomic_sum(&sums[3 * s + 1], bx);
    warp_atomic_sum(&sums[3 * s + 2], by);
}

__global__ void k_ramp_apply(float2 *obj, int64_t H, int64_t W, int64_t y0, int64_t y1, int64_t x0, int64_t x1,
                             const double *sums) {
    const int64_t s = blockIdx.y;
    // normal equations of the rectangle: moments of x and y in closed form
    const double n = (double)((y1 - y0) * (x1 - x0));
    const double nx = (double)(x1 - x0), ny = (double)(y1 - y0);
    auto m1 = [](double lo, double hi) { return (hi - 1.0 + lo) * (hi - lo) / 2.0; };   // sum of lo..hi-1
    auto m2 = [](double lo, double hi) {   // sum of squares of lo..hi-1
        auto f = [](double k) { return k * (k + 1.0) * (2.0 * k + 1.0) / 6.0; };
        return f(hi - 1.0) - f(lo - 1.0);
    };
    const double Sx = ny * m1((double)x0, (double)x1), Sy = nx * m1((double)y0, (double)y1);
    const double Sxx = ny * m2((double)x0, (double)x1), Syy = nx * m2((double)y0, (double)y1);
    const double Sxy = m1((double)x0, (double)x1) * m1((double)y0, (double)y1);
    const double b0 = sums[3 * s], b1 = sums[3 * s + 1], b2 = sums[3 * s + 2];
    // solve [[n Sx Sy][Sx Sxx Sxy][Sy Sxy Syy]] p = b by Cramer's rule
    const double A00 = n, A01 = Sx, A02 = Sy, A11 = Sxx, A12 = Sxy, A22 = Syy;
    const double c00 = A11 * A22 - A12 * A12, c01 = A02 * A12 - A01 * A22, c02 = A01 * A12 - A02 * A11;
    const double det = A00 * c00 + A01 * c01 + A02 * c02;
    const double c11 = A00 * A22 - A02 * A02, c12 = A01 * A02 - A00 * A12, c22 = A00 * A11 - A01 * A01;
    const double p0 = (c00 * b0 + c01 * b1 + c02 * b2) / det;
    const double p1 = (c01 * b0 + c11 * b1 + c12 * b2) / det;
    const double p2 = (c02 * b0 + c12 * b1 + c22 * b2) / det;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < H * W; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t y = i / W, x = i % W;
        float2 *o = obj + s * H * W + i;
        const float2 v = *o;
        const float ph = (float)((double)atan2f(v.y, v.x) - (p0 + p1 * (double)x + p2 * (double)y));
        const float amp = hypotf(v.x, v.y);
        float sn, cs;
        sincosf(ph, &sn, &cs);
        *o = make_float2(amp * cs, amp * sn);
    }
}

// ------------------------------------------------------- cost regularisers
// Values and gradients (g = dL/dRe + i dL/dIm) of the object cost terms of the
// gradient engine, each scaled by cost * (B / n_pos) as in regularizers.py.
__global__ void k_obj_reg(const float2 *obj, int64_t S, int64_t H, int64_t W, const phb_obj_reg r, float2 *grad,
                          double *loss) {
    const int64_t total = S * H * W, HW = H * W;
    double acc = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t s = i / HW, yx = i % HW, y = yx / W, x = yx % W;
        const float2 o = obj[i];
        float2 g = make_float2(0.f, 0.f);
        double c = 0.0;
        const float2 d1 = make_float2(o.x - 1.f, o.y);
        if (r.l1 != 0.f) {   // sum |O - 1|
            const float m = hypotf(d1.x, d1.y);
            c += (double)r.l1 * m;
            if (m > 0.f) g = cadd(g, cscale(d1, r.l1 / m));
        }
        if (r.l2 != 0.f) {   // sum |O - 1|^2
            c += (double)r.l2 * cabs2(d1);
            g = cadd(g, cscale(d1, 2.f * r.l2));
        }
        if (r.phase_l1 != 0.f) {   // sum |angle(O)|
            const float ph = atan2f(o.y, o.x), m2 = cabs2(o);
            c += (double)r.phase_l1 * fabsf(ph);
            if (m2 > 0.f && ph != 0.f) {
                const float sg = ph > 0.f ? r.phase_l1 : -r.phase_l1;
                g = cadd(g, make_float2(-o.y * sg / m2, o.x * sg / m2));
            }
        }
        if (r.tikh != 0.f) {   // sum |diff_x|^2 + |diff_y|^2 (numpy.diff: no wrap)
            if (x + 1 < W) {
                const float2 d = csub(obj[i + 1], o);
                c += (double)r.tikh * cabs2(d);
                g = csub(g, cscale(d, 2.f * r.tikh));
            }
            if (x > 0) g = cadd(g, cscale(csub(o, obj[i - 1]), 2.f * r.tikh));
            if (y + 1 < H) {
                const float2 d = csub(obj[i + W], o);
                c += (double)r.tikh * cabs2(d);
                g = csub(g, cscale(d, 2.f * r.tikh));
            }
            if (y > 0) g = cadd(g, cscale(csub(o, obj[i - W]), 2.f * r.tikh));
        }
        if (r.tv != 0.f) {   // sum sqrt(|g_y|^2 + |g_x|^2 + eps), forward differences, zero at the far edge
            auto term = [&](int64_t j, int64_t yy, int64_t xx, float2 *gy, float2 *gx) {
                const float2 v = obj[j];
                *gy = (yy + 1 < H) ? csub(obj[j + W], v) : make_float2(0.f, 0.f);
                *gx = (xx + 1 < W) ? csub(obj[j + 1], v) : make_float2(0.f, 0.f);
                return sqrtf(cabs2(*gy) + cabs2(*gx) + r.tv_eps);
            };
            float2 gy, gx;
            const float t0 = term(i, y, x, &gy, &gx);
            c += (double)r.tv * t0;
            g = csub(g, cscale(cadd(gy, gx), r.tv / t0));
            if (y > 0) {
                const float t1 = term(i - W, y - 1, x, &gy, &gx);
                g = cadd(g, cscale(gy, r.tv / t1));
            }
            if (x > 0) {
                const float t2 = term(i - 1, y, x - 1, &gy, &gx);
                g = cadd(g, cscale(gx, r.tv / t2));
            }
        }
        if (S > 1 && (r.layers_tikh != 0.f || r.layers_tv != 0.f)) {   // differences along z
            if (s + 1 < S) {
                const float2 d = csub(obj[i + HW], o);
                const float m2 = cabs2(d), m = sqrtf(m2);
                c += (double)r.layers_tikh * m2 + (double)r.layers_tv * m;
                g = csub(g, cscale(d, 2.f * r.layers_tikh));
                if (r.layers_tv != 0.f && m > 0.f) g = csub(g, cscale(d, r.layers_tv / m));
            }
            if (s > 0) {
                const float2 d = csub(o, obj[i - HW]);
                const float m = sqrtf(cabs2(d));
                g = cadd(g, cscale(d, 2.f * r.layers_tikh));
                if (r.layers_tv != 0.f && m > 0.f) g = cadd(g, cscale(d, r.layers_tv / m));
            }
        }
        acc += c;
        if (grad) grad[i] = cadd(grad[i], cscale(g, r.scale));
    }
    if (loss) warp_atomic_sum(loss, acc * (double)r.scale);
}

// ------------------------------------------- Fourier-space cost regularisers
// probe costs on R = fft2(P) (M, N, N), natural order; the recip terms act on
// fftshift(R).  Writes dL/dR (g convention) to gR and adds the value to *loss.
__global__ void k_probe_reg(const float2 *R, int64_t M, int N, const phb_probe_reg r, float2 *gR, double *loss) {
    const int64_t NN = (int64_t)N * N, total = M * NN;
    const int h = N / 2;
    double acc = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t m = i / NN;
        const int y = (int)(i % NN / N), x = (int)(i % N);
        const float2 *Rm = R + m * NN;
        float2 g = make_float2(0.f, 0.f);
        double c = 0.0;
        if (r.phase_tikh != 0.f) {   // sum of squared differences of angle(R), no unwrapping
            auto th = [&](int yy, int xx) { const float2 v = Rm[yy * N + xx]; return atan2f(v.y, v.x); };
            const float t0 = th(y, x);
            float d = 0.f;   // dL/dtheta at (y, x)
            if (x + 1 < N) { const float e = th(y, x + 1) - t0; c += (double)e * e; d -= 2.f * e; }
            if (x > 0) d += 2.f * (t0 - th(y, x - 1));
            if (y + 1 < N) { const float e = th(y + 1, x) - t0; c += (double)e * e; d -= 2.f * e; }
            if (y > 0) d += 2.f * (t0 - th(y - 1, x));
            c *= r.phase_tikh;
            const float2 v = Rm[y * N + x];
            const float m2 = cabs2(v);
            if (m2 > 0.f) g = cadd(g, cscale(make_float2(-v.y, v.x), r.phase_tikh * d / m2));   // d * i R / |R|^2
        }
        if (r.recip_tikh != 0.f || r.recip_tv != 0.f) {
            // shifted coordinates: Rs(ys, xs) = R((ys + h) % N, (xs + h) % N); this element is Rs(ys, xs)
            const int ys = (y + h) % N, xs = (x + h) % N;
            auto rs = [&](int yy, int xx) { return Rm[((yy + h) % N) * N + (xx + h) % N]; };
            const float2 v = Rm[y * N + x];
            if (r.recip_tikh != 0.f) {
                if (xs + 1 < N) { const float2 e = csub(rs(ys, xs + 1), v); c += (double)r.recip_tikh * cabs2(e);
                                  g = csub(g, cscale(e, 2.f * r.recip_tikh)); }
                if (xs > 0) g = cadd(g, cscale(csub(v, rs(ys, xs - 1)), 2.f * r.recip_tikh));
                if (ys + 1 < N) { const float2 e = csub(rs(ys + 1, xs), v); c += (double)r.recip_tikh * cabs2(e);
                                  g = csub(g, cscale(e, 2.f * r.recip_tikh)); }
                if (ys > 0) g = cadd(g, cscale(csub(v, rs(ys - 1, xs)), 2.f * r.recip_tikh));
            }
            if (r.recip_tv != 0.f) {
                auto term = [&](int yy, int xx, float2 *gy, float2 *gx) {
                    const float2 w = rs(yy, xx);
                    *gy = (yy + 1 < N) ? csub(rs(yy + 1, xx), w) : make_float2(0.f, 0.f);
                    *gx = (xx + 1 < N) ? csub(rs(yy, xx + 1), w) : make_float2(0.f, 0.f);
                    return sqrtf(cabs2(*gy) + cabs2(*gx) + r.tv_eps);
                };
                float2 gy, gx;
                const float t0 = term(ys, xs, &gy, &gx);
                c += (double)r.recip_tv * t0;
                g = csub(g, cscale(cadd(gy, gx), r.recip_tv / t0));
                if (ys > 0) { const float t1 = term(ys - 1, xs, &gy, &gx); g = cadd(g, cscale(gy, r.recip_tv / t1)); }
                if (xs > 0) { const float t2 = term(ys, xs - 1, &gy, &gx); g = cadd(g, cscale(gx, r.recip_tv / t2)); }
            }
        }
        acc += c;
        if (gR) gR[i] = g;
    }
    if (loss) warp_atomic_sum(loss, acc);
}

// U = Z / |Z| (0 where Z = 0); *loss += scale * sum |Z|
__global__ void k_unit_phase(float2 *Z, int64_t n, float scale, double *loss) {
    double acc = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float2 z = Z[i];
        const float m = hypotf(z.x, z.y);
        acc += m;
        Z[i] = m > 0.f ? cscale(z, 1.f / m) : make_float2(0.f, 0.f);
    }
    if (loss) warp_atomic_sum(loss, acc * (double)scale);
}

// grad[s] += scale * gP * conj(prod_{t != s} O_t), prefix products kept in `pre` (S, HW)
__global__ void k_recip_grad(const float2 *obj, int64_t S, int64_t HW, const float2 *gP, float scale, float2 *pre,
                             float2 *grad) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < HW; i += (int64_t)gridDim.x * blockDim.x) {
        float2 p = make_float2(1.f, 0.f);
        for (int64_t s = 0; s < S; ++s) {
            pre[s * HW + i] = p;
            p = cmul(p, obj[s * HW + i]);
        }
        float2 suf = make_float2(1.f, 0.f);
        const float2 g = cscale(gP[i], scale);
        for (int64_t s = S - 1; s >= 0; --s) {
            const float2 others = cmul(pre[s * HW + i], suf);
            grad[s * HW + i] = cadd(grad[s * HW + i], cmulc(g, others));
            suf = cmul(suf, obj[s * HW + i]);
        }
    }
}

// ------------------------------------------------ per-position value smoothing
// UnstructuredGaussian (regularizers.py:430-497): object pixel (r, c) at
// corner + (r, c) * sampling takes the (2-component) value of its nearest scan
// position (brute force; the lowest index wins an exact tie), packed as a complex.
__global__ void __launch_bounds__(256) k_nearest_fill(const float *scan, int64_t n, const float *vals, int64_t H,
                                                      int64_t W, double cy, double cx, double sy, double sx,
                                                      float2 *img) {
    __shared__ float2 sp[1024];
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool ok = i < H * W;
    const double py = cy + (double)(i / W) * sy, px = cx + (double)(i % W) * sx;
    double best = 1e300;
    int64_t arg = 0;
    for (int64_t p0 = 0; p0 < n; p0 += 1024) {
        const int64_t cnt = n - p0 < 1024 ? n - p0 : 1024;
        __syncthreads();
        for (int64_t k = threadIdx.x; k < cnt; k += blockDim.x)
            sp[k] = make_float2(scan[2 * (p0 + k)], scan[2 * (p0 + k) + 1]);
        __syncthreads();
        if (ok)
            for (int64_t k = 0; k < cnt; ++k) {
                const double dy = (double)sp[k].x - py, dx = (double)sp[k].y - px;
                const double d = dy * dy + dx * dx;
                if (d < best) { best = d; arg = p0 + k; }
            }
    }
    if (ok) img[i] = make_float2(vals[2 * arg], vals[2 * arg + 1]);
}

// vals[p] = weight * img[round((pos - corner) / sampling)] + (1 - weight) * vals[p]
__global__ void k_sample_blend(const float2 *img, const float *scan, int64_t n, int64_t H, int64_t W, double cy,
                               double cx, double sy, double sx, float weight, float *vals) {
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x) {
        int64_t r = (int64_t)rint(((double)scan[2 * p] - cy) / sy), c = (int64_t)rint(((double)scan[2 * p + 1] - cx) / sx);
        r = r < 0 ? 0 : (r >= H ? H - 1 : r);
        c = c < 0 ? 0 : (c >= W ? W - 1 : c);
        const float2 b = img[r * W + c];
        vals[2 * p] = weight * b.x + (1.f - weight) * vals[2 * p];
        vals[2 * p + 1] = weight * b.y + (1.f - weight) * vals[2 * p + 1];
    }
}

__global__ void k_add_c(float2 *dst, const float2 *src, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        dst[i] = cadd(dst[i], src[i]);
}

}  // namespace phb

using namespace phb;

static inline unsigned flat_grid(int64_t n, int per = 256) {
    int64_t g = (n + per - 1) / per;
    if (g > 148 * 16) g = 148 * 16;
    return (unsigned)(g < 1 ? 1 : g);
}

extern "C" {

int phb_regularize_layers_c64(void *obj, int64_t S, int64_t H, int64_t W, const float *taps, int32_t n_taps,
                              float weight, void *stream) {
    if (!obj || !taps || S < 1 || H < 1 || W < 1 || n_taps < 1 || (n_taps & 1) == 0) return PHB_ERR_INVALID_ARG;
    if (S > 96) return PHB_ERR_UNSUPPORTED;   // S logs per thread in shared memory (64 threads x 96 x 8 B)
    const int threads = 64;
    const int64_t HW = H * W;
    const size_t smem = (size_t)S * threads * sizeof(float2);
    k_layers<<<(unsigned)((HW + threads - 1) / threads), threads, smem, (cudaStream_t)stream>>>(
        (float2 *)obj, S, HW, taps, n_taps, weight);
    return check_launch();
}

size_t phb_object_filter_scratch_bytes(int64_t S, int64_t H, int64_t W) {
    return (S < 1 || H < 1 || W < 1) ? 0 : (size_t)(S * H * W) * sizeof(float2);
}

int phb_object_filter_c64(void *obj, int64_t S, int64_t H, int64_t W, const float *filter, void *scratch,
                          void *stream) {
    if (!obj || !filter || !scratch || S < 1 || H < 1 || W < 1) return PHB_ERR_INVALID_ARG;
    if (S > 65535) return PHB_ERR_UNSUPPORTED;
    cudaStream_t st = (cudaStream_t)stream;
    float2 *o = (float2 *)obj, *t = (float2 *)scratch;
    auto grid = [&](int64_t R, int64_t C) {
        return dim3((unsigned)((C + DT - 1) / DT), (unsigned)((R + DT - 1) / DT), (unsigned)S);
    };
    int rc;
    // forward: rows (over W) then columns (over H); the filter and 1/(H W) in the second pass
    k_dft_t<<<grid(H, W), 256, 0, st>>>(o, t, H, W, -1, 1.f, nullptr);
    if ((rc = check_launch())) return rc;
    k_dft_t<<<grid(W, H), 256, 0, st>>>(t, o, W, H, -1, (float)(1.0 / ((double)H * (double)W)), filter);
    if ((rc = check_launch())) return rc;
    k_dft_t<<<grid(H, W), 256, 0, st>>>(o, t, H, W, +1, 1.f, nullptr);
    if ((rc = check_launch())) return rc;
    k_dft_t<<<grid(W, H), 256, 0, st>>>(t, o, W, H, +1, 1.f, nullptr);
    return check_launch();
}

int phb_remove_phase_ramp_c64(void *obj, int64_t S, int64_t H, int64_t W, int64_t y0, int64_t y1, int64_t x0,
                              int64_t x1, double *sums, void *stream) {
    if (!obj || !sums || S < 1 || H < 1 || W < 1) return PHB_ERR_INVALID_ARG;
    if (y0 < 0 || x0 < 0 || y1 > H || x1 > W || y1 - y0 < 2 || x1 - x0 < 2) return PHB_ERR_INVALID_ARG;
    if (S > 65535) return PHB_ERR_UNSUPPORTED;
    cudaStream_t st = (cudaStream_t)stream;
    int rc = record_cuda(cudaMemsetAsync(sums, 0, (size_t)S * 3 * sizeof(double), st));
    if (rc) return rc;
    const int64_t n = (y1 - y0) * (x1 - x0);
    k_ramp_sums<<<dim3(flat_grid(n) > 296 ? 296 : flat_grid(n), (unsigned)S), 256, 0, st>>>(
        (const float2 *)obj, H, W, y0, y1, x0, x1, sums);
    if ((rc = check_launch())) return rc;
    k_ramp_apply<<<dim3(flat_grid(H * W) > 296 ? 296 : flat_grid(H * W), (unsigned)S), 256, 0, st>>>(
        (float2 *)obj, H, W, y0, y1, x0, x1, sums);
    return check_launch();
}

int phb_object_regularizers(const void *obj, int64_t S, int64_t H, int64_t W, const phb_obj_reg *reg, void *grad,
                            double *loss, void *stream) {
    if (!obj || !reg || S < 1 || H < 1 || W < 1 || (!grad && !loss)) return PHB_ERR_INVALID_ARG;
    k_obj_reg<<<flat_grid(S * H * W), 256, 0, (cudaStream_t)stream>>>((const float2 *)obj, S, H, W, *reg,
                                                                       (float2 *)grad, loss);
    return check_launch();
}

size_t phb_probe_regularizers_scratch_bytes(int32_t M, int32_t N) {
    return (M < 1 || N < 1) ? 0 : (size_t)2 * M * N * N * sizeof(float2);
}

int phb_probe_regularizers(const void *probe, int32_t M, int32_t N, const phb_probe_reg *reg, void *grad,
                           double *loss, void *scratch, void *stream) {
    if (!probe || !reg || !scratch || M < 1 || (!grad && !loss)) return PHB_ERR_INVALID_ARG;
    if (N != 64 && N != 128) return PHB_ERR_UNSUPPORTED;
    cudaStream_t st = (cudaStream_t)stream;
    const int64_t n = (int64_t)M * N * N;
    float2 *R = (float2 *)scratch, *gR = R + n;
    int rc = phb_fft2_c64(probe, R, M, N, 0, stream);
    if (rc) return rc;
    k_probe_reg<<<flat_grid(n), 256, 0, st>>>(R, M, N, *reg, grad ? gR : nullptr, loss);
    if ((rc = check_launch())) return rc;
    if (!grad) return PHB_OK;
    if ((rc = phb_fft2_c64(gR, R, M, N, 1, stream))) return rc;   // fft2 is unitary: adjoint = ifft2
    k_add_c<<<flat_grid(n), 256, 0, st>>>((float2 *)grad, R, n);
    return check_launch();
}

size_t phb_object_recip_l1_scratch_bytes(int64_t S, int64_t H, int64_t W) {
    return (S < 1 || H < 1 || W < 1) ? 0 : (size_t)(2 + S) * H * W * sizeof(float2);
}

int phb_object_recip_l1(const void *obj, int64_t S, int64_t H, int64_t W, float cost, void *grad, double *loss,
                        void *scratch, void *stream) {
    if (!obj || !scratch || S < 1 || H < 1 || W < 1 || (!grad && !loss)) return PHB_ERR_INVALID_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    const int64_t HW = H * W;
    float2 *a = (float2 *)scratch, *b = a + HW, *pre = b + HW;
    int rc = phb_project_slices(obj, S, HW, a, stream);
    if (rc) return rc;
    const float sc = (float)(1.0 / sqrt((double)HW));
    auto grid = [&](int64_t R, int64_t C) { return dim3((unsigned)((C + DT - 1) / DT), (unsigned)((R + DT - 1) / DT), 1u); };
    // Z = DFT2(P) / sqrt(HW) (the centring shift of fft2 changes only the phases of Z)
    k_dft_t<<<grid(H, W), 256, 0, st>>>(a, b, H, W, -1, 1.f, nullptr);
    if ((rc = check_launch())) return rc;
    k_dft_t<<<grid(W, H), 256, 0, st>>>(b, a, W, H, -1, sc, nullptr);
    if ((rc = check_launch())) return rc;
    k_unit_phase<<<flat_grid(HW), 256, 0, st>>>(a, HW, cost, loss);
    if ((rc = check_launch())) return rc;
    if (!grad) return PHB_OK;
    // gP = IDFT2(Z / |Z|) / sqrt(HW), then the product rule over slices
    k_dft_t<<<grid(H, W), 256, 0, st>>>(a, b, H, W, +1, 1.f, nullptr);
    if ((rc = check_launch())) return rc;
    k_dft_t<<<grid(W, H), 256, 0, st>>>(b, a, W, H, +1, sc, nullptr);
    if ((rc = check_launch())) return rc;
    k_recip_grad<<<flat_grid(HW), 256, 0, st>>>((const float2 *)obj, S, HW, a, cost, pre, (float2 *)grad);
    return check_launch();
}

size_t phb_smooth_positions_scratch_bytes(int64_t H, int64_t W) {
    return (H < 1 || W < 1) ? 0 : (size_t)2 * H * W * sizeof(float2);
}

int phb_smooth_position_values(float *vals, const float *scan, int64_t n, int64_t H, int64_t W, double corner_y,
                               double corner_x, double samp_y, double samp_x, const float *filter, float weight,
                               void *scratch, void *stream) {
    if (!vals || !scan || !filter || !scratch || n < 1 || H < 1 || W < 1) return PHB_ERR_INVALID_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    float2 *img = (float2 *)scratch, *tmp = img + H * W;
    k_nearest_fill<<<(unsigned)((H * W + 255) / 256), 256, 0, st>>>(scan, n, vals, H, W, corner_y, corner_x, samp_y,
                                                                   samp_x, img);
    int rc = check_launch();
    if (rc) return rc;
    // a real, k-symmetric filter keeps the two packed components apart
    if ((rc = phb_object_filter_c64(img, 1, H, W, filter, tmp, stream))) return rc;
    k_sample_blend<<<flat_grid(n), 256, 0, st>>>(img, scan, n, H, W, corner_y, corner_x, samp_y, samp_x, weight, vals);
    return check_launch();
}

}  // extern "C"
