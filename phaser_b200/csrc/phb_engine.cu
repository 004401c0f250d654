// The fused multislice mini-batch step of the LSQ-ML / ePIE / gradient engines.
//
// Reference algorithm: phaser/engines/conventional/solvers.py:132-504 (lsqml_dry_run,
// lsqml_run, epie_dry_run, epie_run), phaser/engines/gradient/run.py:357-438
// (run_model under jax.value_and_grad, dry_run), built from
// phaser/engines/common/simulation.py:160-306 and phaser/utils/object.py.
//
// Design (sm_100a):
//  * one CTA of 512 threads per (position b, probe mode m); the M CTAs of a
//    position form a thread-block cluster and exchange per-pixel mode sums
//    (illumination, far-field intensity, object-update numerators) through
//    distributed shared memory, so every global atomic is issued once per
//    position rather than once per mode;
//  * each CTA keeps its N x N wavefield in registers for the whole forward
//    and adjoint pass (phb_fft.cuh), multiplying cutouts and propagators in
//    as it goes; only the per-slice incident waves travel to HBM (for the
//    adjoint) -- the minimum traffic of the algorithm;
//  * object / probe updates are accumulated during the pass and applied by
//    small follow-up kernels once the group-global step sizes are known
//    (the reference applies them slice by slice, but its cutouts are copies
//    taken before the backward pass, so deferring is exact);
//  * step-size numerators / denominators and the position-gradient sums are
//    accumulated in float64 (block reduce, then one float64 atomic per CTA).
#include <cooperative_groups.h>

#include "phb_fft.cuh"
#include "phb_runtime.h"

namespace cg = cooperative_groups;

namespace phb {

enum Mode : int {
    MODE_LSQML = 0,
    MODE_EPIE = 1,
    MODE_GRAD = 2,
    MODE_PRE_LSQML = 3,
    MODE_PRE_EPIE = 4,
    MODE_PRE_GRAD = 5,
    MODE_SIM = 6,       // forward model only: far-field intensity sum_m |fft2(exit)|^2
};

// ---------------------------------------------------------------- workspace
struct Workspace {
    float2 *psi;        // B_max * M * S * N*N : per-slice incident waves (register order)
    float2 *acc_obj;    // S*H*W : object-update numerator accumulator
    float *illum;       // S*H*W : group illumination (group_probe_mag)
    float2 *acc_probe;  // M*N*N (K order): sum_b FFT(dP) conj(H)
    float *gom;         // N*N : group_obj_mag
    float2 *probe_k;    // M*N*N (K order): DFT(probe) / N^2
    float2 *prop_k;     // max(S-1,1)*N*N (K order)
    float *mask_k;      // N*N (K order)
    double *sums;       // float64 accumulators, see SumIdx
    double *coef;       // S + M step coefficients
    size_t bytes;
};

struct SumIdx {
    int64_t numO, denO, numP, denP, pnum, pden, pnorm, loss, total;
    __host__ __device__ SumIdx(int B, int S, int M) {
        numO = 0;
        denO = numO + (int64_t)B * S;
        numP = denO + S;
        denP = numP + (int64_t)B * M;
        pnum = denP + 1;
        pden = pnum + 2 * (int64_t)B;
        pnorm = pden + 2 * (int64_t)B;
        loss = pnorm + B;
        total = loss + B;
    }
};

static inline size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

static Workspace carve(void *base, int N, int M, int S, int B, int64_t H, int64_t W) {
    Workspace w{};
    char *p = (char *)base;
    size_t off = 0;
    auto take = [&](size_t bytes) {
        char *r = p ? p + off : nullptr;
        off += align256(bytes);
        return r;
    };
    const size_t NN = (size_t)N * N;
    w.psi = (float2 *)take((size_t)B * M * S * NN * sizeof(float2));
    w.acc_obj = (float2 *)take((size_t)S * H * W * sizeof(float2));
    w.illum = (float *)take((size_t)S * H * W * sizeof(float));
    w.acc_probe = (float2 *)take((size_t)M * NN * sizeof(float2));
    w.gom = (float *)take(NN * sizeof(float));
    w.probe_k = (float2 *)take((size_t)M * NN * sizeof(float2));
    w.prop_k = (float2 *)take((size_t)(S > 1 ? S - 1 : 1) * NN * sizeof(float2));
    w.mask_k = (float *)take(NN * sizeof(float));
    w.sums = (double *)take((size_t)SumIdx(B, S, M).total * sizeof(double));
    w.coef = (double *)take((size_t)(S + M + 4) * sizeof(double));
    w.bytes = off;
    return w;
}

// ---------------------------------------------------------------- arguments
struct GroupArgs {
    int M, S, B, B_max, mode, flags, noise;
    int64_t H, W, n_pos;
    double cy, cx, sy, sx;
    float eps, offset, var, beta_object;
    const float2 *object;
    const float *scan, *tilt, *thick;
    const int64_t *group;
    const float *patterns, *mask_k;
    const float2 *prop_k, *probe_k;
    const float *fy, *fx;
    float2 *psi, *acc_obj, *acc_probe;
    float *illum;
    double *sums;
    float *errors;
    double *pre_num, *pre_den;
    float *sim_out;
    const float *group_patterns;
};

template <int N>
__device__ __forceinline__ float2 obj_px(const float2 *Os, const CutoutIndex &ci, int64_t H, int64_t W, int r,
                                         int c) {
    const int64_t y = ci.y0 + r, x = ci.x0 + c;
    return (y >= 0 && y < H && x >= 0 && x < W) ? __ldg(Os + y * W + x) : make_float2(1.f, 0.f);
}

// tilt ramps of slice gap s: exp(2 pi i dz tan(t*1e-3) k) (simulation.py:193-222), separable in (ky, kx)
template <int N>
__device__ __forceinline__ void tilt_tables(const GroupArgs &a, int64_t pos, int s, float2 *ry, float2 *rx) {
    const float dz = a.thick[s];
    const float ty = tanf(a.tilt[2 * pos] * 1e-3f), tx = tanf(a.tilt[2 * pos + 1] * 1e-3f);
    for (int k = threadIdx.x; k < 2 * N; k += blockDim.x) {
        float sn, cs;
        if (k < N) {
            sincospif(2.0f * (dz * (ty * a.fy[k])), &sn, &cs);
            ry[k] = make_float2(cs, sn);
        } else {
            sincospif(2.0f * (dz * (tx * a.fx[k - N])), &sn, &cs);
            rx[k - N] = make_float2(cs, sn);
        }
    }
}

// Per-thread view of one position's cutout in R layout: row base offsets and a
// validity bit per register slot (identical for every slice).
template <int N>
struct CutView {
    int64_t base[FFTCfg<N>::U];   // (y0 + row(u)) * W + x0 + jl
    uint32_t valid;               // bit u*E + q: pixel (row(u), col(q)) inside the object
    __device__ __forceinline__ void init(const CutoutIndex &ci, int64_t H, int64_t W) {
        using I = Idx<N>;
        valid = 0u;
#pragma unroll
        for (int u = 0; u < I::U; ++u) {
            const int64_t y = ci.y0 + I::row(u);
            base[u] = y * W + ci.x0 + (threadIdx.x & 7);
            const bool rowok = y >= 0 && y < H;
#pragma unroll
            for (int q = 0; q < I::E; ++q) {
                const int64_t x = ci.x0 + I::col(q);
                if (rowok && x >= 0 && x < W) valid |= 1u << (u * I::E + q);
            }
        }
    }
    __device__ __forceinline__ float2 at(const float2 *Os, int u, int q) const {
        return (valid >> (u * FFTCfg<N>::E + q)) & 1u ? __ldg(Os + base[u] + FFTCfg<N>::NT * q)
                                                      : make_float2(1.f, 0.f);
    }
};

template <int N, int MODE>
__global__ void __launch_bounds__(FFT_THREADS, 1) k_group(const GroupArgs a) {
    using I = Idx<N>;
    constexpr int U = I::U, E = I::E, NN = N * N, SLOTS = U * E;
    cg::cluster_group cl = cg::this_cluster();
    const int M = a.M, S = a.S;
    const int m = (int)cl.block_rank();
    const int b = blockIdx.x / M;
    const int tid = threadIdx.x;

    extern __shared__ float4 smem_raw[];
    float2 *xb = reinterpret_cast<float2 *>(smem_raw);
    float2 *twid = xb + Lay<N>::BUF;
    float2 *hy = twid + N, *hx = hy + N;
    float2 *ry = hx + N, *rx = ry + N;
    double *dred = reinterpret_cast<double *>(rx + N);
    float *fred = reinterpret_cast<float *>(dred + 64);   // [0..31] block scratch, [32] cluster slot

    constexpr int mode = MODE;
    constexpr bool presolve = mode >= MODE_PRE_LSQML;
    constexpr bool lsqml = mode == MODE_LSQML, epie = mode == MODE_EPIE, grad = mode == MODE_GRAD;
    const bool upd_obj = !presolve && (a.flags & PHB_FLAG_UPDATE_OBJECT);
    const bool upd_probe = !presolve && (a.flags & PHB_FLAG_UPDATE_PROBE);
    const bool upd_pos = !presolve && (a.flags & PHB_FLAG_UPDATE_POSITION);
    const bool calc_err = !presolve && !grad && (a.flags & PHB_FLAG_CALC_ERROR) && a.errors;
    const bool do_illum = a.illum && (mode == MODE_LSQML || mode == MODE_PRE_LSQML);
    const bool tilted = a.tilt != nullptr;
    const SumIdx SI(a.B_max, S, M);
    double *sums = a.sums;

    const int64_t pos = a.group[b];
    const CutoutIndex ci = cutout_index(a.scan, pos, a.cy, a.cx, a.sy, a.sx, N, N);
    CutView<N> cv;
    cv.init(ci, a.H, a.W);

    fft_init_twiddles<N>(twid);
    for (int k = tid; k < N; k += blockDim.x) {
        float sn, cs;
        sincospif(-2.0f * (ci.sy * a.fy[k]), &sn, &cs);
        hy[k] = make_float2(cs, sn);
        sincospif(-2.0f * (ci.sx * a.fx[k]), &sn, &cs);
        hx[k] = make_float2(cs, sn);
    }
    __syncthreads();

    float2 *psi_b = a.psi + (size_t)(b * M + m) * S * NN;
    const int slot0 = (m * SLOTS) / M, slot1 = ((m + 1) * SLOTS) / M;

    // ---------------------------------------------------------- psi_0 = IFFT(FFT(P_m) H_b)
    float2 v[U][E];
    {
        const float2 *pk = a.probe_k + (size_t)m * NN;
#pragma unroll
        for (int u = 0; u < U; ++u)
#pragma unroll
            for (int e = 0; e < E; ++e)
                v[u][e] = cmul(__ldg(pk + I::flat(u, e)), cmul(hy[I::ky(e)], hx[I::kx(u)]));
        ifft2_k2r<N>(v, xb, twid);
    }
    if (upd_pos) {
        double n0 = 0.0;
#pragma unroll
        for (int u = 0; u < U; ++u)
#pragma unroll
            for (int q = 0; q < E; ++q) n0 += (double)cabs2(v[u][q]);
        block_sum_doubles<FFT_THREADS>(&n0, 1, dred);
        if (tid == 0) atomicAdd(sums + SI.pnorm + b, n0);
    }

    // ---------------------------------------------------------- forward multislice
    for (int s = 0; s < S; ++s) {
        const float2 *Os = a.object + (size_t)s * a.H * a.W;
        const bool last = (s == S - 1);
        if (upd_obj) {
            float2 *dst = psi_b + (size_t)s * NN;
#pragma unroll
            for (int u = 0; u < U; ++u)
#pragma unroll
                for (int q = 0; q < E; ++q) dst[I::flat(u, q)] = v[u][q];
        }
        if (do_illum) {   // group_probe_mag[s] += scatter(sum_m |psi_s|^2)
            float *xf = reinterpret_cast<float *>(xb);
#pragma unroll
            for (int u = 0; u < U; ++u)
#pragma unroll
                for (int q = 0; q < E; ++q) xf[I::flat(u, q)] = cabs2(v[u][q]);
            cl.sync();
            float *dst = a.illum + (size_t)s * a.H * a.W;
            for (int sl = slot0; sl < slot1; ++sl) {
                const int f = sl * FFT_THREADS + tid;
                float acc = 0.f;
                for (int r = 0; r < M; ++r) acc += cl.map_shared_rank(xf, r)[f];
                int rr, cc;
                flat_to_rc<N>(f, rr, cc);
                const int64_t y = ci.y0 + rr, x = ci.x0 + cc;
                if (y >= 0 && y < a.H && x >= 0 && x < a.W) atomicAdd(dst + y * a.W + x, acc);
            }
            cl.sync();
        }
        if (last && (mode == MODE_PRE_LSQML || mode == MODE_PRE_EPIE)) {
            // rescale: sum(I_exp * mask) / sum |fft2(psi_last)|^2 (Parseval), psi before transmission
            double t[2] = {0.0, 0.0};
#pragma unroll
            for (int u = 0; u < U; ++u)
#pragma unroll
                for (int q = 0; q < E; ++q) t[0] += (double)cabs2(v[u][q]);
            if (m == 0) {
                const float *pat = a.patterns + pos * NN;
                for (int f = tid; f < NN; f += FFT_THREADS) {
                    int ky, kx;
                    flat_to_k<N>(f, ky, kx);
                    t[1] += (double)(__ldg(pat + ky * N + kx) * __ldg(a.mask_k + f));
                }
            }
            block_sum_doubles<FFT_THREADS>(t, 2, dred);
            if (tid == 0) {
                atomicAdd(a.pre_den + b, t[0]);
                if (m == 0) atomicAdd(a.pre_num + b, t[1]);
            }
            return;
        }
#pragma unroll
        for (int u = 0; u < U; ++u)
#pragma unroll
            for (int q = 0; q < E; ++q) v[u][q] = cmul(v[u][q], cv.at(Os, u, q));
        if (last && mode == MODE_PRE_GRAD) {
            double t[2] = {0.0, 0.0};
#pragma unroll
            for (int u = 0; u < U; ++u)
#pragma unroll
                for (int q = 0; q < E; ++q) t[0] += (double)cabs2(v[u][q]);
            if (m == 0) {
                const float *pat = a.patterns + pos * NN;
                for (int f = tid; f < NN; f += FFT_THREADS) t[1] += (double)__ldg(pat + f);
            }
            block_sum_doubles<FFT_THREADS>(t, 2, dred);
            if (tid == 0) {
                atomicAdd(a.pre_den + b, t[0]);
                if (m == 0) atomicAdd(a.pre_num + b, t[1]);
            }
            return;
        }
        fft2_r2k<N>(v, xb, twid);
        if (!last) {
            if (tilted) {
                tilt_tables<N>(a, pos, s, ry, rx);
                __syncthreads();
            }
            const float2 *pr = a.prop_k + (size_t)s * NN;
            const float sc = 1.0f / (float)NN;
#pragma unroll
            for (int u = 0; u < U; ++u)
#pragma unroll
                for (int e = 0; e < E; ++e) {
                    float2 p = __ldg(pr + I::flat(u, e));
                    if (tilted) p = cmul(p, cmul(ry[I::ky(e)], rx[I::kx(u)]));
                    v[u][e] = cscale(cmul(v[u][e], p), sc);
                }
            ifft2_k2r<N>(v, xb, twid);
        } else {
            // ------------------------------------------------ detector: Psi = fft2(exit), constraint
            const float sc = 1.0f / (float)N;
            float *xf = reinterpret_cast<float *>(xb);
#pragma unroll
            for (int u = 0; u < U; ++u)
#pragma unroll
                for (int e = 0; e < E; ++e) {
                    v[u][e] = cscale(v[u][e], sc);
                    xf[I::flat(u, e)] = cabs2(v[u][e]);
                }
            cl.sync();
            if (mode == MODE_SIM) {
                if (m == 0) {
#pragma unroll
                    for (int u = 0; u < U; ++u)
#pragma unroll
                        for (int e = 0; e < E; ++e) {
                            const int f = I::flat(u, e);
                            float inten = 0.f;
                            for (int r = 0; r < M; ++r) inten += cl.map_shared_rank(xf, r)[f];
                            a.sim_out[(size_t)b * NN + I::ky(e) * N + I::kx(u)] = inten;
                        }
                }
                cl.sync();
                return;
            }
            const float *pat = a.group_patterns ? a.group_patterns + (size_t)b * NN : a.patterns + pos * NN;
            double e2 = 0.0, loss = 0.0;
#pragma unroll
            for (int u = 0; u < U; ++u)
#pragma unroll
                for (int e = 0; e < E; ++e) {
                    const int f = I::flat(u, e);
                    float inten = 0.f;
                    for (int r = 0; r < M; ++r) inten += cl.map_shared_rank(xf, r)[f];
                    const float pv = __ldg(pat + I::ky(e) * N + I::kx(u));
                    const float mk = __ldg(a.mask_k + f);
                    if (calc_err && m == 0) {
                        const float d = inten - pv;
                        if (d == d) e2 += (double)d * (double)d;
                    }
                    const float pm = np_max0(pv);
                    float fac;
                    if (!grad) {
                        // amplitude / anscombe wave update (noise_models.py:47-64)
                        fac = (sqrtf(pm + a.offset) / (sqrtf(inten + a.offset) + a.eps) - 1.0f) * mk;
                    } else if (a.noise == PHB_NOISE_POISSON) {
                        // d/dI of mask*(I + eps + p*(log(p+eps) - log(I+eps) - 1)) (noise_models.py:86-102)
                        if (m == 0)
                            loss += (double)(mk * (inten + a.eps +
                                                   pm * (logf(pm + a.eps) - logf(inten + a.eps) - 1.0f)));
                        fac = 2.0f * mk * (1.0f - pm / (inten + a.eps));
                    } else {
                        // d/dI of 2 mask (sqrt(p+c) - sqrt(I+c) - eps)^2 / var (noise_models.py:29-45)
                        const float sI = sqrtf(inten + a.offset);
                        const float dlt = sqrtf(pm + a.offset) - sI - a.eps;
                        if (m == 0) loss += (double)(2.0f * mk * dlt * dlt / a.var);
                        fac = 2.0f * (-2.0f * mk * dlt / (a.var * sI));
                    }
                    v[u][e] = cscale(v[u][e], fac);
                }
            cl.sync();
            if (m == 0 && (calc_err || grad)) {
                double t[2] = {e2, loss};
                block_sum_doubles<FFT_THREADS>(t, 2, dred);
                if (tid == 0) {
                    if (calc_err) a.errors[pos] = (float)sqrt(t[0]);
                    if (grad) sums[SI.loss + b] = t[1];
                }
            }
            ifft2_k2r<N>(v, xb, twid);
#pragma unroll
            for (int u = 0; u < U; ++u)
#pragma unroll
                for (int q = 0; q < E; ++q) v[u][q] = cscale(v[u][q], sc);
        }
    }

    // ---------------------------------------------------------- adjoint, slice by slice
    for (int s = S - 1; s >= 0; --s) {
        const float2 *Os = a.object + (size_t)s * a.H * a.W;
        float2 *ps = psi_b + (size_t)s * NN;
        if (!epie) {
            // LSQ-ML: dO = chi conj(psi), dP = chi conj(O) (solvers.py:242-271); gradient: same adjoint
            double t[4] = {0.0, 0.0, 0.0, 0.0};
            float2 *xc = xb;
#pragma unroll
            for (int u = 0; u < U; ++u)
#pragma unroll
                for (int q = 0; q < E; ++q) {
                    const int f = I::flat(u, q);
                    const float2 c = v[u][q];
                    const float2 o = cv.at(Os, u, q);
                    const float c2 = cabs2(c);
                    if (upd_obj) {
                        const float2 p = ps[f];
                        xc[f] = cmulc(c, p);
                        const float p2 = cabs2(p);
                        t[0] += (double)(c2 * p2);
                        t[1] += (double)(c2 * p2) * (double)p2;
                    }
                    if (s == 0) {
                        if (lsqml && upd_probe) {
                            const float o2 = cabs2(o);
                            t[2] += (double)(c2 * o2);
                            t[3] += (double)(c2 * o2) * (double)o2;
                        }
                        if (upd_pos) ps[f] = c;   // exit-wave update of slice 0 for the position step
                    }
                    v[u][q] = cmulc(c, o);
                }
            if (upd_obj) {
                cl.sync();
                float2 *dst = a.acc_obj + (size_t)s * a.H * a.W;
                for (int sl = slot0; sl < slot1; ++sl) {
                    const int f = sl * FFT_THREADS + tid;
                    float2 acc = make_float2(0.f, 0.f);
                    for (int r = 0; r < M; ++r) acc = cadd(acc, cl.map_shared_rank(xc, r)[f]);
                    int rr, cc;
                    flat_to_rc<N>(f, rr, cc);
                    const int64_t y = ci.y0 + rr, x = ci.x0 + cc;
                    if (y >= 0 && y < a.H && x >= 0 && x < a.W) atomic_add_c(dst + y * a.W + x, acc);
                }
                cl.sync();
            }
            if (lsqml && (upd_obj || (s == 0 && upd_probe))) {
                block_sum_doubles<FFT_THREADS>(t, 4, dred);
                if (tid == 0) {
                    if (upd_obj) {
                        atomicAdd(sums + SI.numO + (int64_t)b * S + s, t[0]);
                        atomicAdd(sums + SI.denO + s, t[1]);
                    }
                    if (s == 0 && upd_probe) {
                        atomicAdd(sums + SI.numP + (int64_t)b * M + m, t[2]);
                        atomicAdd(sums + SI.denP, t[3]);
                    }
                }
            }
        } else {
            // ePIE: dP = conj(O) chi / max|O|^2; O += beta/S sum_m conj(psi) chi / max sum_m |psi|^2
            // (solvers.py:459-486)
            float omax = 0.f;
            float *xf = reinterpret_cast<float *>(xb);
#pragma unroll
            for (int u = 0; u < U; ++u)
#pragma unroll
                for (int q = 0; q < E; ++q) {
                    const float2 o = cv.at(Os, u, q);
                    omax = fmaxf(omax, cabs2(o));
                    if (upd_obj) xf[I::flat(u, q)] = cabs2(ps[I::flat(u, q)]);
                }
            omax = block_max_float<FFT_THREADS>(omax, fred);
            if (upd_obj) {
                cl.sync();
                float lmax = 0.f;
                for (int sl = slot0; sl < slot1; ++sl) {
                    const int f = sl * FFT_THREADS + tid;
                    float w = 0.f;
                    for (int r = 0; r < M; ++r) w += cl.map_shared_rank(xf, r)[f];
                    lmax = fmaxf(lmax, w);
                }
                lmax = block_max_float<FFT_THREADS>(lmax, fred);
                if (tid == 0) fred[32] = lmax;
                cl.sync();
                float wmax = 0.f;
                for (int r = 0; r < M; ++r) wmax = fmaxf(wmax, cl.map_shared_rank(fred, r)[32]);
                float2 *xc = xb;
#pragma unroll
                for (int u = 0; u < U; ++u)
#pragma unroll
                    for (int q = 0; q < E; ++q) xc[I::flat(u, q)] = cmulc(v[u][q], ps[I::flat(u, q)]);
                cl.sync();
                const float scl = a.beta_object / (float)S / wmax;
                float2 *dst = a.acc_obj + (size_t)s * a.H * a.W;
                for (int sl = slot0; sl < slot1; ++sl) {
                    const int f = sl * FFT_THREADS + tid;
                    float2 acc = make_float2(0.f, 0.f);
                    for (int r = 0; r < M; ++r) acc = cadd(acc, cl.map_shared_rank(xc, r)[f]);
                    int rr, cc;
                    flat_to_rc<N>(f, rr, cc);
                    const int64_t y = ci.y0 + rr, x = ci.x0 + cc;
                    if (y >= 0 && y < a.H && x >= 0 && x < a.W) atomic_add_c(dst + y * a.W + x, cscale(acc, scl));
                }
                cl.sync();
            }
            const float inv = 1.0f / omax;
#pragma unroll
            for (int u = 0; u < U; ++u)
#pragma unroll
                for (int q = 0; q < E; ++q) {
                    const float2 c = v[u][q];
                    if (s == 0 && upd_pos) ps[I::flat(u, q)] = c;
                    const float2 o = cv.at(Os, u, q);
                    v[u][q] = cscale(cmulc(c, o), inv);
                }
        }

        if (s > 0) {
            if (tilted) tilt_tables<N>(a, pos, s - 1, ry, rx);   // read after the FFT's barriers
            fft2_r2k<N>(v, xb, twid);
            const float2 *pr = a.prop_k + (size_t)(s - 1) * NN;
            const float sc = 1.0f / (float)NN;
#pragma unroll
            for (int u = 0; u < U; ++u)
#pragma unroll
                for (int e = 0; e < E; ++e) {
                    float2 p = __ldg(pr + I::flat(u, e));
                    if (tilted) p = cmul(p, cmul(ry[I::ky(e)], rx[I::kx(u)]));
                    v[u][e] = cscale(cmulc(v[u][e], p), sc);
                }
            ifft2_k2r<N>(v, xb, twid);
        } else if (upd_probe) {
            // sum_b fft2(dP) conj(H_b): accumulated per mode in K order (solvers.py:265, 484)
            fft2_r2k<N>(v, xb, twid);
            float2 *ap = a.acc_probe + (size_t)m * NN;
            const float sc = 1.0f / (float)N;
#pragma unroll
            for (int u = 0; u < U; ++u)
#pragma unroll
                for (int e = 0; e < E; ++e) {
                    const float2 h = cmul(hy[I::ky(e)], hx[I::kx(u)]);
                    atomic_add_c(ap + I::flat(u, e), cscale(cmulc(v[u][e], h), sc));
                }
        }
    }

    // ---------------------------------------------------------- position step (solvers.py:275-288)
    if (upd_pos) {
        const float2 *pk = a.probe_k + (size_t)m * NN;
        const float2 *ps0 = psi_b;
        const float twopi = 6.283185307179586f;
        for (int dir = 0; dir < 2; ++dir) {
#pragma unroll
            for (int u = 0; u < U; ++u)
#pragma unroll
                for (int e = 0; e < E; ++e) {
                    const int ky = I::ky(e), kx = I::kx(u);
                    const float k = dir == 0 ? a.fy[ky] : a.fx[kx];
                    const float2 g = cmul(__ldg(pk + I::flat(u, e)), cmul(hy[ky], hx[kx]));
                    const float w = twopi * k;
                    v[u][e] = make_float2(w * g.y, -w * g.x);   // g * (-2 pi i k)
                }
            ifft2_k2r<N>(v, xb, twid);
            double t[2] = {0.0, 0.0};
#pragma unroll
            for (int u = 0; u < U; ++u)
#pragma unroll
                for (int q = 0; q < E; ++q) {
                    const float2 o = cv.at(a.object, u, q);
                    const float2 c = ps0[I::flat(u, q)];
                    const float2 pr = cmul(v[u][q], o);
                    t[0] += (double)(c.x * pr.x + c.y * pr.y);
                    t[1] += (double)cabs2(pr);
                }
            block_sum_doubles<FFT_THREADS>(t, 2, dred);
            if (tid == 0) {
                atomicAdd(sums + SI.pnum + 2 * b + dir, t[0]);
                atomicAdd(sums + SI.pden + 2 * b + dir, t[1]);
            }
        }
    }
}

// ---------------------------------------------------------------- group_obj_mag
// gom[r, c] += sum_b |prod_s O_s[y0_b + r, x0_b + c]|^2  (solvers.py:203)
template <int N>
__global__ void k_gom(const GroupArgs a, float *out) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    const int r = f / N, c = f % N;
    const int nsplit = gridDim.y;
    const int b0 = (a.B * blockIdx.y) / nsplit, b1 = (a.B * (blockIdx.y + 1)) / nsplit;
    float acc = 0.f;
    for (int b = b0; b < b1; ++b) {
        const CutoutIndex ci = cutout_index(a.scan, a.group[b], a.cy, a.cx, a.sy, a.sx, N, N);
        float2 prod = make_float2(1.f, 0.f);
        for (int s = 0; s < a.S; ++s)
            prod = cmul(prod, obj_px<N>(a.object + (size_t)s * a.H * a.W, ci, a.H, a.W, r, c));
        acc += cabs2(prod);
    }
    if (f < N * N) atomicAdd(out + f, acc);
}

// ---------------------------------------------------------------- group-global scalars
struct FinArgs {
    int mode, flags, S, M, B, B_max;
    float beta_object, beta_probe, gamma;
    const int64_t *group;
    double *sums, *coef;
    float *pos_update, *grad_pos, *loss;
};

__global__ void k_finalize(const FinArgs f) {
    const SumIdx SI(f.B_max, f.S, f.M);
    double *sums = f.sums;
    __shared__ double red[2][32];
    const int tid = threadIdx.x;
    if (f.mode == MODE_LSQML) {
        for (int s = tid; s < f.S; s += blockDim.x) {
            double acc = 0.0;
            for (int b = 0; b < f.B; ++b) acc += sums[SI.numO + (int64_t)b * f.S + s];
            f.coef[s] = (double)f.beta_object * acc / (sums[SI.denO + s] + (double)f.gamma);
        }
        for (int m = tid; m < f.M; m += blockDim.x) {
            double acc = 0.0;
            for (int b = 0; b < f.B; ++b) acc += sums[SI.numP + (int64_t)b * f.M + m];
            f.coef[f.S + m] = (double)f.beta_probe * acc / (sums[SI.denP] + (double)f.gamma);
        }
    }
    const bool pos = (f.flags & PHB_FLAG_UPDATE_POSITION) && (f.mode <= MODE_GRAD);
    if (pos && f.mode != MODE_GRAD && f.pos_update) {
        double d[2] = {0.0, 0.0};
        for (int b = tid; b < f.B; b += blockDim.x) {
            const double n = sums[SI.pnorm + b];
            d[0] += sums[SI.pden + 2 * b] / (n * n);
            d[1] += sums[SI.pden + 2 * b + 1] / (n * n);
        }
        for (int k = 0; k < 2; ++k) {
            double v = d[k];
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if ((tid & 31) == 0) red[k][tid >> 5] = v;
        }
        __syncthreads();
        if (tid < 32) {
            for (int k = 0; k < 2; ++k) {
                double v = (tid < (int)(blockDim.x >> 5)) ? red[k][tid] : 0.0;
                for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
                if (tid == 0) red[k][0] = v;
            }
        }
        __syncthreads();
        for (int b = tid; b < f.B; b += blockDim.x) {
            const double n = sums[SI.pnorm + b];
            const int64_t p = f.group[b];
            f.pos_update[2 * p] = (float)(sums[SI.pnum + 2 * b] / n / red[0][0]);
            f.pos_update[2 * p + 1] = (float)(sums[SI.pnum + 2 * b + 1] / n / red[1][0]);
        }
    }
    if (f.mode == MODE_GRAD) {
        for (int b = tid; b < f.B; b += blockDim.x) {
            const int64_t p = f.group[b];
            if (pos && f.grad_pos) {
                f.grad_pos[2 * p] = (float)sums[SI.pnum + 2 * b];
                f.grad_pos[2 * p + 1] = (float)sums[SI.pnum + 2 * b + 1];
            }
            if (f.loss) f.loss[p] = (float)sums[SI.loss + b];
        }
    }
    __syncthreads();
    for (int64_t i = tid; i < SI.total; i += blockDim.x) sums[i] = 0.0;
}

// ---------------------------------------------------------------- object apply
struct ObjApplyArgs {
    int mode, S;
    int64_t HW;
    float reg, eps;
    float2 *object, *acc;
    float *illum, *new_probe_mag;
    const double *coef;
    int32_t *status;
    int32_t group_index;
    int update;
};

__global__ void k_obj_apply(const ObjApplyArgs a) {
    const int64_t total = (int64_t)a.S * a.HW;
    bool bad = false;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (int64_t)gridDim.x * blockDim.x) {
        float2 o = a.object[i];
        if (a.update) {
            const float2 acc = a.acc[i];
            if (a.mode == MODE_LSQML) {
                const float g = a.illum[i];
                const float cs = (float)a.coef[i / a.HW];
                // O += beta * sum_b(alpha_b) * (acc / (g + reg)) * g / (g + 1e-16)   (solvers.py:252-257)
                const float2 avg = cscale(acc, 1.0f / (g + a.reg));
                o = cadd(o, cscale(avg, cs * g / (g + a.eps)));
            } else {
                o = cadd(o, acc);
            }
            a.object[i] = o;
            a.acc[i] = make_float2(0.f, 0.f);
        }
        if (a.illum) {
            if (a.new_probe_mag) a.new_probe_mag[i] += a.illum[i];
            a.illum[i] = 0.f;
        }
        bad |= !finite2(o);
    }
    if (bad && a.status) atomicCAS(a.status, -1, a.group_index);
}

// ---------------------------------------------------------------- probe apply / spectrum refresh
struct ProbeApplyArgs {
    int mode, M, B;
    float reg, eps;
    float2 *probe, *probe_k, *acc;
    const float *gom;
    float *new_obj_mag;
    const double *coef;
    int S;
    float beta_probe;
    float2 *grad_probe;
    int32_t *status;
    int32_t group_index;
    int update;
};

// One CTA per mode: P_m += update (LSQ-ML solvers.py:262-269, ePIE 483-485, or the gradient
// output), then refresh the cached spectrum DFT(P_m)/N^2 in K order for the next group.
template <int N>
__global__ void __launch_bounds__(FFT_THREADS, 1) k_probe_apply(const ProbeApplyArgs a) {
    using I = Idx<N>;
    constexpr int U = I::U, E = I::E, NN = N * N;
    extern __shared__ float4 smem_raw[];
    float2 *xb = reinterpret_cast<float2 *>(smem_raw);
    float2 *twid = xb + Lay<N>::BUF;
    float *fred = reinterpret_cast<float *>(twid + N);
    fft_init_twiddles<N>(twid);
    __syncthreads();
    const int m = blockIdx.x;
    float2 *P = a.probe + (size_t)m * NN;
    float2 v[U][E];
    bool bad = false;
    if (a.update) {
        float2 *acc = a.acc + (size_t)m * NN;
#pragma unroll
        for (int u = 0; u < U; ++u)
#pragma unroll
            for (int e = 0; e < E; ++e) {
                v[u][e] = acc[I::flat(u, e)];
                acc[I::flat(u, e)] = make_float2(0.f, 0.f);
            }
        ifft2_k2r<N>(v, xb, twid);
        const float sc = 1.0f / (float)N;
#pragma unroll
        for (int u = 0; u < U; ++u)
#pragma unroll
            for (int q = 0; q < E; ++q) {
                const int idx = I::row(u) * N + I::col(q);
                float2 d = cscale(v[u][q], sc);
                if (a.mode == MODE_GRAD) {
                    a.grad_probe[(size_t)m * NN + idx] = cadd(a.grad_probe[(size_t)m * NN + idx], d);
                    continue;
                }
                float2 p = P[idx];
                if (a.mode == MODE_LSQML) {
                    const float g = a.gom[idx];
                    const float cs = (float)a.coef[a.S + m];
                    d = cscale(d, 1.0f / (g + a.reg));
                    p = cadd(p, cscale(d, cs * g / (g + a.eps)));
                } else {
                    p = cadd(p, cscale(d, a.beta_probe / (float)a.B));
                }
                P[idx] = p;
            }
        __syncthreads();
    }
    if (m == 0 && a.new_obj_mag && a.gom)
        for (int i = threadIdx.x; i < NN; i += blockDim.x) a.new_obj_mag[i] += a.gom[i];
    if (a.mode == MODE_GRAD) return;
    // refresh spectrum
#pragma unroll
    for (int u = 0; u < U; ++u)
#pragma unroll
        for (int q = 0; q < E; ++q) {
            v[u][q] = P[I::row(u) * N + I::col(q)];
            bad |= !finite2(v[u][q]);
        }
    __syncthreads();
    fft2_r2k<N>(v, xb, twid);
    const float sc = 1.0f / (float)NN;
#pragma unroll
    for (int u = 0; u < U; ++u)
#pragma unroll
        for (int e = 0; e < E; ++e) a.probe_k[(size_t)m * NN + I::flat(u, e)] = cscale(v[u][e], sc);
    if (bad && a.status) atomicCAS(a.status, -1, a.group_index);
    (void)fred;
}

// ---------------------------------------------------------------- K-order packing
template <int N>
__global__ void k_pack_c64(const float2 *src, float2 *dst) {
    using I = Idx<N>;
    const size_t base = (size_t)blockIdx.x * N * N;
#pragma unroll
    for (int u = 0; u < I::U; ++u)
#pragma unroll
        for (int e = 0; e < I::E; ++e) dst[base + I::flat(u, e)] = src[base + I::ky(e) * N + I::kx(u)];
}
template <int N>
__global__ void k_pack_f32(const float *src, float *dst) {
    using I = Idx<N>;
#pragma unroll
    for (int u = 0; u < I::U; ++u)
#pragma unroll
        for (int e = 0; e < I::E; ++e) dst[I::flat(u, e)] = src[I::ky(e) * N + I::kx(u)];
}

// ---------------------------------------------------------------- per-iteration helpers
template <int NT>
__device__ double block_sum1(double v, double *red) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32) {
        double w = threadIdx.x < NT / 32 ? red[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) w += __shfl_xor_sync(0xffffffffu, w, o);
        if (threadIdx.x == 0) red[0] = w;
    }
    __syncthreads();
    double r = red[0];
    __syncthreads();
    return r;
}

// run.py:95-110 and position_correction.py:21-61 (numpy aliasing: the momentum state is the
// same array as the update, so it also receives the second mean subtraction).
__global__ void __launch_bounds__(1024) k_position_update(float *scan, float *upd, float *state, int64_t n,
                                                         int use_mom, float step, float maxs, float mom,
                                                         double y0, double x0, double y1, double x1,
                                                         int32_t *n_out) {
    __shared__ double red[32];
    double sy = 0.0, sx = 0.0;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
        sy += upd[2 * i];
        sx += upd[2 * i + 1];
    }
    const float my = (float)(block_sum1<1024>(sy, red) / (double)n);
    const float mx = (float)(block_sum1<1024>(sx, red) / (double)n);
    sy = 0.0;
    sx = 0.0;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
        const float gy = upd[2 * i] - my, gx = upd[2 * i + 1] - mx;
        float uy = step * gy, ux = step * gx;
        if (use_mom) {
            uy += mom * state[2 * i];
            ux += mom * state[2 * i + 1];
        }
        if (maxs > 0.f) {
            const float mag = sqrtf(uy * uy + ux * ux);
            const float fct = fminf(mag, maxs) / mag;
            uy *= fct;
            ux *= fct;
        }
        upd[2 * i] = uy;
        upd[2 * i + 1] = ux;
        sy += uy;
        sx += ux;
    }
    const float my2 = (float)(block_sum1<1024>(sy, red) / (double)n);
    const float mx2 = (float)(block_sum1<1024>(sx, red) / (double)n);
    int outside = 0;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
        const float uy = upd[2 * i] - my2, ux = upd[2 * i + 1] - mx2;
        upd[2 * i] = uy;
        upd[2 * i + 1] = ux;
        if (use_mom) {
            state[2 * i] = uy;
            state[2 * i + 1] = ux;
        }
        const float py = scan[2 * i] + uy, px = scan[2 * i + 1] + ux;
        scan[2 * i] = py;
        scan[2 * i + 1] = px;
        outside += ((double)py < y0) || ((double)py > y1) || ((double)px < x0) || ((double)px > x1);
    }
    const double tot = block_sum1<1024>((double)outside, red);
    if (threadIdx.x == 0) *n_out = (int32_t)tot;
}

__global__ void __launch_bounds__(1024) k_nanmean(const float *v, int64_t n, double *out, int64_t *count) {
    __shared__ double red[32];
    double s = 0.0, c = 0.0;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
        const float x = v[i];
        if (x == x) {
            s += x;
            c += 1.0;
        }
    }
    s = block_sum1<1024>(s, red);
    c = block_sum1<1024>(c, red);
    if (threadIdx.x == 0) {
        *out = c > 0 ? s / c : (double)NAN;
        if (count) *count = (int64_t)c;
    }
}

__global__ void k_iteration_reset(int32_t *status, float *errors, int64_t n) {
    const int64_t i0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i0 == 0) *status = -1;
    for (int64_t i = i0; i < n; i += (int64_t)gridDim.x * blockDim.x) errors[i] = NAN;
}

__global__ void __launch_bounds__(1024) k_iteration_report(const int32_t *status, const int32_t *n_out,
                                                           const float *errors, int64_t n, double *out) {
    __shared__ double red[32];
    double s = 0.0, c = 0.0;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
        const float x = errors[i];
        if (x == x) {
            s += x;
            c += 1.0;
        }
    }
    s = block_sum1<1024>(s, red);
    c = block_sum1<1024>(c, red);
    if (threadIdx.x == 0) {
        out[0] = (double)*status;
        out[1] = n_out ? (double)*n_out : 0.0;
        out[2] = c > 0 ? s / c : (double)NAN;
        out[3] = c;
    }
}

__global__ void k_check_finite(const float2 *v, int64_t n, int32_t *status, int32_t code) {
    bool bad = false;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        bad |= !finite2(v[i]);
    if (bad) atomicCAS(status, -1, code);
}

// ---------------------------------------------------------------- host glue
template <int N>
static size_t group_smem_bytes() {
    return (size_t)Lay<N>::BUF * sizeof(float2) + 5 * N * sizeof(float2) + 64 * sizeof(double) + 64 * sizeof(float);
}
template <int N>
static size_t fft_smem_bytes() {
    return (size_t)Lay<N>::BUF * sizeof(float2) + N * sizeof(float2) + 64 * sizeof(float);
}

template <int N>
static int configure_kernels() {
    static int done = -1;
    if (done >= 0) return done;
    int rc = PHB_OK;
    if (cudaFuncSetAttribute(k_probe_apply<N>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)fft_smem_bytes<N>()) != cudaSuccess)
        rc = record_cuda(cudaGetLastError());
    done = rc;
    return rc;
}

static int validate(const phb_engine *e) {
    if (!e) return PHB_ERR_INVALID_ARG;
    if (e->N != 64 && e->N != 128) return PHB_ERR_UNSUPPORTED;
    if (e->M < 1 || e->M > 8) return PHB_ERR_UNSUPPORTED;
    if (e->S < 1 || e->B_max < 1 || e->H < 1 || e->W < 1 || e->n_pos < 1) return PHB_ERR_INVALID_ARG;
    if (!e->object || !e->probe || !e->scan || !e->patterns || !e->pattern_mask || !e->ky || !e->kx)
        return PHB_ERR_INVALID_ARG;
    if (e->S > 1 && !e->propagators) return PHB_ERR_INVALID_ARG;
    if (e->tilt && !e->thicknesses) return PHB_ERR_INVALID_ARG;
    if (!(e->samp_y > 0) || !(e->samp_x > 0)) return PHB_ERR_INVALID_ARG;
    if (!e->workspace || ((uintptr_t)e->workspace & 255)) return PHB_ERR_INVALID_ARG;
    const size_t need = carve(nullptr, e->N, e->M, e->S, e->B_max, e->H, e->W).bytes;
    if (e->workspace_bytes < need) return PHB_ERR_INVALID_ARG;
    return PHB_OK;
}

static GroupArgs make_args(const phb_engine *e, const Workspace &w, int mode, int flags, const int64_t *group,
                           int B) {
    GroupArgs a{};
    a.M = e->M;
    a.S = e->S;
    a.B = B;
    a.B_max = e->B_max;
    a.mode = mode;
    a.flags = flags;
    a.noise = e->noise;
    a.H = e->H;
    a.W = e->W;
    a.n_pos = e->n_pos;
    a.cy = e->corner_y;
    a.cx = e->corner_x;
    a.sy = e->samp_y;
    a.sx = e->samp_x;
    a.eps = e->noise_eps;
    a.offset = e->noise_offset;
    a.var = e->noise_var;
    a.object = (const float2 *)e->object;
    a.scan = e->scan;
    a.tilt = e->tilt;
    a.thick = e->thicknesses;
    a.group = group;
    a.patterns = e->patterns;
    a.mask_k = w.mask_k;
    a.prop_k = w.prop_k;
    a.probe_k = w.probe_k;
    a.fy = e->ky;
    a.fx = e->kx;
    a.psi = w.psi;
    a.acc_obj = w.acc_obj;
    a.acc_probe = w.acc_probe;
    a.illum = w.illum;
    a.sums = w.sums;
    return a;
}

template <int N, int MODE>
static int launch_group_mode(const GroupArgs &a, cudaStream_t st) {
    static bool configured = false;
    if (!configured) {
        if (cudaFuncSetAttribute(k_group<N, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)group_smem_bytes<N>()) != cudaSuccess)
            return record_cuda(cudaGetLastError());
        configured = true;
    }
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3((unsigned)(a.B * a.M), 1, 1);
    cfg.blockDim = dim3(FFT_THREADS, 1, 1);
    cfg.dynamicSmemBytes = group_smem_bytes<N>();
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)a.M;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    const int rc = record_cuda(cudaLaunchKernelEx(&cfg, k_group<N, MODE>, a));
    if (rc == PHB_OK) count_launch();
    return rc;
}

template <int N>
static int launch_group(const GroupArgs &a, cudaStream_t st) {
    switch (a.mode) {
        case MODE_LSQML: return launch_group_mode<N, MODE_LSQML>(a, st);
        case MODE_EPIE: return launch_group_mode<N, MODE_EPIE>(a, st);
        case MODE_GRAD: return launch_group_mode<N, MODE_GRAD>(a, st);
        case MODE_PRE_LSQML: return launch_group_mode<N, MODE_PRE_LSQML>(a, st);
        case MODE_PRE_EPIE: return launch_group_mode<N, MODE_PRE_EPIE>(a, st);
        case MODE_PRE_GRAD: return launch_group_mode<N, MODE_PRE_GRAD>(a, st);
        case MODE_SIM: return launch_group_mode<N, MODE_SIM>(a, st);
        default: return PHB_ERR_INVALID_ARG;
    }
}

template <int N>
static int probe_spectrum(const phb_engine *e, const Workspace &w, cudaStream_t st) {
    ProbeApplyArgs p{};
    p.mode = MODE_LSQML;
    p.M = e->M;
    p.probe = (float2 *)e->probe;
    p.probe_k = w.probe_k;
    p.update = 0;
    k_probe_apply<N><<<e->M, FFT_THREADS, fft_smem_bytes<N>(), st>>>(p);
    return check_launch();
}

template <int N>
static int engine_init(const phb_engine *e, cudaStream_t st) {
    int rc = configure_kernels<N>();
    if (rc) return rc;
    Workspace w = carve(e->workspace, N, e->M, e->S, e->B_max, e->H, e->W);
    const size_t NN = (size_t)N * N;
    rc = record_cuda(cudaMemsetAsync(w.acc_obj, 0, (size_t)e->S * e->H * e->W * sizeof(float2), st));
    if (!rc) rc = record_cuda(cudaMemsetAsync(w.illum, 0, (size_t)e->S * e->H * e->W * sizeof(float), st));
    if (!rc) rc = record_cuda(cudaMemsetAsync(w.acc_probe, 0, (size_t)e->M * NN * sizeof(float2), st));
    if (!rc) rc = record_cuda(cudaMemsetAsync(w.gom, 0, NN * sizeof(float), st));
    if (!rc)
        rc = record_cuda(cudaMemsetAsync(w.sums, 0, (size_t)SumIdx(e->B_max, e->S, e->M).total * sizeof(double), st));
    if (rc) return rc;
    if (e->S > 1) {
        k_pack_c64<N><<<e->S - 1, FFT_THREADS, 0, st>>>((const float2 *)e->propagators, w.prop_k);
        if ((rc = check_launch())) return rc;
    }
    k_pack_f32<N><<<1, FFT_THREADS, 0, st>>>(e->pattern_mask, w.mask_k);
    if ((rc = check_launch())) return rc;
    return probe_spectrum<N>(e, w, st);
}

template <int N>
static int presolve(const phb_engine *e, const int64_t *group, int B, int solver, int gradient_form, double *num,
                    double *den, cudaStream_t st) {
    int rc = configure_kernels<N>();
    if (rc) return rc;
    Workspace w = carve(e->workspace, N, e->M, e->S, e->B_max, e->H, e->W);
    const int mode = gradient_form ? MODE_PRE_GRAD : (solver == PHB_SOLVER_EPIE ? MODE_PRE_EPIE : MODE_PRE_LSQML);
    GroupArgs a = make_args(e, w, mode, 0, group, B);
    a.pre_num = num;
    a.pre_den = den;
    a.illum = (mode == MODE_PRE_LSQML) ? e->new_probe_mag : nullptr;
    if (mode == MODE_PRE_LSQML && e->new_obj_mag) {
        k_gom<N><<<dim3((N * N + 255) / 256, 8), 256, 0, st>>>(a, e->new_obj_mag);
        if ((rc = check_launch())) return rc;
    }
    return launch_group<N>(a, st);
}

template <int N>
static int simulate(const phb_engine *e, const int64_t *group, int B, float *out, cudaStream_t st) {
    int rc = configure_kernels<N>();
    if (rc) return rc;
    Workspace w = carve(e->workspace, N, e->M, e->S, e->B_max, e->H, e->W);
    GroupArgs a = make_args(e, w, MODE_SIM, 0, group, B);
    a.illum = nullptr;
    a.sim_out = out;
    return launch_group<N>(a, st);
}

template <int N>
static int solver_group(const phb_engine *e, const phb_step *sp, const int64_t *group, int B, cudaStream_t st) {
    int rc = configure_kernels<N>();
    if (rc) return rc;
    Workspace w = carve(e->workspace, N, e->M, e->S, e->B_max, e->H, e->W);
    const int mode = sp->solver == PHB_SOLVER_EPIE ? MODE_EPIE : (sp->solver == PHB_SOLVER_GRAD ? MODE_GRAD : MODE_LSQML);
    const int flags = sp->flags;
    const bool upd_obj = flags & PHB_FLAG_UPDATE_OBJECT, upd_probe = flags & PHB_FLAG_UPDATE_PROBE;
    GroupArgs a = make_args(e, w, mode, flags, group, B);
    a.errors = sp->errors;
    a.beta_object = sp->beta_object;
    if (mode == MODE_LSQML) {
        if (!upd_obj && !e->new_probe_mag) a.illum = nullptr;
        if (upd_probe || e->new_obj_mag) {
            if ((rc = record_cuda(cudaMemsetAsync(w.gom, 0, (size_t)N * N * sizeof(float), st)))) return rc;
            k_gom<N><<<dim3((N * N + 255) / 256, 8), 256, 0, st>>>(a, w.gom);
            if ((rc = check_launch())) return rc;
        }
    } else {
        a.illum = nullptr;
    }
    if (mode == MODE_GRAD) a.acc_obj = (float2 *)sp->grad_object;
    a.group_patterns = sp->group_patterns;
    if (sp->event_begin && (rc = record_cuda(cudaEventRecord((cudaEvent_t)sp->event_begin, st)))) return rc;
    if ((rc = launch_group<N>(a, st))) return rc;
    if (sp->event_end && (rc = record_cuda(cudaEventRecord((cudaEvent_t)sp->event_end, st)))) return rc;

    FinArgs f{};
    f.mode = mode;
    f.flags = flags;
    f.S = e->S;
    f.M = e->M;
    f.B = B;
    f.B_max = e->B_max;
    f.beta_object = sp->beta_object;
    f.beta_probe = sp->beta_probe;
    f.gamma = sp->gamma;
    f.group = group;
    f.sums = w.sums;
    f.coef = w.coef;
    f.pos_update = sp->pos_update;
    f.grad_pos = sp->grad_pos;
    f.loss = sp->loss;
    k_finalize<<<1, 256, 0, st>>>(f);
    if ((rc = check_launch())) return rc;

    if (mode != MODE_GRAD && (upd_obj || a.illum)) {
        ObjApplyArgs o{};
        o.mode = mode;
        o.S = e->S;
        o.HW = e->H * e->W;
        o.reg = sp->illum_reg_object;
        o.eps = 1e-16f;
        o.object = (float2 *)e->object;
        o.acc = w.acc_obj;
        o.illum = a.illum;
        o.new_probe_mag = e->new_probe_mag;
        o.coef = w.coef;
        o.status = sp->status;
        o.group_index = sp->group_index;
        o.update = upd_obj;
        const int64_t total = (int64_t)e->S * e->H * e->W;
        int64_t g = (total + 255) / 256;
        if (g > 148 * 16) g = 148 * 16;
        k_obj_apply<<<(unsigned)g, 256, 0, st>>>(o);
        if ((rc = check_launch())) return rc;
    }
    if (upd_probe || (mode == MODE_LSQML && e->new_obj_mag)) {
        ProbeApplyArgs p{};
        p.mode = mode;
        p.M = e->M;
        p.B = B;
        p.S = e->S;
        p.reg = sp->illum_reg_probe;
        p.eps = 1e-16f;
        p.probe = (float2 *)e->probe;
        p.probe_k = w.probe_k;
        p.acc = w.acc_probe;
        p.gom = (mode == MODE_LSQML) ? w.gom : nullptr;
        p.new_obj_mag = (mode == MODE_LSQML) ? e->new_obj_mag : nullptr;
        p.coef = w.coef;
        p.beta_probe = sp->beta_probe;
        p.grad_probe = (float2 *)sp->grad_probe;
        p.status = sp->status;
        p.group_index = sp->group_index;
        p.update = upd_probe;
        if (mode == MODE_GRAD && !sp->grad_probe) p.update = 0;
        k_probe_apply<N><<<e->M, FFT_THREADS, fft_smem_bytes<N>(), st>>>(p);
        if ((rc = check_launch())) return rc;
    }
    return PHB_OK;
}

}  // namespace phb

using namespace phb;

extern "C" {

size_t phb_engine_workspace_bytes(int32_t N, int32_t M, int32_t S, int32_t B_max, int64_t H, int64_t W) {
    if (N <= 0 || M <= 0 || S <= 0 || B_max <= 0 || H <= 0 || W <= 0) return 0;
    return carve(nullptr, N, M, S, B_max, H, W).bytes;
}

int phb_engine_init(const phb_engine *e, void *stream) {
    int rc = validate(e);
    if (rc) return rc;
    return e->N == 128 ? engine_init<128>(e, (cudaStream_t)stream) : engine_init<64>(e, (cudaStream_t)stream);
}

int phb_engine_probe_changed(const phb_engine *e, void *stream) {
    int rc = validate(e);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    if (e->N == 128) {
        if ((rc = configure_kernels<128>())) return rc;
        return probe_spectrum<128>(e, carve(e->workspace, 128, e->M, e->S, e->B_max, e->H, e->W), st);
    }
    if ((rc = configure_kernels<64>())) return rc;
    return probe_spectrum<64>(e, carve(e->workspace, 64, e->M, e->S, e->B_max, e->H, e->W), st);
}

int phb_presolve_group(const phb_engine *e, const int64_t *group, int32_t B, int32_t solver, int32_t gradient_form,
                       double *rescale_num, double *rescale_den, void *stream) {
    int rc = validate(e);
    if (rc) return rc;
    if (!group || !rescale_num || !rescale_den || B < 1 || B > e->B_max) return PHB_ERR_INVALID_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    return e->N == 128 ? presolve<128>(e, group, B, solver, gradient_form, rescale_num, rescale_den, st)
                       : presolve<64>(e, group, B, solver, gradient_form, rescale_num, rescale_den, st);
}

int phb_simulate_group(const phb_engine *e, const int64_t *group, int32_t B, float *intensity, void *stream) {
    int rc = validate(e);
    if (rc) return rc;
    if (!group || !intensity || B < 1 || B > e->B_max) return PHB_ERR_INVALID_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    return e->N == 128 ? simulate<128>(e, group, B, intensity, st) : simulate<64>(e, group, B, intensity, st);
}

int phb_solver_group(const phb_engine *e, const phb_step *st, const int64_t *group, int32_t B, void *stream) {
    int rc = validate(e);
    if (rc) return rc;
    if (!st || !group || B < 1 || B > e->B_max) return PHB_ERR_INVALID_ARG;
    if (st->solver < PHB_SOLVER_LSQML || st->solver > PHB_SOLVER_GRAD) return PHB_ERR_INVALID_ARG;
    if (st->solver != PHB_SOLVER_GRAD && e->noise == PHB_NOISE_POISSON) return PHB_ERR_UNSUPPORTED;
    if (st->solver == PHB_SOLVER_GRAD && (st->flags & PHB_FLAG_UPDATE_OBJECT) && !st->grad_object)
        return PHB_ERR_INVALID_ARG;
    if ((st->flags & PHB_FLAG_UPDATE_POSITION) && st->solver != PHB_SOLVER_GRAD && !st->pos_update)
        return PHB_ERR_INVALID_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    return e->N == 128 ? solver_group<128>(e, st, group, B, s) : solver_group<64>(e, st, group, B, s);
}

int phb_position_update(float *scan, float *pos_update, float *momentum_state, int64_t n_pos, int32_t use_momentum,
                        float step_size, float max_step, float momentum, double obj_min_y, double obj_min_x,
                        double obj_max_y, double obj_max_x, int32_t *n_outside, void *stream) {
    if (!scan || !pos_update || !n_outside || n_pos < 1) return PHB_ERR_INVALID_ARG;
    if (use_momentum && !momentum_state) return PHB_ERR_INVALID_ARG;
    k_position_update<<<1, 1024, 0, (cudaStream_t)stream>>>(scan, pos_update, momentum_state, n_pos, use_momentum,
                                                            step_size, max_step, momentum, obj_min_y, obj_min_x,
                                                            obj_max_y, obj_max_x, n_outside);
    return check_launch();
}

int phb_iteration_reset(int32_t *status, float *errors, int64_t n, void *stream) {
    if (!status || (!errors && n > 0) || n < 0) return PHB_ERR_INVALID_ARG;
    int64_t g = (n + 255) / 256;
    if (g < 1) g = 1;
    if (g > 148 * 4) g = 148 * 4;
    k_iteration_reset<<<(unsigned)g, 256, 0, (cudaStream_t)stream>>>(status, errors, n);
    return check_launch();
}

int phb_iteration_report(const int32_t *status, const int32_t *n_outside, const float *errors, int64_t n,
                         double *out, void *stream) {
    if (!status || !errors || !out || n < 0) return PHB_ERR_INVALID_ARG;
    k_iteration_report<<<1, 1024, 0, (cudaStream_t)stream>>>(status, n_outside, errors, n, out);
    return check_launch();
}

int phb_nanmean(const float *values, int64_t n, double *out, int64_t *count, void *stream) {
    if (!values || !out || n < 0) return PHB_ERR_INVALID_ARG;
    k_nanmean<<<1, 1024, 0, (cudaStream_t)stream>>>(values, n, out, count);
    return check_launch();
}

int phb_check_finite_c64(const void *arr, int64_t n, int32_t *status, int32_t code, void *stream) {
    if (!arr || !status || n < 0) return PHB_ERR_INVALID_ARG;
    if (n == 0) return PHB_OK;
    int64_t g = (n + 255) / 256;
    if (g > 148 * 16) g = 148 * 16;
    k_check_finite<<<(unsigned)g, 256, 0, (cudaStream_t)stream>>>((const float2 *)arr, n, status, code);
    return check_launch();
}

}  // extern "C"
