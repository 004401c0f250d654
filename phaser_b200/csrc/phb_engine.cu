// The fused multislice mini-batch step of the LSQ-ML / ePIE / gradient engines.
//
// Reference algorithm: phaser/engines/conventional/solvers.py:132-504 (lsqml_dry_run,
// lsqml_run, epie_dry_run, epie_run), phaser/engines/gradient/run.py:357-438
// (run_model under jax.value_and_grad, dry_run), built from
// phaser/engines/common/simulation.py:160-306 and phaser/utils/object.py.
//
// Design (sm_100a):
//  * one CTA of 512 threads per (position b, probe mode m); each CTA keeps its
//    N x N wavefield in registers for the whole forward and adjoint pass
//    (phb_fft.cuh), multiplying cutouts and propagators in as it goes; only the
//    per-slice incident waves travel to HBM (for the adjoint) -- the minimum
//    traffic of the algorithm;
//  * the modes of a position meet only at the detector (the intensity is their
//    sum).  LSQ-ML and the gradient engine split the step there into two launches:
//    the forward launch stores Psi_m = fft2(exit wave) / N and adds |Psi_m / N|^2
//    into a per-position intensity buffer with float32 atomics; the second launch
//    resumes at the detector with the summed intensity and runs the constraint and
//    the adjoint.  The CTAs of a launch are independent, so they run without
//    clusters on every SM (4-CTA clusters of these 157 KB CTAs placed only 33 clusters,
//    132 of the 148 SMs).  ePIE keeps the M CTAs of a position in one cluster: its far
//    field and its per-slice maximum over the modes go through distributed shared
//    memory;
//  * object / probe updates are accumulated during the pass and applied by
//    small follow-up kernels once the group-global step sizes are known
//    (the reference applies them slice by slice, but its cutouts are copies
//    taken before the backward pass, so deferring is exact);
//  * step-size numerators / denominators and the position-gradient sums are
//    accumulated in float64 (block reduce, then one float64 atomic per CTA);
//  * N = 256: a tile needs four SMs (512 KB of complex64), so a cluster of 4 CTAs
//    holds one (position, mode), one 128 x 128 polyphase part each in real space and
//    a quarter of the spectrum in Fourier space (the 4-CTA transform of phb_fft.cuh),
//    with the same two-launch far field.  The gradient engine's position gradient
//    needs no step-size denominator, so it is formed from the probe-gradient spectrum
//    by Parseval (PH_PROBE) instead of by two more transforms.
#include <cooperative_groups.h>

#include "phb_fft.cuh"
#include "phb_runtime.h"

namespace cg = cooperative_groups;

// Elements of a thread's 32 whose global loads (object cutout, stored wavefield) are
// issued together in the incident-wave and adjoint loops of the fused kernel (a build-time
// tuning constant: more loads in flight, more registers).
#ifndef PHB_START_CHUNK
#define PHB_START_CHUNK 8
#endif
#ifndef PHB_BACK_CHUNK
#define PHB_BACK_CHUNK 8
#endif
// 1: prefetch part of the next phase's object cutout into L1 during the inverse transform
// (measured +0.65% on the 128^2 x 4-mode LSQ-ML step; 0 builds the kernel without it)
#ifndef PHB_L1_PREFETCH
#define PHB_L1_PREFETCH 1
#endif

namespace phb {

// Optional per-phase cycle accounting of the fused kernel (off unless the
// library is built with -DPHB_PHASE_TIMING; then phb_debug_phase_cycles reads it).
#ifdef PHB_PHASE_TIMING
__device__ unsigned long long g_phase_cycles[16];
#define PHB_T_BEGIN() long long phb_t0_ = clock64()
#define PHB_T_MARK(k)                                                                               \
    do {                                                                                            \
        const long long phb_t1_ = clock64();                                                        \
        if (threadIdx.x == 0) atomicAdd(&g_phase_cycles[(k)], (unsigned long long)(phb_t1_ - phb_t0_)); \
        phb_t0_ = phb_t1_;                                                                          \
    } while (0)
#else
#define PHB_T_BEGIN() (void)0
#define PHB_T_MARK(k) (void)0
#endif

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
    float2 *prop1d;     // max(S-1,1) * 2N: per slice gap, propagator factors p(ky) then p(kx)
    uint32_t *band;     // N*N/32 band-limit bits (propagator support)
    float *mask_k;      // N*N (K order)
    int32_t *info;      // [0] pattern mask is all ones, [1] propagators separable, [2] max deviation (float bits)
    double *sums;       // float64 accumulators, see SumIdx
    double *coef;       // S + M step coefficients
    float2 *far;        // B_max * M * N*N far-field waves Psi_m / N (register order)
    float *far_int;     // B_max * N*N far-field intensity sum_m |Psi_m / N|^2 (register order)
    size_t bytes;
};

struct SumIdx {
    int64_t numO, denO, numP, denP, pnum, pden, pnorm, loss, tilt, err, total;
    __host__ __device__ SumIdx(int B, int S, int M) {
        numO = 0;
        denO = numO + (int64_t)B * S;
        numP = denO + S;
        denP = numP + (int64_t)B * M;
        pnum = denP + 1;
        pden = pnum + 2 * (int64_t)B;
        pnorm = pden + 2 * (int64_t)B;
        loss = pnorm + B;
        tilt = loss + B;
        err = tilt + 2 * (int64_t)B;      // N = 256: per-position squared detector error
        total = err + B;
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
    w.prop1d = (float2 *)take((size_t)(S > 1 ? S - 1 : 1) * 2 * N * sizeof(float2));
    w.band = (uint32_t *)take(NN / 32 * sizeof(uint32_t));
    w.mask_k = (float *)take(NN * sizeof(float));
    w.info = (int32_t *)take(4 * sizeof(int32_t));
    w.sums = (double *)take((size_t)SumIdx(B, S, M).total * sizeof(double));
    w.coef = (double *)take((size_t)(S + M + 4) * sizeof(double));
    w.far = (float2 *)take((size_t)B * M * NN * sizeof(float2));
    w.far_int = (float *)take((size_t)B * NN * sizeof(float));
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
    const float2 *prop1d, *probe_k;
    const uint32_t *band;
    const int32_t *info;   // device: [0] mask is all ones
    int32_t *err_word;     // device: set to 1 if a kernel ran past its bounded program
    int32_t *status;       // optional sticky status of the step (see phb_step.status)
    int32_t group_index;
    // float64 accumulator offsets (SumIdx for B_max), precomputed on the host
    int64_t o_numO, o_denO, o_numP, o_denP, o_pnum, o_pden, o_pnorm, o_loss, o_tilt, o_err;
    const float *fy, *fx;
    float2 *psi, *acc_obj, *acc_probe;
    float *illum;
    double *sums;
    float *errors;
    double *pre_num, *pre_den;
    float *sim_out;
    const float *group_patterns;
    const uint16_t *patterns16;   // resident uint16 counts (patterns == nullptr then)
    float2 *far;                  // far-field waves (see Workspace)
    float *far_int;               // far-field intensity
    int resume;                   // 0 = forward launch, 1 = launch resumed at the detector
};

// One position's measured pattern: host-streamed float32 rows (group_patterns),
// resident float32, or resident uint16 counts converted exactly to float32.
struct PatRow {
    const float *f;
    const uint16_t *h;
    __device__ __forceinline__ PatRow(const GroupArgs &a, int64_t pos, int b, int64_t NN) {
        if (a.group_patterns) {
            f = a.group_patterns + (size_t)b * NN;
            h = nullptr;
        } else if (a.patterns16) {
            f = nullptr;
            h = a.patterns16 + pos * NN;
        } else {
            f = a.patterns + pos * NN;
            h = nullptr;
        }
    }
    __device__ __forceinline__ float at(int64_t i) const { return h ? (float)__ldg(h + i) : __ldg(f + i); }
};

template <int N>
__device__ __forceinline__ float2 obj_px(const float2 *Os, const CutoutIndex &ci, int64_t H, int64_t W, int r,
                                         int c) {
    const int64_t y = ci.y0 + r, x = ci.x0 + c;
    return (y >= 0 && y < H && x >= 0 && x < W) ? __ldg(Os + y * W + x) : make_float2(1.f, 0.f);
}

// Per-thread view of one position's cutout in R layout: row base offsets and a
// validity bit per register slot (identical for every slice).
template <int N>
struct CutView {
    int32_t base[FFTCfg<N>::U];   // (y0 + row(u, 0)) * W + x0 + col(u, 0), inside one slice (H*W < 2^31)
    int32_t w;                    // object row length W
    uint64_t valid;               // bit u*E + q: pixel (row(u, q), col(u, q)) inside the object
    static_assert(FFTCfg<N>::U * FFTCfg<N>::E <= 64, "per-thread slot bits must fit 64 bits");
    __device__ __forceinline__ void init(const CutoutIndex &ci, int64_t H, int64_t W) {
        using I = Idx<N>;
        valid = 0ull;
        w = (int32_t)W;
#pragma unroll
        for (int u = 0; u < I::U; ++u) {
            base[u] = (int32_t)((ci.y0 + I::row(u, 0)) * W + ci.x0 + I::col(u, 0));
#pragma unroll
            for (int q = 0; q < I::E; ++q) {
                const int64_t y = ci.y0 + I::row(u, q), x = ci.x0 + I::col(u, q);
                if (y >= 0 && y < H && x >= 0 && x < W) valid |= 1ull << (u * I::E + q);
            }
        }
    }
    __device__ __forceinline__ bool ok(int u, int q) const { return (valid >> (u * FFTCfg<N>::E + q)) & 1ull; }
    // offset of pixel (row(u, q), col(u, q)) inside one object slice (valid only if ok(u, q))
    __device__ __forceinline__ int32_t off(int u, int q) const {
        return base[u] + Idx<N>::drow(q) * w + Idx<N>::dcol(q);
    }
    __device__ __forceinline__ float2 at(const float2 *Os, int u, int q) const {
        return (valid >> (u * FFTCfg<N>::E + q)) & 1ull ? __ldg(Os + off(u, q)) : make_float2(1.f, 0.f);
    }
};

// Phases of the fused mini-batch program.  Each is the elementwise work that
// follows one transform (R = real-space layout after an inverse transform,
// K = Fourier layout after a forward transform).  The kernel body contains
// exactly one forward and one inverse 2D FFT, so the instruction footprint
// stays small however many slices the program walks through.
enum Phase : int {
    PH_START = 0,   // R: incident wave of slice s: store, illuminate, transmit
    PH_PROP = 1,    // K: propagate to slice s+1
    PH_FAR = 2,     // K: detector plane, constraint / loss gradient
    PH_BACK = 3,    // R: adjoint of slice s (object/probe update terms)
    PH_BPROP = 4,   // K: adjoint propagation to slice s-1
    PH_PROBE = 5,   // K: probe-update accumulation
    PH_POS = 6,     // R: position-gradient dot products (direction `dir`)
    PH_TILT = 7,    // K: tilt-gradient dot products of gap s-1 (gradient engine), then BPROP
};

// MC > 0: the number of probe modes (cluster size) is the compile-time constant MC,
// so every cross-mode loop unrolls and its remote loads issue back to back;
// MC == 0 handles any M at run time.
template <int N, int MODE, int MC>
__global__ void __launch_bounds__(FFT_THREADS, 1) k_group(const GroupArgs a) {
    using I = Idx<N>;
    constexpr int U = I::U, E = I::E, NN = N * N, SLOTS = U * E;
    constexpr int mode = MODE;
    constexpr int MR = MC > 0 ? MC : 8;   // capacity of the remote-pointer arrays
    constexpr bool presolve = mode >= MODE_PRE_LSQML;
    constexpr bool lsqml = mode == MODE_LSQML, epie = mode == MODE_EPIE, grad = mode == MODE_GRAD;
    constexpr bool QUAD = N == 256;   // 4 CTAs per (position, mode)
    // Far field through global memory (two launches): the modes of a position are then
    // independent CTAs, launched without clusters, and every SM takes work (4-CTA clusters
    // occupied only 132 of the 148 SMs).  ePIE keeps its modes in one cluster: its
    // per-slice maximum over the modes goes through distributed shared memory.
    constexpr bool SPLIT = mode != MODE_EPIE;
    static_assert(!QUAD || (mode != MODE_EPIE && mode != MODE_PRE_EPIE), "ePIE needs the modes in one cluster");
    cg::cluster_group cl = cg::this_cluster();
    const int M = MC > 0 ? MC : a.M;
    const int S = a.S;
    const int m = QUAD ? (int)((blockIdx.x >> 2) % M) : SPLIT ? (int)(blockIdx.x % M) : (int)cl.block_rank();
    const int b = QUAD ? (int)((blockIdx.x >> 2) / M) : (int)(blockIdx.x / M);
    const int tid = threadIdx.x;
    const bool resume = SPLIT && a.resume;

    extern __shared__ float4 smem_raw[];
    float2 *xb = reinterpret_cast<float2 *>(smem_raw);
    float2 *twid = xb + Lay<N>::BUF;
    float2 *hy = twid + TileCfg<N>::TW, *hx = hy + N;   // sub-pixel shift filter factors
    float2 *py = hx + N, *px = py + N;             // propagator factors of the current slice gap
    double *dred = reinterpret_cast<double *>(px + N);
    float *fred = reinterpret_cast<float *>(dred + 64);              // [0..31] block scratch, [32] cluster slot
    uint32_t *band = reinterpret_cast<uint32_t *>(fred + 64);        // N*N/32 band-limit bits
    // per-thread cutout view and band bits live in shared memory between phases,
    // leaving the registers to the wavefield while the transforms run
    uint64_t *s_bits = reinterpret_cast<uint64_t *>(band + NN / 32);   // [valid | kband][FFT_THREADS]
    int32_t *s_base = reinterpret_cast<int32_t *>(s_bits + 2 * FFT_THREADS);   // [U][FFT_THREADS]

    const bool upd_obj = !presolve && (a.flags & PHB_FLAG_UPDATE_OBJECT);
    const bool upd_probe = !presolve && (a.flags & PHB_FLAG_UPDATE_PROBE);
    const bool upd_pos = !presolve && (a.flags & PHB_FLAG_UPDATE_POSITION);
    const bool upd_tilt = grad && (a.flags & PHB_FLAG_UPDATE_TILT) && a.tilt != nullptr;
    const bool calc_err = !presolve && !grad && (a.flags & PHB_FLAG_CALC_ERROR) && a.errors;
    const bool do_illum = a.illum && (mode == MODE_LSQML || mode == MODE_PRE_LSQML);
    const bool tilted = a.tilt != nullptr;
    const bool mask_ones = __ldg(a.info) != 0;
    double *sums = a.sums;

    const int64_t pos = a.group[b];
#if PHB_BOUNDS_CHECK
    // before any barrier and any access through pos; every CTA of a cluster has the same
    // position, so a cluster returns whole and none of its CTAs waits on another
    if (!pos_ok(pos, a.n_pos)) {
        if (tid == 0) report_bounds(a.err_word, a.status, a.group_index);
        return;
    }
#endif
    const CutoutIndex ci = cutout_index(a.scan, pos, a.cy, a.cx, a.sy, a.sx, N, N);
    {
        CutView<N> c0;
        c0.init(ci, a.H, a.W);
        s_bits[tid] = c0.valid;
#pragma unroll
        for (int u = 0; u < U; ++u) s_base[u * FFT_THREADS + tid] = c0.base[u];
    }
    auto load_cv = [&]() {
        CutView<N> c;
        c.valid = s_bits[tid];
#pragma unroll
        for (int u = 0; u < U; ++u) c.base[u] = s_base[u * FFT_THREADS + tid];
        c.w = (int32_t)a.W;
        return c;
    };

    fft_init_twiddles<N>(twid);
    for (int k = tid; k < N; k += blockDim.x) {
        float sn, cs;
        sincospif(-2.0f * (ci.sy * a.fy[k]), &sn, &cs);
        hy[k] = make_float2(cs, sn);
        sincospif(-2.0f * (ci.sx * a.fx[k]), &sn, &cs);
        hx[k] = make_float2(cs, sn);
    }
    for (int k = tid; k < NN / 32; k += blockDim.x) band[k] = a.band[k];
    __syncthreads();

    float2 *psi_b = a.psi + (size_t)(b * M + m) * S * NN;
    const int slot0 = (m * SLOTS) / M, slot1 = ((m + 1) * SLOTS) / M;
    const float inv_n = 1.0f / (float)N, inv_nn = 1.0f / (float)NN;

    float2 v[U][E];
    // propagator of slice gap g (and this position's tilt ramp) into py/px; px carries the
    // 1/N^2 of the unnormalised transform pair, so the propagation multiply needs no scaling
    auto load_prop = [&](int g) {
        const float2 *src = a.prop1d + (size_t)g * 2 * N;
        for (int k = tid; k < 2 * N; k += blockDim.x) {
            float2 p = src[k];
            if (tilted) {
                const float dz = a.thick[g];
                const float t = tanf(a.tilt[2 * pos + (k < N ? 0 : 1)] * 1e-3f);
                const float f = k < N ? a.fy[k] : a.fx[k - N];
                float sn, cs;
                sincospif(2.0f * (dz * (t * f)), &sn, &cs);
                p = cmul(p, make_float2(cs, sn));
            }
            py[k] = k < N ? p : cscale(p, inv_nn);   // py[0..N) then px[0..N): contiguous
        }
        __syncthreads();
    };
    // band-limit bits of this thread's K-layout elements (same for every slice gap)
    {
        uint64_t kb = 0ull;
        static_assert(U * E <= 64, "per-thread slot bits must fit 64 bits");
#pragma unroll
        for (int u = 0; u < U; ++u)
#pragma unroll
            for (int e = 0; e < E; ++e) {
                const int f = I::ky(u, e) * N + I::kx(u, e);
                if ((band[f >> 5] >> (f & 31)) & 1u) kb |= 1ull << (u * E + e);
            }
        s_bits[FFT_THREADS + tid] = kb;
    }
    // v (K layout) = DFT(P_m)/N^2 * H_b [* (-2 pi i k_dir)]
    auto load_probe_spectrum = [&](int dir) {
        const float2 *pk = a.probe_k + (size_t)m * NN;
        const float twopi = 6.283185307179586f;
#pragma unroll
        for (int u = 0; u < U; ++u)
#pragma unroll
            for (int e = 0; e < E; ++e) {
                const int ky = I::ky(u, e), kx = I::kx(u, e);
                float2 g = cmul(__ldg(pk + I::flat(u, e)), cmul(hy[ky], hx[kx]));
                if (dir >= 0) {
                    const float w = twopi * (dir == 0 ? a.fy[ky] : a.fx[kx]);
                    g = make_float2(w * g.y, -w * g.x);
                }
                v[u][e] = g;
            }
    };

    int phase = PH_START, s = 0, dir = 0;
    bool fwd = false;
    if (resume) {
        // second launch at N = 256: the far-field wave stored by the forward launch
        const float2 *src = a.far + (size_t)(b * M + m) * NN;
#pragma unroll
        for (int u = 0; u < U; ++u)
#pragma unroll
            for (int e = 0; e < E; ++e) v[u][e] = src[I::flat(u, e)];
        phase = PH_FAR;
    } else {
        load_probe_spectrum(-1);
    }

    // The program is 4 S + 2 transforms at most (forward, adjoint, probe, two
    // position directions); the bound turns a logic error into a recorded error
    // (info[3] and the step's status word) instead of a kernel that never ends.
    const int max_steps = 5 * S + 8;
    PHB_T_BEGIN();
    for (int step = 0;; ++step) {
        if (step >= max_steps) {
            if (tid == 0) {
                atomicExch(a.err_word, 1);
                if (a.status) atomicCAS(a.status, -1, PHB_STATUS_INTERNAL | a.group_index);
            }
            return;
        }
        if (!(resume && step == 0)) {
#if PHB_L1_PREFETCH
            // the phase after this inverse transform reads the object cutout of slice s:
            // pull the first half of this warp's rows into L1 while the transform runs
            // (a warp's elements 0..15 span 8 rows x 2 column blocks of 32 pixels: one
            // 128-byte line per lane)
            if (!fwd && (phase == PH_START || phase == PH_BACK) && N == 128) {
                const int l = tid & 31, row = I::row(0, 0) + 16 * (l >> 2), col = I::col(0, 0) - (tid & 31) +
                                                                                     32 * ((l >> 1) & 1) + 16 * (l & 1);
                const int64_t y = ci.y0 + row, x = ci.x0 + col;
                if (y >= 0 && y < a.H && x >= 0 && x + 15 < a.W)
                    asm volatile("prefetch.global.L1 [%0];" ::"l"(a.object + ((size_t)s * a.H + y) * a.W + x));
            }
#endif
            if (fwd) fft2_r2k<N>(v, xb, twid);
            else ifft2_k2r<N>(v, xb, twid);
        }
        PHB_T_MARK(fwd ? 0 : 1);
        const int timed_phase = phase;

        if (phase == PH_START) {
            // ------------------------------------------- incident wave of slice s (R layout)
            const CutView<N> cv = load_cv();
            const float2 *Os = a.object + (size_t)s * a.H * a.W;
            if (s == 0 && upd_pos && !grad) {
                float n0 = 0.f;
#pragma unroll
                for (int u = 0; u < U; ++u)
#pragma unroll
                    for (int q = 0; q < E; ++q) n0 += cabs2(v[u][q]);
                warp_atomic_sum(sums + a.o_pnorm + b, (double)n0);
            }
            if constexpr (!presolve) {
                // one chunked pass: the object loads of a chunk are issued first, then the
                // wavefield store (for the adjoint; the tilt gradient transforms it), the
                // illumination scatter group_probe_mag[s] += |psi_s,m|^2 and the transmission
                const bool store = upd_obj || upd_tilt;
                float2 *dst = psi_b + (size_t)s * NN;
                float *ill = do_illum ? a.illum + (size_t)s * a.H * a.W : nullptr;
                constexpr int CH = PHB_START_CHUNK < E ? PHB_START_CHUNK : E;
#pragma unroll
                for (int u = 0; u < U; ++u)
#pragma unroll
                    for (int q0 = 0; q0 < E; q0 += CH) {
                        float2 oo[CH];
#pragma unroll
                        for (int j = 0; j < CH; ++j) oo[j] = cv.at(Os, u, q0 + j);
#pragma unroll
                        for (int j = 0; j < CH; ++j) {
                            const int q = q0 + j;
                            if (store) dst[I::flat(u, q)] = v[u][q];
                            if (ill && cv.ok(u, q)) atomicAdd(ill + cv.off(u, q), cabs2(v[u][q]));
                            v[u][q] = cmul(v[u][q], oo[j]);
                        }
                    }
                PHB_T_MARK(11);
                if (s != S - 1) load_prop(s);
                fwd = true;
                phase = s == S - 1 ? PH_FAR : PH_PROP;
            } else {
            if (do_illum) {   // group_probe_mag[s] += scatter(|psi_s,m|^2): one red per pixel and mode
                float *dst = a.illum + (size_t)s * a.H * a.W;
#pragma unroll
                for (int u = 0; u < U; ++u)
#pragma unroll
                    for (int q = 0; q < E; ++q)
                        if (cv.ok(u, q)) atomicAdd(dst + cv.off(u, q), cabs2(v[u][q]));
            }
            PHB_T_MARK(11);
            const bool last = s == S - 1;
            if constexpr (mode == MODE_PRE_LSQML || mode == MODE_PRE_EPIE) {
                if (last) {   // rescale: sum(I_exp*mask) / sum|psi_last|^2 (Parseval), before transmission
                    double t[2] = {0.0, 0.0};
#pragma unroll
                    for (int u = 0; u < U; ++u)
#pragma unroll
                        for (int q = 0; q < E; ++q) t[0] += (double)cabs2(v[u][q]);
                    if (m == 0) {
                        const PatRow pat(a, pos, b, NN);
                        const int f0 = QUAD ? (cluster_rank() << 14) : 0, f1 = QUAD ? f0 + NN / 4 : NN;
                        for (int f = f0 + tid; f < f1; f += FFT_THREADS) {
                            int ky, kx;
                            flat_to_k<N>(f, ky, kx);
                            t[1] += (double)(pat.at(ky * N + kx) * __ldg(a.mask_k + f));
                        }
                    }
                    block_sum_doubles<FFT_THREADS>(t, 2, dred);
                    if (tid == 0) {
                        atomicAdd(a.pre_den + b, t[0]);
                        if (m == 0) atomicAdd(a.pre_num + b, t[1]);
                    }
                    return;
                }
            }
#pragma unroll
            for (int u = 0; u < U; ++u)
#pragma unroll
                for (int q = 0; q < E; ++q) v[u][q] = cmul(v[u][q], cv.at(Os, u, q));
            if constexpr (mode == MODE_PRE_GRAD) {
                if (last) {
                    double t[2] = {0.0, 0.0};
#pragma unroll
                    for (int u = 0; u < U; ++u)
#pragma unroll
                        for (int q = 0; q < E; ++q) t[0] += (double)cabs2(v[u][q]);
                    if (m == 0) {
                        const PatRow pat(a, pos, b, NN);
                        const int f0 = QUAD ? (cluster_rank() << 14) : 0, f1 = QUAD ? f0 + NN / 4 : NN;
                        for (int f = f0 + tid; f < f1; f += FFT_THREADS) t[1] += (double)pat.at(f);
                    }
                    block_sum_doubles<FFT_THREADS>(t, 2, dred);
                    if (tid == 0) {
                        atomicAdd(a.pre_den + b, t[0]);
                        if (m == 0) atomicAdd(a.pre_num + b, t[1]);
                    }
                    return;
                }
            }
            if (!last) load_prop(s);
            fwd = true;
            phase = last ? PH_FAR : PH_PROP;
            }
        } else if (phase == PH_PROP) {
            // ------------------------------------------- propagate (K layout)
            const uint64_t kband = s_bits[FFT_THREADS + tid];
#pragma unroll
            for (int u = 0; u < U; ++u)
#pragma unroll
                for (int e = 0; e < E; ++e) {
                    const int ky = I::ky(u, e), kx = I::kx(u, e);
                    const float2 p = ((kband >> (u * E + e)) & 1ull) ? cmul(py[ky], px[kx]) : make_float2(0.f, 0.f);
                    v[u][e] = cmul(v[u][e], p);
                }
            fwd = false;
            phase = PH_START;
            ++s;
        } else if (phase == PH_FAR) {
            // ------------------------------------------- detector: Psi = fft2(exit), constraint
            float *xf = reinterpret_cast<float *>(xb);
            const float *rxf[MR];
            if constexpr (SPLIT) {
                if (!resume) {
                    // the forward launch ends at the detector: store Psi_m / N and add |Psi_m / N|^2
                    // into the position's intensity (or, simulating, into the output pattern)
                    float2 *dst = a.far + (size_t)(b * M + m) * NN;
                    float *itn = a.far_int + (size_t)b * NN;
#pragma unroll
                    for (int u = 0; u < U; ++u)
#pragma unroll
                        for (int e = 0; e < E; ++e) {
                            const float2 w = cscale(v[u][e], inv_n);
                            if constexpr (mode == MODE_SIM) {
                                atomicAdd(a.sim_out + (size_t)b * NN + I::ky(u, e) * N + I::kx(u, e), cabs2(w));
                            } else {
                                dst[I::flat(u, e)] = w;
                                atomicAdd(itn + I::flat(u, e), cabs2(w));
                            }
                        }
                    return;
                }
            } else {
#pragma unroll
                for (int u = 0; u < U; ++u)
#pragma unroll
                    for (int e = 0; e < E; ++e) {
                        v[u][e] = cscale(v[u][e], inv_n);
                        xf[I::flat(u, e)] = cabs2(v[u][e]);
                    }
                cl.sync();
                // the exchange buffer of every CTA of the cluster (distributed shared memory)
#pragma unroll
                for (int r = 0; r < MR; ++r) rxf[r] = r < M ? cl.map_shared_rank(xf, r) : xf;
            }
            if constexpr (mode == MODE_SIM && !SPLIT) {
                if (m == 0) {
#pragma unroll
                    for (int u = 0; u < U; ++u)
#pragma unroll
                        for (int e = 0; e < E; ++e) {
                            const int f = I::flat(u, e);
                            float inten = 0.f;
                            for (int r = 0; r < MR; ++r)
                                if (r < M) inten += rxf[r][f];
                            a.sim_out[(size_t)b * NN + I::ky(u, e) * N + I::kx(u, e)] = inten;
                        }
                }
                cl.sync();
                return;
            } else {
                const PatRow pat(a, pos, b, NN);
                double e2 = 0.0, loss = 0.0;
#pragma unroll
                for (int u = 0; u < U; ++u)
#pragma unroll
                    for (int e = 0; e < E; ++e) {
                        const int f = I::flat(u, e);
                        float inten = 0.f;
                        if constexpr (SPLIT) {
                            inten = __ldg(a.far_int + (size_t)b * NN + f);
                        } else {
                            for (int r = 0; r < MR; ++r)
                                if (r < M) inten += rxf[r][f];
                        }
                        const float pv = pat.at(I::ky(u, e) * N + I::kx(u, e));
                        const float mk = mask_ones ? 1.0f : __ldg(a.mask_k + f);
                        if (calc_err && m == 0) {
                            const float d = inten - pv;
                            if (d == d) e2 += (double)d * (double)d;
                        }
                        const float pm = np_max0(pv);
                        float fac;
                        if constexpr (!grad) {
                            // amplitude / anscombe wave update (noise_models.py:47-64)
                            fac = (sqrtf(pm + a.offset) / (sqrtf(inten + a.offset) + a.eps) - 1.0f) * mk;
                        } else {
                            if (a.noise == PHB_NOISE_POISSON) {
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
                        }
                        v[u][e] = cscale(v[u][e], fac);
                    }
                if constexpr (!SPLIT) cl.sync();
                if (m == 0 && (calc_err || grad)) {
                    double t[2] = {e2, loss};
                    block_sum_doubles<FFT_THREADS>(t, 2, dred);
                    if (tid == 0) {
                        if constexpr (SPLIT) {   // per-CTA partial sums: the finish kernel takes the root
                            if (calc_err) atomicAdd(sums + a.o_err + b, t[0]);
                            if (grad) atomicAdd(sums + a.o_loss + b, t[1]);
                        } else {
                            if (calc_err) a.errors[pos] = (float)sqrt(t[0]);
                            if (grad) sums[a.o_loss + b] = t[1];
                        }
                    }
                }
                fwd = false;
                phase = PH_BACK;
                s = S - 1;
            }
        } else if (phase == PH_BACK) {
            // ------------------------------------------- adjoint of slice s (R layout)
            const CutView<N> cv = load_cv();
            if (s == S - 1) {
#pragma unroll
                for (int u = 0; u < U; ++u)
#pragma unroll
                    for (int q = 0; q < E; ++q) v[u][q] = cscale(v[u][q], inv_n);   // chi = ifft2(.)
            }
            const float2 *Os = a.object + (size_t)s * a.H * a.W;
            float2 *ps = psi_b + (size_t)s * NN;
            if constexpr (!epie) {
                // LSQ-ML: dO = chi conj(psi), dP = chi conj(O) (solvers.py:242-271); gradient: same adjoint.
                // Each mode scatters its own dO (the sum over modes is linear).
                float t4[4] = {0.f, 0.f, 0.f, 0.f};   // per-thread partials, reduced in float64
                float2 *__restrict__ dst = a.acc_obj + (size_t)s * a.H * a.W;
                // chunks of 8 elements: issue all object / wavefield loads of a chunk before
                // its atomics, so they are in flight together
                constexpr int CH = PHB_BACK_CHUNK < E ? PHB_BACK_CHUNK : E;
#pragma unroll
                for (int u = 0; u < U; ++u)
#pragma unroll
                    for (int q0 = 0; q0 < E; q0 += CH) {
                        float2 oo[CH], pp[CH];
#pragma unroll
                        for (int j = 0; j < CH; ++j) {
                            oo[j] = cv.at(Os, u, q0 + j);
                            pp[j] = upd_obj ? ps[I::flat(u, q0 + j)] : make_float2(0.f, 0.f);
                        }
#pragma unroll
                        for (int j = 0; j < CH; ++j) {
                            const int q = q0 + j;
                            const int f = I::flat(u, q);
                            const float2 c = v[u][q];
                            const float2 o = oo[j];
                            const float c2 = cabs2(c);
                            if (upd_obj) {
                                const float2 p = pp[j];
                                if (cv.ok(u, q)) atomic_add_c(dst + cv.off(u, q), cmulc(c, p));
                                if (lsqml) {
                                    const float p2 = cabs2(p);
                                    t4[0] += c2 * p2;
                                    t4[1] += (c2 * p2) * p2;
                                }
                            }
                            if (s == 0) {
                                if (lsqml && upd_probe) {
                                    const float o2 = cabs2(o);
                                    t4[2] += c2 * o2;
                                    t4[3] += (c2 * o2) * o2;
                                }
                                if (upd_pos && !grad) ps[f] = c;   // exit-wave update of slice 0 for the position step
                            }
                            v[u][q] = cmulc(c, o);
                        }
                    }
                PHB_T_MARK(9);
                if (lsqml) {
                    if (upd_obj) {
                        warp_atomic_sum(sums + a.o_numO + (int64_t)b * S + s, (double)t4[0]);
                        warp_atomic_sum(sums + a.o_denO + s, (double)t4[1]);
                    }
                    if (s == 0 && upd_probe) {
                        warp_atomic_sum(sums + a.o_numP + (int64_t)b * M + m, (double)t4[2]);
                        warp_atomic_sum(sums + a.o_denP, (double)t4[3]);
                    }
                }
                PHB_T_MARK(10);
            } else {
                // ePIE: dP = conj(O) chi / max|O|^2; O += beta/S sum_m conj(psi) chi / max sum_m |psi|^2
                // (solvers.py:459-486)
                float omax = 0.f;
                float *xf = reinterpret_cast<float *>(xb);
#pragma unroll
                for (int u = 0; u < U; ++u)
#pragma unroll
                    for (int q = 0; q < E; ++q) {
                        omax = fmaxf(omax, cabs2(cv.at(Os, u, q)));
                        if (upd_obj) xf[I::flat(u, q)] = cabs2(ps[I::flat(u, q)]);
                    }
                omax = block_max_float<FFT_THREADS>(omax, fred);
                float scl = 0.f;
                if (upd_obj) {
                    cl.sync();
                    float lmax = 0.f;
                    for (int sl = slot0; sl < slot1; ++sl) {
                        const int f = sl * FFT_THREADS + tid;
                        float w = 0.f;
                        for (int r = 0; r < MR; ++r)
                            if (r < M) w += cl.map_shared_rank(xf, r)[f];
                        lmax = fmaxf(lmax, w);
                    }
                    lmax = block_max_float<FFT_THREADS>(lmax, fred);
                    // slot by slice parity: a rank may write the next slice's maximum while
                    // others still read this one (the exchange barrier orders slice s-2's reads)
                    const int slot = 32 + (s & 1);
                    if (tid == 0) fred[slot] = lmax;
                    cl.sync();
                    float wmax = 0.f;
                    for (int r = 0; r < M; ++r) wmax = fmaxf(wmax, cl.map_shared_rank(fred, r)[slot]);
                    // last remote access of the program: no rank may leave (and release its
                    // shared memory) before every rank has read the slice-0 maxima
                    if (s == 0) cl.sync();
                    scl = a.beta_object / (float)S / wmax;
                }
                // one pass: object update (atomics), exit-wave update and the next adjoint,
                // loads of a chunk issued together
                const float inv = 1.0f / omax;
                float2 *dst = a.acc_obj + (size_t)s * a.H * a.W;
                constexpr int CH = 8;
#pragma unroll
                for (int u = 0; u < U; ++u)
#pragma unroll
                    for (int q0 = 0; q0 < E; q0 += CH) {
                        float2 oo[CH], pp[CH];
#pragma unroll
                        for (int j = 0; j < CH; ++j) {
                            oo[j] = cv.at(Os, u, q0 + j);
                            pp[j] = upd_obj ? ps[I::flat(u, q0 + j)] : make_float2(0.f, 0.f);
                        }
#pragma unroll
                        for (int j = 0; j < CH; ++j) {
                            const int q = q0 + j;
                            const float2 c = v[u][q];
                            if (upd_obj && cv.ok(u, q)) atomic_add_c(dst + cv.off(u, q), cscale(cmulc(c, pp[j]), scl));
                            if (s == 0 && upd_pos) ps[I::flat(u, q)] = c;
                            v[u][q] = cscale(cmulc(c, oo[j]), inv);
                        }
                    }
            }
            if (s > 0) {
                // the adjoint of slice s-1 reads its stored incident wave after the next
                // transform pair: start moving it from HBM into L2 now
                if (upd_obj && tid == 0) {
                    if constexpr (QUAD)
                        prefetch_l2(psi_b + (size_t)(s - 1) * NN + ((size_t)cluster_rank() << 14),
                                    (NN / 4) * sizeof(float2));
                    else
                        prefetch_l2(psi_b + (size_t)(s - 1) * NN, NN * sizeof(float2));
                }
                load_prop(s - 1);
                fwd = true;
                phase = PH_BPROP;
            } else if (upd_probe || (grad && upd_pos)) {   // gradient engine: positions from this spectrum
                fwd = true;
                phase = PH_PROBE;
            } else if (upd_pos) {
                load_probe_spectrum(0);
                fwd = false;
                phase = PH_POS;
                dir = 0;
            } else {
                return;
            }
        } else if (grad && (phase == PH_TILT || (phase == PH_BPROP && upd_tilt))) {
            if (phase == PH_BPROP) {
                // tilt gradient of gap s-1 (gradient/run.py:357-400 through tilt_propagators,
                // engines/common/simulation.py:193-222): sum_k conj(G) Y 2 pi i dz k (1 + tan^2) 1e-3 / N^2
                // with G = FFT(adjoint of psi_s) (in v) and Y = FFT(psi_s).  Swap G into psi_s's
                // stack slot (no longer needed) and transform psi_s.
                float2 *slot = psi_b + (size_t)s * NN;
#pragma unroll
                for (int u = 0; u < U; ++u)
#pragma unroll
                    for (int e = 0; e < E; ++e) {
                        const int f = I::flat(u, e);
                        const float2 w = slot[f];
                        slot[f] = v[u][e];
                        v[u][e] = w;
                    }
                fwd = true;
                phase = PH_TILT;
                continue;
            }
            const float2 *slot = psi_b + (size_t)s * NN;
            double ty = 0.0, tx = 0.0;
#pragma unroll
            for (int u = 0; u < U; ++u)
#pragma unroll
                for (int e = 0; e < E; ++e) {
                    const float2 G = slot[I::flat(u, e)];
                    const float im = G.x * v[u][e].y - G.y * v[u][e].x;   // Im(conj(G) Y)
                    ty += (double)(im * a.fy[I::ky(u, e)]);
                    tx += (double)(im * a.fx[I::kx(u, e)]);
                    v[u][e] = G;
                }
            {
                const double dz = (double)a.thick[s - 1];
                const double t0 = tan((double)a.tilt[2 * pos] * 1e-3), t1 = tan((double)a.tilt[2 * pos + 1] * 1e-3);
                const double c = -2.0 * 3.141592653589793 * dz * 1e-3 / (double)NN;   // Re(i z) = -Im z
                warp_atomic_sum(sums + a.o_tilt + 2 * b, ty * c * (1.0 + t0 * t0));
                warp_atomic_sum(sums + a.o_tilt + 2 * b + 1, tx * c * (1.0 + t1 * t1));
            }
            const uint64_t kband = s_bits[FFT_THREADS + tid];
#pragma unroll
            for (int u = 0; u < U; ++u)
#pragma unroll
                for (int e = 0; e < E; ++e) {
                    const int ky = I::ky(u, e), kx = I::kx(u, e);
                    const float2 p = ((kband >> (u * E + e)) & 1ull) ? cmul(py[ky], px[kx]) : make_float2(0.f, 0.f);
                    v[u][e] = cmulc(v[u][e], p);
                }
            fwd = false;
            phase = PH_BACK;
            --s;
        } else if (phase == PH_BPROP) {
            // ------------------------------------------- adjoint propagation (K layout)
            const uint64_t kband = s_bits[FFT_THREADS + tid];
#pragma unroll
            for (int u = 0; u < U; ++u)
#pragma unroll
                for (int e = 0; e < E; ++e) {
                    const int ky = I::ky(u, e), kx = I::kx(u, e);
                    const float2 p = ((kband >> (u * E + e)) & 1ull) ? cmul(py[ky], px[kx]) : make_float2(0.f, 0.f);
                    v[u][e] = cmulc(v[u][e], p);
                }
            fwd = false;
            phase = PH_BACK;
            --s;
        } else if (phase == PH_PROBE) {
            // ------------------------------------------- sum_b fft2(dP) conj(H_b) (solvers.py:265, 484)
            if (upd_probe) {
                float2 *ap = a.acc_probe + (size_t)m * NN;
#pragma unroll
                for (int u = 0; u < U; ++u)
#pragma unroll
                    for (int e = 0; e < E; ++e) {
                        const float2 h = cmul(hy[I::ky(u, e)], hx[I::kx(u, e)]);
                        atomic_add_c(ap + I::flat(u, e), cscale(cmulc(v[u][e], h), inv_n));
                    }
            }
            if constexpr (grad) {
                if (upd_pos) {
                    // The gradient engine's position gradient is sum_r Re(conj(chi) D_dir O_0) alone (no
                    // step-size denominator), D_dir = ifft2(DFT(P_m)/N^2 H_b (-2 pi i k_dir)).  By Parseval
                    // it is sum_k 2 pi k_dir Im(conj(F) g), F = fft2(chi conj(O_0)) (this spectrum),
                    // g = DFT(P_m)/N^2 H_b: no inverse transforms and no real-space pass.
                    const float2 *pk = a.probe_k + (size_t)m * NN;
                    const float twopi = 6.283185307179586f;
                    float t2[2] = {0.f, 0.f};
#pragma unroll
                    for (int u = 0; u < U; ++u)
#pragma unroll
                        for (int e = 0; e < E; ++e) {
                            const int ky = I::ky(u, e), kx = I::kx(u, e);
                            const float2 g = cmul(__ldg(pk + I::flat(u, e)), cmul(hy[ky], hx[kx]));
                            const float im = v[u][e].x * g.y - v[u][e].y * g.x;   // Im(conj(F) g)
                            t2[0] += (twopi * a.fy[ky]) * im;
                            t2[1] += (twopi * a.fx[kx]) * im;
                        }
                    warp_atomic_sum(sums + a.o_pnum + 2 * b, (double)t2[0]);
                    warp_atomic_sum(sums + a.o_pnum + 2 * b + 1, (double)t2[1]);
                }
                return;
            }
            if (!upd_pos) return;
            load_probe_spectrum(0);
            fwd = false;
            phase = PH_POS;
            dir = 0;
        } else {
            // ------------------------------------------- position step (solvers.py:275-288), R layout
            const CutView<N> cv = load_cv();
            const float2 *ps0 = psi_b;   // slot 0 holds the slice-0 exit-wave update
            float t2[2] = {0.f, 0.f};
#pragma unroll
            for (int u = 0; u < U; ++u)
#pragma unroll
                for (int q0 = 0; q0 < E; q0 += 8) {
                    float2 oo[8], cc[8];
#pragma unroll
                    for (int j = 0; j < 8; ++j) {
                        oo[j] = cv.at(a.object, u, q0 + j);
                        cc[j] = ps0[I::flat(u, q0 + j)];
                    }
#pragma unroll
                    for (int j = 0; j < 8; ++j) {
                        const float2 pr = cmul(v[u][q0 + j], oo[j]);
                        t2[0] += cc[j].x * pr.x + cc[j].y * pr.y;
                        t2[1] += cabs2(pr);
                    }
                }
            warp_atomic_sum(sums + a.o_pnum + 2 * b + dir, (double)t2[0]);
            warp_atomic_sum(sums + a.o_pden + 2 * b + dir, (double)t2[1]);
            if (dir == 1) return;
            dir = 1;
            load_probe_spectrum(1);
            fwd = false;
        }
        PHB_T_MARK(2 + timed_phase);
    }
}

// ---------------------------------------------------------------- group_obj_mag
// positions split over gridDim.y: each thread walks B / GOM_SPLIT positions (its loads of
// different positions are independent; more splits, more of them in flight per SM)
constexpr int GOM_SPLIT = 32;
// gom[r, c] += sum_b |prod_s O_s[y0_b + r, x0_b + c]|^2  (solvers.py:203)
template <int N>
__global__ void k_gom(const GroupArgs a, float *out) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    const int r = f / N, c = f % N;
    const int nsplit = gridDim.y;
    const int b0 = (a.B * blockIdx.y) / nsplit, b1 = (a.B * (blockIdx.y + 1)) / nsplit;
    float acc = 0.f;
    for (int b = b0; b < b1; ++b) {
        if (!pos_ok(a.group[b], a.n_pos)) continue;   // recorded by the fused kernel of the group
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
    float grad_pos_scale;
    double *group_loss;
    float *grad_tilt;
    float grad_tilt_scale;
    float *errors;   // N = 256: per-position errors, the root of the summed squares in `sums`
    int64_t n_pos;   // bounds-checking build: group rows outside [0, n_pos) are skipped
};

__global__ void k_finalize(const FinArgs f) {
    const SumIdx SI(f.B_max, f.S, f.M);
    double *sums = f.sums;
    __shared__ double red[2][32];
    const int tid = threadIdx.x;
    if (f.mode == MODE_LSQML) {
        // coef[k] for the S slices then the M modes: sum over the group's positions of the
        // per-position numerators, split over the block (up to 64 k at a time, blockDim / n
        // threads per k, each a contiguous run of positions) and combined in a fixed order
        __shared__ double part[256];
        const int K = f.S + f.M;
        for (int k0 = 0; k0 < K; k0 += 64) {
            const int n = min(64, K - k0), parts = (int)blockDim.x / n;
            const int k = k0 + tid % n, pi = tid / n;
            double acc = 0.0;
            if (pi < parts) {
                const int b0 = (f.B * pi) / parts, b1 = (f.B * (pi + 1)) / parts;
                for (int b = b0; b < b1; ++b)
                    acc += k < f.S ? sums[SI.numO + (int64_t)b * f.S + k] : sums[SI.numP + (int64_t)b * f.M + (k - f.S)];
            }
            part[tid] = acc;
            __syncthreads();
            if (tid < n) {
                double s = 0.0;
                for (int q = 0; q < parts; ++q) s += part[q * n + tid];
                const int kk = k0 + tid;
                f.coef[kk] = kk < f.S ? (double)f.beta_object * s / (sums[SI.denO + kk] + (double)f.gamma)
                                      : (double)f.beta_probe * s / (sums[SI.denP] + (double)f.gamma);
            }
            __syncthreads();
        }
    }
    const bool pos = (f.flags & PHB_FLAG_UPDATE_POSITION) && (f.mode <= MODE_GRAD);
    if (pos && f.mode != MODE_GRAD && f.pos_update) {
        double d[2] = {0.0, 0.0};
        for (int b = tid; b < f.B; b += blockDim.x) {
            if (!pos_ok(f.group[b], f.n_pos)) continue;   // a skipped row's sums are 0 (0 / 0 here)
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
            if (!pos_ok(p, f.n_pos)) continue;
            f.pos_update[2 * p] = (float)(sums[SI.pnum + 2 * b] / n / red[0][0]);
            f.pos_update[2 * p + 1] = (float)(sums[SI.pnum + 2 * b + 1] / n / red[1][0]);
        }
    }
    if (f.mode == MODE_GRAD) {
        const double gs = f.grad_pos_scale != 0.f ? (double)f.grad_pos_scale : 1.0;
        double lsum = 0.0;
        for (int b = tid; b < f.B; b += blockDim.x) {
            const int64_t p = f.group[b];
            if (!pos_ok(p, f.n_pos)) continue;
            if (pos && f.grad_pos) {
                f.grad_pos[2 * p] = (float)(gs * sums[SI.pnum + 2 * b]);
                f.grad_pos[2 * p + 1] = (float)(gs * sums[SI.pnum + 2 * b + 1]);
            }
            if (f.loss) f.loss[p] = (float)sums[SI.loss + b];
            lsum += sums[SI.loss + b];
            if (f.grad_tilt && (f.flags & PHB_FLAG_UPDATE_TILT)) {
                const double ts = f.grad_tilt_scale != 0.f ? (double)f.grad_tilt_scale : 1.0;
                f.grad_tilt[2 * p] = (float)(ts * sums[SI.tilt + 2 * b]);
                f.grad_tilt[2 * p + 1] = (float)(ts * sums[SI.tilt + 2 * b + 1]);
            }
        }
        if (f.group_loss) {
            for (int o = 16; o > 0; o >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
            if ((tid & 31) == 0) atomicAdd(f.group_loss, lsum);
        }
    }
    if (f.errors && (f.flags & PHB_FLAG_CALC_ERROR) && f.mode != MODE_GRAD)
        for (int b = tid; b < f.B; b += blockDim.x)
            if (pos_ok(f.group[b], f.n_pos)) f.errors[f.group[b]] = (float)sqrt(sums[SI.err + b]);
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

// blocks [0, nblocks) of a grid-stride loop over the S*H*W object values, this block = blk
__device__ __forceinline__ void obj_apply_body(const ObjApplyArgs &a, int64_t blk, int64_t nblocks) {
    const int64_t total = (int64_t)a.S * a.HW;
    bool bad = false;
    for (int64_t i = blk * blockDim.x + threadIdx.x; i < total; i += nblocks * blockDim.x) {
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

__global__ void k_obj_apply(const ObjApplyArgs a) { obj_apply_body(a, blockIdx.x, gridDim.x); }

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
// mode m's CTA (N = 256: the 4-CTA cluster of mode m); all threads of the CTA call it
template <int N>
__device__ __forceinline__ void probe_apply_body(const ProbeApplyArgs &a, int m) {
    using I = Idx<N>;
    constexpr int U = I::U, E = I::E, NN = N * N, CTAS = TileCfg<N>::CTAS;
    extern __shared__ float4 smem_raw[];
    float2 *xb = reinterpret_cast<float2 *>(smem_raw);
    float2 *twid = xb + Lay<N>::BUF;
    float *fred = reinterpret_cast<float *>(twid + TileCfg<N>::TW);
    fft_init_twiddles<N>(twid);
    __syncthreads();
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
                const int idx = I::row(u, q) * N + I::col(u, q);
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
    if (m == 0 && a.new_obj_mag && a.gom && (CTAS == 1 || cluster_rank() == 0))
        for (int i = threadIdx.x; i < NN; i += blockDim.x) a.new_obj_mag[i] += a.gom[i];
    if (a.mode == MODE_GRAD) return;
    // refresh spectrum
#pragma unroll
    for (int u = 0; u < U; ++u)
#pragma unroll
        for (int q = 0; q < E; ++q) {
            v[u][q] = P[I::row(u, q) * N + I::col(u, q)];
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

template <int N>
__global__ void __launch_bounds__(FFT_THREADS, 1) k_probe_apply(const ProbeApplyArgs a) {
    probe_apply_body<N>(a, (int)(blockIdx.x / TileCfg<N>::CTAS));
}

// N <= 128: the probe and object updates of a mini-batch are independent, so one launch
// runs both -- CTAs [0, M) the probe modes (one 128^2 transform pair each), the rest a
// grid-stride pass over the object -- and the object work fills the SMs the M probe CTAs
// leave idle instead of waiting in the stream for them.
template <int N>
__global__ void __launch_bounds__(FFT_THREADS, 1) k_apply(const ObjApplyArgs o, const ProbeApplyArgs p,
                                                          int probe_ctas, int obj_on) {
    static_assert(TileCfg<N>::CTAS == 1, "one CTA per probe mode");
    if ((int)blockIdx.x < probe_ctas) {
        probe_apply_body<N>(p, (int)blockIdx.x);
        return;
    }
    if (obj_on) obj_apply_body(o, (int64_t)blockIdx.x - probe_ctas, (int64_t)gridDim.x - probe_ctas);
}

// ---------------------------------------------------------------- propagator factors
// phaser's propagators (simulation.py:160-190) are band-limited Fresnel kernels,
// exp(-i pi dz lambda (ky^2 + kx^2)) * band, i.e. p(ky) p(kx) inside the band with
// p(0) = 1.  Extract p(ky) = P[ky, 0] and p(kx) = P[0, kx], the band bits (P != 0), and
// check |P - band p(ky) p(kx)| <= 1e-5 max|P| (the reference's own float32 rounding is
// ~1e-6); info[0] = pattern mask is all ones, info[1] = separable.
template <int N>
__global__ void __launch_bounds__(1024) k_prop_init(const float2 *props, int G, const float *mask, float2 *prop1d,
                                                   uint32_t *band, int32_t *info) {
    __shared__ int ok_mask, ok_sep;
    if (threadIdx.x == 0) {
        ok_mask = 1;
        ok_sep = 1;
    }
    __syncthreads();
    for (int f = threadIdx.x; f < N * N; f += blockDim.x)
        if (mask[f] != 1.0f) ok_mask = 0;
    if (G <= 0) {
        for (int k = threadIdx.x; k < N * N / 32; k += blockDim.x) band[k] = 0xffffffffu;
    } else {
        for (int k = threadIdx.x; k < N * N / 32; k += blockDim.x) {
            uint32_t bits = 0;
            for (int j = 0; j < 32; ++j) {
                const float2 p = props[k * 32 + j];
                if (p.x != 0.f || p.y != 0.f) bits |= 1u << j;
            }
            band[k] = bits;
        }
        for (int i = threadIdx.x; i < G * 2 * N; i += blockDim.x) {
            const int g = i / (2 * N), k = i % (2 * N);
            prop1d[i] = k < N ? props[(size_t)g * N * N + (size_t)k * N] : props[(size_t)g * N * N + (k - N)];
        }
        __syncthreads();
        for (int i = threadIdx.x; i < G * N * N; i += blockDim.x) {
            const int g = i / (N * N), f = i % (N * N), ky = f / N, kx = f % N;
            const float2 p = props[i];
            const bool in = (band[f >> 5] >> (f & 31)) & 1u;
            const float2 q = in ? cmul(prop1d[g * 2 * N + ky], prop1d[g * 2 * N + N + kx]) : make_float2(0.f, 0.f);
            const float d = fabsf(p.x - q.x) + fabsf(p.y - q.y);
            if (!(d <= 1e-5f * fmaxf(1.0f, sqrtf(cabs2(p))))) ok_sep = 0;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        info[0] = ok_mask;
        info[1] = ok_sep;
    }
}

// ---------------------------------------------------------------- K-order packing
template <int N>
__global__ void k_pack_f32(const float *src, float *dst) {
    for (int f = threadIdx.x; f < N * N; f += blockDim.x) {
        int ky, kx;
        flat_to_k<N>(f, ky, kx);
        dst[f] = src[ky * N + kx];
    }
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

// positions completely outside the object (the reference's check in utils/object.py:288-289)
__global__ void __launch_bounds__(1024) k_count_outside(const float *scan, int64_t n, double y0, double x0,
                                                        double y1, double x1, int32_t *n_out) {
    __shared__ double red[32];
    int outside = 0;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
        const double py = scan[2 * i], px = scan[2 * i + 1];
        outside += (py < y0) || (py > y1) || (px < x0) || (px > x1);
    }
    const double tot = block_sum1<1024>((double)outside, red);
    if (threadIdx.x == 0) *n_out = (int32_t)tot;
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
    return (size_t)Lay<N>::BUF * sizeof(float2) + (TileCfg<N>::TW + 4 * N) * sizeof(float2) + 64 * sizeof(double) +
           64 * sizeof(float) +
           (size_t)N * N / 32 * sizeof(uint32_t) + 2 * FFT_THREADS * sizeof(uint64_t) +
           (size_t)FFTCfg<N>::U * FFT_THREADS * sizeof(int32_t);
}
template <int N>
static size_t fft_smem_bytes() {
    return (size_t)Lay<N>::BUF * sizeof(float2) + TileCfg<N>::TW * sizeof(float2) + 64 * sizeof(float);
}

template <int N>
static int launch_probe_apply(const ProbeApplyArgs &p, cudaStream_t st) {
    constexpr unsigned C = TileCfg<N>::CTAS;
    return launch_clustered(k_probe_apply<N>, (unsigned)p.M * C, FFT_THREADS, C, fft_smem_bytes<N>(), st, p);
}

template <int N>
static int configure_kernels() {
    static int done = -1;
    if (done >= 0) return done;
    int rc = PHB_OK;
    if (cudaFuncSetAttribute(k_probe_apply<N>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)fft_smem_bytes<N>()) != cudaSuccess)
        rc = record_cuda(cudaGetLastError());
    if constexpr (TileCfg<N>::CTAS == 1) {
        if (!rc && cudaFuncSetAttribute(k_apply<N>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)fft_smem_bytes<N>()) != cudaSuccess)
            rc = record_cuda(cudaGetLastError());
    }
    done = rc;
    return rc;
}

static int validate(const phb_engine *e) {
    if (!e) return PHB_ERR_INVALID_ARG;
    if (e->N != 64 && e->N != 128 && e->N != 256) return PHB_ERR_UNSUPPORTED;
    if (e->M < 1 || e->M > 8) return PHB_ERR_UNSUPPORTED;
    if (e->S < 1 || e->B_max < 1 || e->H < 1 || e->W < 1 || e->n_pos < 1) return PHB_ERR_INVALID_ARG;
    if (!e->object || !e->probe || !e->scan || !e->patterns || !e->pattern_mask || !e->ky || !e->kx)
        return PHB_ERR_INVALID_ARG;
    if (e->S > 1 && !e->propagators) return PHB_ERR_INVALID_ARG;
    if (e->tilt && !e->thicknesses) return PHB_ERR_INVALID_ARG;
    if (e->pattern_u16 != 0 && e->pattern_u16 != 1) return PHB_ERR_INVALID_ARG;
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
    if (e->pattern_u16) a.patterns16 = (const uint16_t *)e->patterns;
    else a.patterns = (const float *)e->patterns;
    a.mask_k = w.mask_k;
    a.prop1d = w.prop1d;
    a.band = w.band;
    a.info = w.info;
    a.err_word = w.info + 3;
    const SumIdx SI(e->B_max, e->S, e->M);
    a.o_numO = SI.numO;
    a.o_denO = SI.denO;
    a.o_numP = SI.numP;
    a.o_denP = SI.denP;
    a.o_pnum = SI.pnum;
    a.o_pden = SI.pden;
    a.o_pnorm = SI.pnorm;
    a.o_loss = SI.loss;
    a.o_tilt = SI.tilt;
    a.o_err = SI.err;
    a.far = w.far;
    a.far_int = w.far_int;
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

template <int N, int MODE, int MC>
static int launch_group_mode(const GroupArgs &a, cudaStream_t st) {
    static bool configured = false;
    if (!configured) {
        if (cudaFuncSetAttribute(k_group<N, MODE, MC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)group_smem_bytes<N>()) != cudaSuccess)
            return record_cuda(cudaGetLastError());
        configured = true;
    }
    // N = 256: one cluster of 4 CTAs (the polyphase parts) per (position, mode); ePIE at N <= 128:
    // one cluster of M CTAs (the modes) per position; otherwise independent CTAs
    constexpr unsigned C = TileCfg<N>::CTAS;
    const unsigned cluster = C > 1 ? C : (MODE == MODE_EPIE ? (unsigned)a.M : 1u);
    return launch_clustered(k_group<N, MODE, MC>, (unsigned)(a.B * a.M) * C, FFT_THREADS, cluster, group_smem_bytes<N>(),
                            st, a);
}

template <int N, int MODE>
static int launch_group_m(const GroupArgs &a, cudaStream_t st) {
    switch (a.M) {
        case 1: return launch_group_mode<N, MODE, 1>(a, st);
        case 2: return launch_group_mode<N, MODE, 2>(a, st);
        case 4: return launch_group_mode<N, MODE, 4>(a, st);
        case 8: return launch_group_mode<N, MODE, 8>(a, st);
        default: return launch_group_mode<N, MODE, 0>(a, st);
    }
}

template <int N>
static int launch_group(const GroupArgs &a, cudaStream_t st) {
    if constexpr (N == 256) {   // modes run in separate clusters: no per-mode template, no ePIE
        switch (a.mode) {
            case MODE_LSQML: return launch_group_mode<N, MODE_LSQML, 0>(a, st);
            case MODE_GRAD: return launch_group_mode<N, MODE_GRAD, 0>(a, st);
            case MODE_PRE_LSQML: return launch_group_mode<N, MODE_PRE_LSQML, 0>(a, st);
            case MODE_PRE_GRAD: return launch_group_mode<N, MODE_PRE_GRAD, 0>(a, st);
            case MODE_SIM: return launch_group_mode<N, MODE_SIM, 0>(a, st);
            case MODE_EPIE:
            case MODE_PRE_EPIE: return PHB_ERR_UNSUPPORTED;
            default: return PHB_ERR_INVALID_ARG;
        }
    } else {
        switch (a.mode) {
            case MODE_LSQML: return launch_group_m<N, MODE_LSQML>(a, st);
            case MODE_EPIE: return launch_group_m<N, MODE_EPIE>(a, st);
            case MODE_GRAD: return launch_group_m<N, MODE_GRAD>(a, st);
            case MODE_PRE_LSQML: return launch_group_mode<N, MODE_PRE_LSQML, 0>(a, st);
            case MODE_PRE_EPIE: return launch_group_mode<N, MODE_PRE_EPIE, 0>(a, st);
            case MODE_PRE_GRAD: return launch_group_mode<N, MODE_PRE_GRAD, 0>(a, st);
            case MODE_SIM: return launch_group_m<N, MODE_SIM>(a, st);
            default: return PHB_ERR_INVALID_ARG;
        }
    }
}

// the fused step of one group: for LSQ-ML and the gradient engine the forward launch,
// which leaves the far-field waves and the summed intensity in the workspace, and the
// launch resumed at the detector; ePIE in one launch
template <int N>
static int launch_step(GroupArgs a, const Workspace &w, cudaStream_t st) {
    const bool split = a.mode == MODE_LSQML || a.mode == MODE_GRAD;
    if (split) {
        const int rc = record_cuda(cudaMemsetAsync(w.far_int, 0, (size_t)a.B * N * N * sizeof(float), st));
        if (rc) return rc;
    }
    a.resume = 0;
    int rc = launch_group<N>(a, st);
    if (rc || !split) return rc;
    a.resume = 1;
    return launch_group<N>(a, st);
}

template <int N>
static int probe_spectrum(const phb_engine *e, const Workspace &w, cudaStream_t st) {
    ProbeApplyArgs p{};
    p.mode = MODE_LSQML;
    p.M = e->M;
    p.probe = (float2 *)e->probe;
    p.probe_k = w.probe_k;
    p.update = 0;
    return launch_probe_apply<N>(p, st);
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
    k_prop_init<N><<<1, 1024, 0, st>>>((const float2 *)e->propagators, e->S - 1, e->pattern_mask, w.prop1d, w.band,
                                        w.info);
    if ((rc = check_launch())) return rc;
    k_pack_f32<N><<<1, 1024, 0, st>>>(e->pattern_mask, w.mask_k);
    if ((rc = check_launch())) return rc;
    if ((rc = probe_spectrum<N>(e, w, st))) return rc;
    // the propagator check is the only result the host needs from init
    int32_t info[4];
    if ((rc = record_cuda(cudaMemcpyAsync(info, w.info, sizeof(info), cudaMemcpyDeviceToHost, st)))) return rc;
    if ((rc = record_cuda(cudaStreamSynchronize(st)))) return rc;
    if (e->S > 1 && !info[1]) return PHB_ERR_UNSUPPORTED;   // not a separable (Fresnel) propagator
    return PHB_OK;
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
        k_gom<N><<<dim3((N * N + 255) / 256, GOM_SPLIT), 256, 0, st>>>(a, e->new_obj_mag);
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
    // the CTAs (clusters) of the modes add their intensities into the output
    if ((rc = record_cuda(cudaMemsetAsync(out, 0, (size_t)B * N * N * sizeof(float), st)))) return rc;
    return launch_group<N>(a, st);
}

template <int N>
static int solver_finish(const phb_engine *e, const phb_step *sp, const int64_t *group, int B, cudaStream_t st);

template <int N>
static int solver_group(const phb_engine *e, const phb_step *sp, const int64_t *group, int B, cudaStream_t st) {
    int rc = configure_kernels<N>();
    if (rc) return rc;
    Workspace w = carve(e->workspace, N, e->M, e->S, e->B_max, e->H, e->W);
    const int mode = sp->solver == PHB_SOLVER_EPIE ? MODE_EPIE : (sp->solver == PHB_SOLVER_GRAD ? MODE_GRAD : MODE_LSQML);
    const int flags = sp->flags;
    const bool upd_obj = flags & PHB_FLAG_UPDATE_OBJECT, upd_probe = flags & PHB_FLAG_UPDATE_PROBE;
    // partial launch: rows [b_begin, b_end) of the group; the accumulators then hold this
    // share only, and the caller sums them over ranks before phb_solver_group_finish
    const bool partial = flags & PHB_FLAG_PARTIAL;
    const int b0 = partial ? sp->b_begin : 0, b1 = partial ? sp->b_end : B;
    GroupArgs a = make_args(e, w, mode, flags, group + b0, b1 - b0);
    if (b0) {   // per-position sums of this launch's rows sit at group rows b0.. (group-wide layout)
        a.o_numO += (int64_t)b0 * e->S;
        a.o_numP += (int64_t)b0 * e->M;
        a.o_pnum += 2 * (int64_t)b0;
        a.o_pden += 2 * (int64_t)b0;
        a.o_pnorm += b0;
        a.o_loss += b0;
        a.o_tilt += 2 * (int64_t)b0;
        a.o_err += b0;
    }
    a.errors = sp->errors;
    a.beta_object = sp->beta_object;
    if (mode == MODE_LSQML) {
        if (!upd_obj && !e->new_probe_mag) a.illum = nullptr;
        if (upd_probe || e->new_obj_mag) {
            if ((rc = record_cuda(cudaMemsetAsync(w.gom, 0, (size_t)N * N * sizeof(float), st)))) return rc;
            k_gom<N><<<dim3((N * N + 255) / 256, GOM_SPLIT), 256, 0, st>>>(a, w.gom);
            if ((rc = check_launch())) return rc;
        }
    } else {
        a.illum = nullptr;
    }
    if (mode == MODE_GRAD) a.acc_obj = (float2 *)sp->grad_object;
    a.group_patterns = sp->group_patterns;
    a.status = sp->status;
    a.group_index = sp->group_index;
    if (sp->event_begin && (rc = record_cuda(cudaEventRecord((cudaEvent_t)sp->event_begin, st)))) return rc;
    if ((rc = launch_step<N>(a, w, st))) return rc;
    if (sp->event_end && (rc = record_cuda(cudaEventRecord((cudaEvent_t)sp->event_end, st)))) return rc;
    if (partial) return PHB_OK;
    return solver_finish<N>(e, sp, group, B, st);
}

// Step sizes, position / probe / object updates of one mini-batch from the
// accumulators in the workspace (all of the group's rows present).
template <int N>
static int solver_finish(const phb_engine *e, const phb_step *sp, const int64_t *group, int B, cudaStream_t st) {
    int rc = configure_kernels<N>();
    if (rc) return rc;
    Workspace w = carve(e->workspace, N, e->M, e->S, e->B_max, e->H, e->W);
    const int mode = sp->solver == PHB_SOLVER_EPIE ? MODE_EPIE : (sp->solver == PHB_SOLVER_GRAD ? MODE_GRAD : MODE_LSQML);
    const int flags = sp->flags & ~PHB_FLAG_PARTIAL;
    const bool upd_obj = flags & PHB_FLAG_UPDATE_OBJECT, upd_probe = flags & PHB_FLAG_UPDATE_PROBE;
    float *illum = (mode == MODE_LSQML && (upd_obj || e->new_probe_mag)) ? w.illum : nullptr;

    FinArgs f{};
    f.mode = mode;
    f.flags = flags;
    f.S = e->S;
    f.M = e->M;
    f.B = B;
    f.n_pos = e->n_pos;
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
    f.grad_pos_scale = sp->grad_pos_scale;
    f.group_loss = sp->group_loss;
    f.grad_tilt = sp->grad_tilt;
    f.grad_tilt_scale = sp->grad_tilt_scale;
    f.errors = mode == MODE_LSQML ? sp->errors : nullptr;   // the split far field leaves squared sums
    k_finalize<<<1, 256, 0, st>>>(f);
    if ((rc = check_launch())) return rc;

    const bool obj_on = mode != MODE_GRAD && (upd_obj || illum);
    const bool probe_on = upd_probe || (mode == MODE_LSQML && e->new_obj_mag);
    ObjApplyArgs o{};
    if (obj_on) {
        o.mode = mode;
        o.S = e->S;
        o.HW = e->H * e->W;
        o.reg = sp->illum_reg_object;
        o.eps = 1e-16f;
        o.object = (float2 *)e->object;
        o.acc = w.acc_obj;
        o.illum = illum;
        o.new_probe_mag = e->new_probe_mag;
        o.coef = w.coef;
        o.status = sp->status;
        o.group_index = sp->group_index;
        o.update = upd_obj;
    }
    ProbeApplyArgs p{};
    if (probe_on) {
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
    }
    const int64_t total = (int64_t)e->S * e->H * e->W;
    if constexpr (TileCfg<N>::CTAS == 1) {
        if (obj_on && probe_on) {   // one launch: M probe CTAs + object CTAs on the other SMs
            int64_t g = (total + FFT_THREADS - 1) / FFT_THREADS;
            if (g > 148 - e->M) g = 148 - e->M > 1 ? 148 - e->M : 1;   // one wave beside the probe CTAs
            k_apply<N><<<(unsigned)(e->M + g), FFT_THREADS, fft_smem_bytes<N>(), st>>>(o, p, e->M, 1);
            return check_launch();
        }
    }
    if (obj_on) {
        int64_t g = (total + 255) / 256;
        if (g > 148 * 16) g = 148 * 16;
        k_obj_apply<<<(unsigned)g, 256, 0, st>>>(o);
        if ((rc = check_launch())) return rc;
    }
    if (probe_on) {
        if ((rc = launch_probe_apply<N>(p, st))) return rc;
    }
    return PHB_OK;
}

}  // namespace phb

using namespace phb;

#ifdef PHB_PHASE_TIMING
extern "C" int phb_debug_phase_cycles(unsigned long long *out16, int reset) {
    int rc = phb::record_cuda(cudaMemcpyFromSymbol(out16, phb::g_phase_cycles, 16 * sizeof(unsigned long long)));
    if (!rc && reset) {
        unsigned long long z[16] = {0};
        rc = phb::record_cuda(cudaMemcpyToSymbol(phb::g_phase_cycles, z, sizeof(z)));
    }
    return rc;
}
#endif

extern "C" {

size_t phb_engine_workspace_bytes(int32_t N, int32_t M, int32_t S, int32_t B_max, int64_t H, int64_t W) {
    if (N <= 0 || M <= 0 || S <= 0 || B_max <= 0 || H <= 0 || W <= 0) return 0;
    return carve(nullptr, N, M, S, B_max, H, W).bytes;
}

// call F<N>(args...) for the engine's probe size
#define PHB_DISPATCH_N(n, F, ...) \
    ((n) == 256 ? F<256>(__VA_ARGS__) : (n) == 128 ? F<128>(__VA_ARGS__) : F<64>(__VA_ARGS__))

int phb_engine_init(const phb_engine *e, void *stream) {
    const NvtxRange range("phb_engine_init");
    int rc = validate(e);
    if (rc) return rc;
    return PHB_DISPATCH_N(e->N, engine_init, e, (cudaStream_t)stream);
}

int phb_engine_probe_changed(const phb_engine *e, void *stream) {
    int rc = validate(e);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    if ((rc = PHB_DISPATCH_N(e->N, configure_kernels))) return rc;
    const Workspace w = carve(e->workspace, e->N, e->M, e->S, e->B_max, e->H, e->W);
    return PHB_DISPATCH_N(e->N, probe_spectrum, e, w, st);
}

int phb_presolve_group(const phb_engine *e, const int64_t *group, int32_t B, int32_t solver, int32_t gradient_form,
                       double *rescale_num, double *rescale_den, void *stream) {
    const NvtxRange range("phb_presolve_group");
    int rc = validate(e);
    if (rc) return rc;
    if (!group || !rescale_num || !rescale_den || B < 1 || B > e->B_max) return PHB_ERR_INVALID_ARG;
    if (e->N == 256 && solver == PHB_SOLVER_EPIE && !gradient_form) return PHB_ERR_UNSUPPORTED;
    cudaStream_t st = (cudaStream_t)stream;
    return PHB_DISPATCH_N(e->N, presolve, e, group, B, solver, gradient_form, rescale_num, rescale_den, st);
}

int phb_simulate_group(const phb_engine *e, const int64_t *group, int32_t B, float *intensity, void *stream) {
    const NvtxRange range("phb_simulate_group");
    int rc = validate(e);
    if (rc) return rc;
    if (!group || !intensity || B < 1 || B > e->B_max) return PHB_ERR_INVALID_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    return PHB_DISPATCH_N(e->N, simulate, e, group, B, intensity, st);
}

int phb_solver_group_finish(const phb_engine *e, const phb_step *st, const int64_t *group, int32_t B, void *stream) {
    const NvtxRange range("phb_solver_group_finish");
    int rc = validate(e);
    if (rc) return rc;
    if (!st || !group || B < 1 || B > e->B_max) return PHB_ERR_INVALID_ARG;
    if (st->solver < PHB_SOLVER_LSQML || st->solver > PHB_SOLVER_GRAD) return PHB_ERR_INVALID_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    return PHB_DISPATCH_N(e->N, solver_finish, e, st, group, B, s);
}

int phb_engine_reduce_layout(int32_t N, int32_t M, int32_t S, int32_t B_max, int64_t H, int64_t W, int64_t *out4) {
    if (!out4 || N <= 0 || M <= 0 || S <= 0 || B_max <= 0 || H <= 0 || W <= 0) return PHB_ERR_INVALID_ARG;
    // carve at a stand-in base address (never dereferenced) to read the offsets
    char *const origin = reinterpret_cast<char *>(uintptr_t(1) << 20);
    const Workspace w = carve(origin, N, M, S, B_max, H, W);
    out4[0] = (int64_t)(reinterpret_cast<char *>(w.acc_obj) - origin);
    out4[1] = (int64_t)(reinterpret_cast<char *>(w.gom + (size_t)N * N) - reinterpret_cast<char *>(w.acc_obj));
    out4[2] = (int64_t)(reinterpret_cast<char *>(w.sums) - origin);
    out4[3] = (int64_t)SumIdx(B_max, S, M).total * (int64_t)sizeof(double);
    return PHB_OK;
}

int phb_solver_group(const phb_engine *e, const phb_step *st, const int64_t *group, int32_t B, void *stream) {
    const NvtxRange range("phb_solver_group");
    int rc = validate(e);
    if (rc) return rc;
    if (!st || !group || B < 1 || B > e->B_max) return PHB_ERR_INVALID_ARG;
    if (st->solver < PHB_SOLVER_LSQML || st->solver > PHB_SOLVER_GRAD) return PHB_ERR_INVALID_ARG;
    if (st->solver != PHB_SOLVER_GRAD && e->noise == PHB_NOISE_POISSON) return PHB_ERR_UNSUPPORTED;
    if (st->solver == PHB_SOLVER_GRAD && (st->flags & PHB_FLAG_UPDATE_OBJECT) && !st->grad_object)
        return PHB_ERR_INVALID_ARG;
    if (st->solver == PHB_SOLVER_GRAD && (st->flags & PHB_FLAG_UPDATE_PROBE) && !st->grad_probe)
        return PHB_ERR_INVALID_ARG;
    if (st->solver == PHB_SOLVER_GRAD && (st->flags & PHB_FLAG_UPDATE_POSITION) && !st->grad_pos)
        return PHB_ERR_INVALID_ARG;
    if ((st->flags & PHB_FLAG_UPDATE_TILT) && (st->solver != PHB_SOLVER_GRAD || !st->grad_tilt || !e->tilt))
        return PHB_ERR_INVALID_ARG;
    if ((st->flags & PHB_FLAG_UPDATE_POSITION) && st->solver != PHB_SOLVER_GRAD && !st->pos_update)
        return PHB_ERR_INVALID_ARG;
    if ((st->flags & PHB_FLAG_PARTIAL) && (st->b_begin < 0 || st->b_end > B || st->b_begin >= st->b_end))
        return PHB_ERR_INVALID_ARG;
    if (e->N == 256 && st->solver == PHB_SOLVER_EPIE) return PHB_ERR_UNSUPPORTED;
    cudaStream_t s = (cudaStream_t)stream;
    return PHB_DISPATCH_N(e->N, solver_group, e, st, group, B, s);
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

int phb_count_outside(const float *scan, int64_t n_pos, double obj_min_y, double obj_min_x, double obj_max_y,
                      double obj_max_x, int32_t *n_outside, void *stream) {
    if (!scan || !n_outside || n_pos < 1) return PHB_ERR_INVALID_ARG;
    k_count_outside<<<1, 1024, 0, (cudaStream_t)stream>>>(scan, n_pos, obj_min_y, obj_min_x, obj_max_y, obj_max_x,
                                                          n_outside);
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

// ---------------------------------------------------------------- allocation-free variant
// phb_solver_group_static: the same mini-batch step as phb_solver_group, but its
// scratch (wavefield stack, accumulators, tables) lives in a fixed device array that
// is part of this library, so the call needs no workspace and allocates nothing.
namespace phb {

constexpr size_t kStaticScratchBytes = (size_t)64 << 20;   // 64 MiB, held by every GPU that loads the library
static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];
constexpr int kMaxDevices = 64;
static void *g_static_scratch_ptr[kMaxDevices] = {nullptr};   // device address of the array, per device

}  // namespace phb

extern "C" int phb_solver_group_static(const phb_engine *e, const phb_step *st, const int64_t *group, int32_t B,
                                       void *stream) {
    using namespace phb;
    const NvtxRange range("phb_solver_group_static");
    if (!e || !st || !group || B < 1) return PHB_ERR_INVALID_ARG;
    // a partial launch leaves its share in the accumulators for a later finish call, but
    // the next call here clears them (and the caller cannot reach this array): refuse it
    if (st->flags & PHB_FLAG_PARTIAL) return PHB_ERR_UNSUPPORTED;
    int dev = 0;
    int rc = record_cuda(cudaGetDevice(&dev));
    if (rc) return rc;
    if (dev < 0 || dev >= kMaxDevices) return PHB_ERR_UNSUPPORTED;
    if (!g_static_scratch_ptr[dev]) {
        // one-time set-up on this device (the array's host-side name is not a device address)
        void *p = nullptr;
        rc = record_cuda(cudaGetSymbolAddress(&p, g_static_scratch));
        if (rc) return rc;
        g_static_scratch_ptr[dev] = p;
    }
    phb_engine ws = *e;
    ws.B_max = B;
    ws.workspace = g_static_scratch_ptr[dev];
    ws.workspace_bytes = kStaticScratchBytes;
    if (ws.N <= 0 || ws.M <= 0 || ws.S <= 0 || ws.H <= 0 || ws.W <= 0) return PHB_ERR_INVALID_ARG;
    if (carve(nullptr, ws.N, ws.M, ws.S, B, ws.H, ws.W).bytes > kStaticScratchBytes) return PHB_ERR_SCRATCH_LIMIT;
    if ((rc = validate(&ws))) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    // the array keeps the previous call's contents: engine_init clears every accumulator and
    // rebuilds the tables (propagator factors, mask, probe spectrum) from this call's inputs
    rc = PHB_DISPATCH_N(ws.N, engine_init, &ws, s);
    if (rc) return rc;
    return phb_solver_group(&ws, st, group, B, stream);
}
