// Register-resident 2D FFT of one N x N complex64 tile per CTA (N = 64, 128).
//
// A CTA of 512 threads holds the whole tile in registers and exchanges through
// one shared-memory buffer (Lay<N>::BUF complex values).  Forward transforms
// leave the spectrum in a fixed permuted register order ("K layout"), inverse
// transforms consume that order and return natural order ("R layout").
// Pointwise work between the two (propagators, the detector constraint, shift
// filters) is done in K layout with explicit (ky, kx) indices from Idx<N>, so
// no reorder pass is ever needed.  Transforms are unnormalised DFTs with
// exp(-2 pi i nk/N) forward.
//
// N = 128 (32 values per thread, TWO exchanges per 2D transform):
//   x = xt + 32 j, kx = k1 + 4 k2;  y = yt + 16 m, ky = ky2 + 8 ky1
//   pass A  thread (xt = t%32, yt = t/32): DFT-4 over j -> k1, DFT-8 over m -> ky2,
//                                          twiddles W128^{xt k1} W128^{yt ky2}
//   pass B  thread (yt = t%16, ky2 = t/16%8, k1 = t/128): DFT-32 over xt -> k2
//   pass C  thread (ky2 = t/64, kx = t%64 + 64c, c = 0, 1): DFT-16 over yt -> ky1
//   R layout: v[0][8j + m]   = x[y = t/32 + 16m][x = t%32 + 32j]   (a warp covers 32
//                              consecutive pixels of one row: coalesced object access)
//   K layout: v[0][16c + i]  = X[ky = t/64 + 8i][kx = t%64 + 64c]
//   Exchange 1 stores row (yt + 16 (ky2 + 8 k1)) with stride 33, exchange 2 row
//   (128 ky2 + kx) with stride 17: both sides of both exchanges are conflict-free
//   (two wavefronts per warp-wide 8-byte access) and every address is a
//   per-thread base plus a compile-time offset.
//
// N = 256 (a cluster of 4 CTAs per tile, each holding one 128 x 128 part):
//   real space: CTA rank r = 2 a + b holds the polyphase component x[2 y' + a, 2 x' + b] in
//   the N = 128 R layout of (y', x');  Fourier space: it holds a quarter of the spectrum,
//   the points of N = 128 K-layout slots 8r .. 8r + 7, each at its four (ky' + 128p,
//   kx' + 128q).  The forward transform is the CTA's own 128 x 128 transform followed by one
//   radix-2 x 2 decimation-in-time stage across the cluster (an all-to-all through
//   distributed shared memory, twiddles W256^(a ky' + b kx')); the inverse runs the same
//   steps in reverse order with conjugate twiddles.
//
// N = 64 (8 values per thread, three exchanges): a line FFT of length
// N = E * NT runs as a radix-E DFT in registers (elements strided by NT) ->
// twiddle -> exchange among the NT threads of the line -> radix-NT DFTs:
//   R layout: v[u][q]        = x[row = t/8 + RPP u][col = t%8 + 8q]
//   K layout: v[u][p NT + k2] = X[ky = (t%8) P + p + E k2][kx = t/8 + RPP u]
#pragma once

#include <cooperative_groups.h>

#include "phb_common.cuh"

namespace phb {

// rank of this CTA in its thread-block cluster
__device__ __forceinline__ int cluster_rank() {
    unsigned r;
    asm("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return (int)r;
}

#ifndef PHB_FFT_THREADS
#define PHB_FFT_THREADS 512
#endif
constexpr int FFT_THREADS = PHB_FFT_THREADS;  // threads per tile (256: 4 lines each; 512: 2)
constexpr int RPP = FFT_THREADS / 8;          // rows (lines) handled per pass: 8 threads per line

template <int N> struct FFTCfg;
template <> struct FFTCfg<256> { static constexpr int E = 32, U = 1; };   // per CTA of the 4-CTA cluster
template <> struct FFTCfg<128> { static constexpr int E = 32, U = 1; };

// CTAs per tile (thread-block cluster of the transform) and twiddle-table entries
template <int N> struct TileCfg { static constexpr int CTAS = 1, TW = N; };
template <> struct TileCfg<256> { static constexpr int CTAS = 4, TW = 128 + 256; };
template <> struct FFTCfg<64>  { static constexpr int E = 8,  NT = 8, P = 1, U = 64 / RPP; };

// ----------------------------------------------------------------- small DFTs
template <bool INV>
__device__ __forceinline__ void dft4(float2 &a0, float2 &a1, float2 &a2, float2 &a3) {
    float2 t0 = cadd(a0, a2), t1 = csub(a0, a2), t2 = cadd(a1, a3), t3 = csub(a1, a3);
    float2 r3 = INV ? make_float2(-t3.y, t3.x) : make_float2(t3.y, -t3.x);   // * (+-i)
    a0 = cadd(t0, t2);
    a2 = csub(t0, t2);
    a1 = cadd(t1, r3);
    a3 = csub(t1, r3);
}

// multiply by W^e for the 16-point twiddles (forward sign); INV conjugates.
template <int EXP>
struct Tw16 {   // exp(-2 pi i EXP / 16)
    static constexpr float C1 = 0.92387953251128674f, S1 = 0.38268343236508978f, R = 0.70710678118654752f;
    static constexpr float re = EXP == 1 ? C1 : EXP == 2 ? R : EXP == 3 ? S1 : EXP == 6 ? -R : EXP == 9 ? -C1 : 1.f;
    static constexpr float im = EXP == 1 ? -S1 : EXP == 2 ? -R : EXP == 3 ? -C1 : EXP == 6 ? -R : EXP == 9 ? S1 : 0.f;
    static_assert(EXP == 0 || EXP == 1 || EXP == 2 || EXP == 3 || EXP == 4 || EXP == 6 || EXP == 9,
                  "unsupported twiddle");
};

template <bool INV, int EXP>
__device__ __forceinline__ float2 tw16(float2 a) {
    if constexpr (EXP == 0) {
        return a;
    } else if constexpr (EXP == 4) {
        return INV ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
    } else {
        return cmul(a, make_float2(Tw16<EXP>::re, INV ? -Tw16<EXP>::im : Tw16<EXP>::im));
    }
}

template <bool INV>
__device__ __forceinline__ void dft8(float2 *x) {
    constexpr float R = 0.70710678118654752f;
    float2 e0 = x[0], e1 = x[2], e2 = x[4], e3 = x[6];
    float2 o0 = x[1], o1 = x[3], o2 = x[5], o3 = x[7];
    dft4<INV>(e0, e1, e2, e3);
    dft4<INV>(o0, o1, o2, o3);
    // o_k *= W8^k
    float2 w1 = INV ? make_float2(R * (o1.x - o1.y), R * (o1.x + o1.y))
                    : make_float2(R * (o1.x + o1.y), R * (o1.y - o1.x));
    float2 w2 = INV ? make_float2(-o2.y, o2.x) : make_float2(o2.y, -o2.x);
    float2 w3 = INV ? make_float2(-R * (o3.x + o3.y), R * (o3.x - o3.y))
                    : make_float2(R * (o3.y - o3.x), -R * (o3.x + o3.y));
    x[0] = cadd(e0, o0); x[4] = csub(e0, o0);
    x[1] = cadd(e1, w1); x[5] = csub(e1, w1);
    x[2] = cadd(e2, w2); x[6] = csub(e2, w2);
    x[3] = cadd(e3, w3); x[7] = csub(e3, w3);
}

template <bool INV>
__device__ __forceinline__ void dft16(float2 *x) {
    // n = q0 + 4*n1, k = k1 + 4*k2
#pragma unroll
    for (int q0 = 0; q0 < 4; ++q0) dft4<INV>(x[q0], x[q0 + 4], x[q0 + 8], x[q0 + 12]);
    // x[q0 + 4*k1] = A[q0][k1]; twiddle W16^{q0*k1}
    x[5] = tw16<INV, 1>(x[5]);  x[9] = tw16<INV, 2>(x[9]);  x[13] = tw16<INV, 3>(x[13]);
    x[6] = tw16<INV, 2>(x[6]);  x[10] = tw16<INV, 4>(x[10]); x[14] = tw16<INV, 6>(x[14]);
    x[7] = tw16<INV, 3>(x[7]);  x[11] = tw16<INV, 6>(x[11]); x[15] = tw16<INV, 9>(x[15]);
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1) dft4<INV>(x[4 * k1], x[4 * k1 + 1], x[4 * k1 + 2], x[4 * k1 + 3]);
    // slot 4*k1 + k2 holds X[k1 + 4*k2]: transpose 4x4 to natural order
    float2 t[16];
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1)
#pragma unroll
        for (int k2 = 0; k2 < 4; ++k2) t[k1 + 4 * k2] = x[4 * k1 + k2];
#pragma unroll
    for (int i = 0; i < 16; ++i) x[i] = t[i];
}

template <int L, bool INV>
__device__ __forceinline__ void dftL(float2 *x) {
    if constexpr (L == 16) dft16<INV>(x);
    else if constexpr (L == 8) dft8<INV>(x);
    else static_assert(L < 0, "unsupported radix");
}

// cos(2 pi j / 32) and multiplication by W32^j (forward sign; INV conjugates).
// Called with j a compile-time constant after unrolling, so it folds to
// constants, and the trivial angles cost no multiplication.
__device__ __forceinline__ constexpr float cos32(int j) {
    j &= 31;
    const int a = j <= 8 ? j : j <= 16 ? 16 - j : j <= 24 ? j - 16 : 32 - j;
    const float c = a == 0 ? 1.0f : a == 1 ? 0.98078528040323043f : a == 2 ? 0.92387953251128674f
                  : a == 3 ? 0.83146961230254524f : a == 4 ? 0.70710678118654752f : a == 5 ? 0.55557023301960218f
                  : a == 6 ? 0.38268343236508977f : a == 7 ? 0.19509032201612825f : 0.0f;
    return (j <= 8 || j >= 24) ? c : -c;
}

template <bool INV>
__device__ __forceinline__ float2 tw32(float2 a, int j) {
    j &= 31;
    if (j == 0) return a;
    if (j == 16) return make_float2(-a.x, -a.y);
    if (j == 8) return INV ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);     // * -i (fwd)
    if (j == 24) return INV ? make_float2(a.y, -a.x) : make_float2(-a.y, a.x);
    const float c = cos32(j), s = cos32(j - 8);   // sin(2 pi j / 32)
    return cmul(a, make_float2(c, INV ? s : -s));
}

// --------------------------------------------------------------- addressing
// Every shared-memory access below is (per-thread base) + (compile-time
// offset), so the compiler keeps a handful of base registers instead of one
// address per element.
//
// Line exchange (the NT threads of one row / column): line L starts at L*LS
// with LS = N + 8 complex, so the two lines a half-warp touches sit in
// opposite 64-byte halves of the bank space; inside a line, element
// (thread jj, k1) lives at k1*NT + (jj ^ k1/P).
//
// Transpose tile: (r, c) at r*N + (c ^ g(r)); for every access pattern used
// here g(r) depends only on per-thread bits, so the XOR folds into the base.
template <int N>
struct Lay;

template <>
struct Lay<128> {
    static constexpr int S1 = 33, S2 = 17;   // row strides of exchanges 1 and 2
    static constexpr int BUF = 1024 * S2;    // complex elements of the exchange buffer (>= 512 * S1)
};
template <>
struct Lay<256> {
    static constexpr int BUF = Lay<128>::BUF;   // the 128 x 128 part's exchanges; also holds the
                                                // 16384 values a CTA publishes to its cluster
};

template <int N>
struct Lay {
    using C = FFTCfg<N>;
    static constexpr int E = C::E, NT = C::NT, P = C::P, U = C::U;
    static constexpr int LS = N + 8;                    // padded line stride
    static constexpr int BUF = N * LS;                  // complex elements of the exchange buffer
    static __device__ __forceinline__ int g(int r) {
        if constexpr (N == 128) return (2 * r + (r & 1)) & 15;
        else return ((r & 1) << 3) | (r & 6);
    }
};

// twiddle table, TileCfg<N>::TW entries: N = 128: twid[j] = exp(-2 pi i j / 128);
// N = 64: twid[k1 * NT + jj] = exp(-2 pi i jj k1 / 64);
// N = 256: the N = 128 table, then twid[128 + j] = exp(-2 pi i j / 256)
template <int N>
__device__ __forceinline__ void fft_init_twiddles(float2 *twid) {
    for (int i = threadIdx.x; i < TileCfg<N>::TW; i += blockDim.x) {
        int e, n;
        if constexpr (N == 256) {
            e = i < 128 ? i : i - 128;
            n = i < 128 ? 128 : 256;
        } else if constexpr (N == 128) {
            e = i;
            n = 128;
        } else {
            e = (i % FFTCfg<N>::NT) * (i / FFTCfg<N>::NT);
            n = N;
        }
        float s, c;
        sincospif(-2.0f * (float)e / (float)n, &s, &c);
        twid[i] = make_float2(c, s);
    }
}

// ------------------------------------------------- N = 128: two-exchange form
// Forward: R layout in, K layout out.
__device__ __forceinline__ void fft128_r2k(float2 (&v)[1][32], float2 *xb, const float2 *twid) {
    static_assert(FFT_THREADS == 512, "the 128-point transform is laid out for 512 threads");
    constexpr int S1 = Lay<128>::S1, S2 = Lay<128>::S2;
    const int t = threadIdx.x;
    float2 *x = v[0];
    {   // pass A: thread (xt, yt), slot 8 j + m
        const int xt = t & 31, yt = t >> 5;
#pragma unroll
        for (int m = 0; m < 8; ++m) dft4<false>(x[m], x[8 + m], x[16 + m], x[24 + m]);   // j -> k1
        float2 wy[8];
#pragma unroll
        for (int ky2 = 1; ky2 < 8; ++ky2) wy[ky2] = twid[yt * ky2];
        float2 *wb = xb + yt * S1 + xt;                     // row yt + 16 (ky2 + 8 k1)
        // each k1 group is finished and stored before the next is transformed, so the
        // exchange stores of one group overlap the arithmetic of the next
#pragma unroll
        for (int k1 = 0; k1 < 4; ++k1) {
            dft8<false>(&x[8 * k1]);                                                     // m -> ky2
            if (k1 > 0) {
                const float2 w = twid[xt * k1];
#pragma unroll
                for (int ky2 = 0; ky2 < 8; ++ky2) x[8 * k1 + ky2] = cmul(x[8 * k1 + ky2], w);
            }
#pragma unroll
            for (int ky2 = 1; ky2 < 8; ++ky2) x[8 * k1 + ky2] = cmul(x[8 * k1 + ky2], wy[ky2]);
#pragma unroll
            for (int ky2 = 0; ky2 < 8; ++ky2) wb[16 * (ky2 + 8 * k1) * S1] = x[8 * k1 + ky2];
        }
    }
    __syncthreads();
    {   // pass B: this thread's row t, DFT-32 over xt
        const float2 *rb = xb + t * S1;
#pragma unroll
        for (int i = 0; i < 32; ++i) x[i] = rb[i];
    }
    __syncthreads();
    {   // DFT-32 (n = n2 + 8 n1, k = k1' + 4 k2') with each DFT-8 group's outputs stored as
        // soon as they are final: row 128 ky2 + kx, kx = k1 + 4 k, k = k1' + 4 k2'
        const int yt = t & 15, ky2 = (t >> 4) & 7, k1 = t >> 7;
        float2 *wb = xb + (ky2 * 128 + k1) * S2 + yt;
#pragma unroll
        for (int n2 = 0; n2 < 8; ++n2) dft4<false>(x[n2], x[n2 + 8], x[n2 + 16], x[n2 + 24]);
#pragma unroll
        for (int g = 1; g < 4; ++g)
#pragma unroll
            for (int n2 = 1; n2 < 8; ++n2) x[n2 + 8 * g] = tw32<false>(x[n2 + 8 * g], n2 * g);
#pragma unroll
        for (int g = 0; g < 4; ++g) {
            dft8<false>(&x[8 * g]);                           // slot 8 g + k2' holds X[g + 4 k2']
#pragma unroll
            for (int k2 = 0; k2 < 8; ++k2) wb[4 * (g + 4 * k2) * S2] = x[8 * g + k2];
        }
    }
    __syncthreads();
    {   // pass C: DFT-16 over yt for two columns
        const float2 *rb = xb + ((t >> 6) * 128 + (t & 63)) * S2;
#pragma unroll
        for (int c = 0; c < 2; ++c)
#pragma unroll
            for (int y = 0; y < 16; ++y) x[16 * c + y] = rb[64 * c * S2 + y];
    }
    dft16<false>(&x[0]);
    dft16<false>(&x[16]);
    __syncthreads();   // every read of the exchange buffer is done before its next writer
}

// Inverse (unnormalised): K layout in, R layout out.
__device__ __forceinline__ void fft128_k2r(float2 (&v)[1][32], float2 *xb, const float2 *twid) {
    constexpr int S1 = Lay<128>::S1, S2 = Lay<128>::S2;
    const int t = threadIdx.x;
    float2 *x = v[0];
    {   // pass C: ky1 -> yt, each column stored once transformed
        float2 *wb = xb + ((t >> 6) * 128 + (t & 63)) * S2;
#pragma unroll
        for (int c = 0; c < 2; ++c) {
            dft16<true>(&x[16 * c]);
#pragma unroll
            for (int y = 0; y < 16; ++y) wb[64 * c * S2 + y] = x[16 * c + y];
        }
    }
    __syncthreads();
    {   // pass B: k2 -> xt
        const int yt = t & 15, ky2 = (t >> 4) & 7, k1 = t >> 7;
        const float2 *rb = xb + (ky2 * 128 + k1) * S2 + yt;
#pragma unroll
        for (int k2 = 0; k2 < 32; ++k2) x[k2] = rb[4 * k2 * S2];
    }
    __syncthreads();
    {   // inverse DFT-32, each DFT-8 group's outputs stored as soon as they are final
        float2 *wb = xb + t * S1;
#pragma unroll
        for (int n2 = 0; n2 < 8; ++n2) dft4<true>(x[n2], x[n2 + 8], x[n2 + 16], x[n2 + 24]);
#pragma unroll
        for (int g = 1; g < 4; ++g)
#pragma unroll
            for (int n2 = 1; n2 < 8; ++n2) x[n2 + 8 * g] = tw32<true>(x[n2 + 8 * g], n2 * g);
#pragma unroll
        for (int g = 0; g < 4; ++g) {
            dft8<true>(&x[8 * g]);                            // slot 8 g + k2' holds X[g + 4 k2']
#pragma unroll
            for (int k2 = 0; k2 < 8; ++k2) wb[g + 4 * k2] = x[8 * g + k2];
        }
    }
    __syncthreads();
    {   // pass A: conj twiddles, ky2 -> m, k1 -> j
        const int xt = t & 31, yt = t >> 5;
        const float2 *rb = xb + yt * S1 + xt;
        float2 wy[8];
#pragma unroll
        for (int ky2 = 1; ky2 < 8; ++ky2) wy[ky2] = twid[yt * ky2];
        // group by group: the exchange loads of the next k1 group overlap this group's arithmetic
#pragma unroll
        for (int k1 = 0; k1 < 4; ++k1) {
#pragma unroll
            for (int ky2 = 0; ky2 < 8; ++ky2) x[8 * k1 + ky2] = rb[16 * (ky2 + 8 * k1) * S1];
#pragma unroll
            for (int ky2 = 1; ky2 < 8; ++ky2) x[8 * k1 + ky2] = cmulc(x[8 * k1 + ky2], wy[ky2]);
            if (k1 > 0) {
                const float2 w = twid[xt * k1];
#pragma unroll
                for (int ky2 = 0; ky2 < 8; ++ky2) x[8 * k1 + ky2] = cmulc(x[8 * k1 + ky2], w);
            }
            dft8<true>(&x[8 * k1]);                                                      // ky2 -> m
        }
        __syncthreads();
#pragma unroll
        for (int m = 0; m < 8; ++m) dft4<true>(x[m], x[8 + m], x[16 + m], x[24 + m]);    // k1 -> j
    }
}

// ------------------------------------------------- N = 256: 4-CTA cluster form
// Decimation in time across the cluster.  In real space the CTA of rank r = 2a + b holds
// the polyphase component x[2y' + a][2x' + b] in the N = 128 R layout of (y', x'), and its
// own 128 x 128 transform gives Y_ab[ky'][kx'] in the N = 128 K layout.  Then
//   X[ky' + 128p][kx' + 128q] = sum_ab (-1)^(ap + bq) W256^(a ky' + b kx') Y_ab[ky'][kx'],
// so one output point needs the four CTAs' values at the same (ky', kx').  Rank r takes the
// points of register slots 8r .. 8r + 7 (a quarter of the spectrum) from all four CTAs --
// one all-to-all through distributed shared memory, 3 x 32 KB of remote reads per CTA --
// and keeps the four outputs: slot 8 (2p + q) + j of thread t holds X[ky' + 128p][kx' + 128q]
// for (ky', kx') = the N = 128 K-layout point of slot 8r + j.  The inverse runs the
// butterflies first (conjugate twiddles), the all-to-all back, then the 128 x 128 inverse.
// Each exchange: publish (two register slots per float4), cluster barrier, read, cluster
// barrier (no CTA rewrites its buffer before the others have read it).
__device__ __forceinline__ void quad_a2a_fwd(float2 (&v)[1][32], float2 *xb, const float2 *tw256) {
    namespace cg = cooperative_groups;
    cg::cluster_group cl = cg::this_cluster();
    const int t = threadIdx.x, r = cluster_rank() & 3;
    float2 *x = v[0];
    float4 *mine = reinterpret_cast<float4 *>(xb);
#pragma unroll
    for (int i = 0; i < 16; ++i) mine[i * 512 + t] = make_float4(x[2 * i].x, x[2 * i].y, x[2 * i + 1].x, x[2 * i + 1].y);
    cl.sync();
    float2 y[4][8];   // [source rank ab][point j]
#pragma unroll
    for (int ab = 0; ab < 4; ++ab) {
        const float4 *src = cl.map_shared_rank(mine, ab) + 4 * r * 512 + t;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const float4 p = src[i * 512];
            y[ab][2 * i] = make_float2(p.x, p.y);
            y[ab][2 * i + 1] = make_float2(p.z, p.w);
        }
    }
    cl.sync();
    const int ky0 = (t >> 6) + 64 * (r & 1), kx = (t & 63) + 64 * (r >> 1);   // point j: ky' = ky0 + 8 j
    const float2 wx = tw256[kx];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const int ky = ky0 + 8 * j;
        const float2 y0 = y[0][j], y1 = cmul(y[1][j], wx), y2 = cmul(y[2][j], tw256[ky]),
                     y3 = cmul(y[3][j], tw256[ky + kx]);   // ky + kx <= 254
        const float2 s02 = cadd(y0, y2), d02 = csub(y0, y2), s13 = cadd(y1, y3), d13 = csub(y1, y3);
        x[j] = cadd(s02, s13);        // (p, q) = (0, 0)
        x[8 + j] = csub(s02, s13);    // (0, 1)
        x[16 + j] = cadd(d02, d13);   // (1, 0)
        x[24 + j] = csub(d02, d13);   // (1, 1)
    }
}

__device__ __forceinline__ void quad_a2a_inv(float2 (&v)[1][32], float2 *xb, const float2 *tw256) {
    namespace cg = cooperative_groups;
    cg::cluster_group cl = cg::this_cluster();
    const int t = threadIdx.x, r = cluster_rank() & 3;
    float2 *x = v[0];
    const int ky0 = (t >> 6) + 64 * (r & 1), kx = (t & 63) + 64 * (r >> 1);
    const float2 wx = tw256[kx];
    float2 y[4][8];   // [destination rank ab][point j]
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const int ky = ky0 + 8 * j;
        const float2 X0 = x[j], X1 = x[8 + j], X2 = x[16 + j], X3 = x[24 + j];
        const float2 s02 = cadd(X0, X2), d02 = csub(X0, X2), s13 = cadd(X1, X3), d13 = csub(X1, X3);
        y[0][j] = cadd(s02, s13);
        y[1][j] = cmulc(csub(s02, s13), wx);
        y[2][j] = cmulc(cadd(d02, d13), tw256[ky]);
        y[3][j] = cmulc(csub(d02, d13), tw256[ky + kx]);
    }
    float4 *mine = reinterpret_cast<float4 *>(xb);
#pragma unroll
    for (int ab = 0; ab < 4; ++ab)
#pragma unroll
        for (int i = 0; i < 4; ++i)
            mine[(4 * ab + i) * 512 + t] = make_float4(y[ab][2 * i].x, y[ab][2 * i].y, y[ab][2 * i + 1].x,
                                                       y[ab][2 * i + 1].y);
    cl.sync();
#pragma unroll
    for (int src_r = 0; src_r < 4; ++src_r) {
        const float4 *src = cl.map_shared_rank(mine, src_r) + 4 * r * 512 + t;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const float4 p = src[i * 512];
            x[8 * src_r + 2 * i] = make_float2(p.x, p.y);
            x[8 * src_r + 2 * i + 1] = make_float2(p.z, p.w);
        }
    }
    cl.sync();
}

// Forward 256 x 256 (cluster of 4): polyphase component in R layout -> spectrum quarter.
__device__ __forceinline__ void fft256_r2k(float2 (&v)[1][32], float2 *xb, const float2 *twid) {
    fft128_r2k(v, xb, twid);
    quad_a2a_fwd(v, xb, twid + 128);
}

// Inverse (unnormalised): spectrum quarter -> polyphase component in R layout.
__device__ __forceinline__ void ifft256_k2r(float2 (&v)[1][32], float2 *xb, const float2 *twid) {
    quad_a2a_inv(v, xb, twid + 128);
    fft128_k2r(v, xb, twid);
}

// ----------------------------------------------------------------- line passes
template <int N>
__device__ __forceinline__ void line_pass_fwd(float2 (&v)[FFTCfg<N>::U][FFTCfg<N>::E], float2 *xb,
                                              const float2 *twid) {
    using Ly = Lay<N>;
    constexpr int E = Ly::E, NT = Ly::NT, P = Ly::P, U = Ly::U, LS = Ly::LS;
    const int rsel = threadIdx.x >> 3, jl = threadIdx.x & 7;
    const float2 *tw = twid + jl;
    float2 *lb = xb + rsel * LS;
#pragma unroll
    for (int u = 0; u < U; ++u) {
        dftL<E, false>(v[u]);
#pragma unroll
        for (int k1 = 1; k1 < E; ++k1) v[u][k1] = cmul(v[u][k1], tw[k1 * NT]);
#pragma unroll
        for (int k1 = 0; k1 < E; ++k1) lb[RPP * u * LS + k1 * NT + (jl ^ (k1 / P))] = v[u][k1];
    }
    __syncthreads();
    const float2 *rb = xb + rsel * LS + jl * P * NT;
#pragma unroll
    for (int u = 0; u < U; ++u)
#pragma unroll
        for (int p = 0; p < P; ++p)
#pragma unroll
            for (int jj = 0; jj < NT; ++jj) v[u][p * NT + jj] = rb[RPP * u * LS + p * NT + (jj ^ jl)];
    __syncthreads();
#pragma unroll
    for (int u = 0; u < U; ++u)
#pragma unroll
        for (int p = 0; p < P; ++p) dftL<NT, false>(&v[u][p * NT]);
}

template <int N>
__device__ __forceinline__ void line_pass_inv(float2 (&v)[FFTCfg<N>::U][FFTCfg<N>::E], float2 *xb,
                                              const float2 *twid) {
    using Ly = Lay<N>;
    constexpr int E = Ly::E, NT = Ly::NT, P = Ly::P, U = Ly::U, LS = Ly::LS;
    const int rsel = threadIdx.x >> 3, jl = threadIdx.x & 7;
    float2 *wb = xb + rsel * LS + jl * P * NT;
#pragma unroll
    for (int u = 0; u < U; ++u)
#pragma unroll
        for (int p = 0; p < P; ++p) {
            dftL<NT, true>(&v[u][p * NT]);
#pragma unroll
            for (int jj = 0; jj < NT; ++jj) wb[RPP * u * LS + p * NT + (jj ^ jl)] = v[u][p * NT + jj];
        }
    __syncthreads();
    const float2 *lb = xb + rsel * LS;
#pragma unroll
    for (int u = 0; u < U; ++u)
#pragma unroll
        for (int k1 = 0; k1 < E; ++k1) v[u][k1] = lb[RPP * u * LS + k1 * NT + (jl ^ (k1 / P))];
    __syncthreads();
    const float2 *tw = twid + jl;
#pragma unroll
    for (int u = 0; u < U; ++u) {
#pragma unroll
        for (int k1 = 1; k1 < E; ++k1) v[u][k1] = cmulc(v[u][k1], tw[k1 * NT]);
        dftL<E, true>(v[u]);
    }
}

// row-pass output (K form of rows) -> column-pass input (R form of columns), and back.
// Row r = rsel + RPP*u holds kx = (jl*P + p) + E*k2; column c = rsel + RPP*u holds rows jl + NT*q.
// tile(r, c) = r*N + (c ^ g(r)); g(rsel + RPP*u) == g(rsel) and g(jl + NT*q) == g(jl).
template <int N, bool TO_COLUMNS>
__device__ __forceinline__ void transpose(float2 (&v)[FFTCfg<N>::U][FFTCfg<N>::E], float2 *xb) {
    using Ly = Lay<N>;
    constexpr int E = Ly::E, NT = Ly::NT, P = Ly::P, U = Ly::U;
    const int rsel = threadIdx.x >> 3, jl = threadIdx.x & 7;
    // row side: element (u, p, k2) at rsel*N + RPP*u*N + (((jl*P + p) + E*k2) ^ gr)
    const int gr = Ly::g(rsel);
    // column side: element (u, q) at jl*N + NT*q*N + ((rsel + RPP*u) ^ gc)
    const int gc = Ly::g(jl);
    float2 *rowb = xb + rsel * N;
    float2 *colb = xb + jl * N + (rsel ^ gc);           // gc < 16 <= RPP: (rsel + RPP*u) ^ gc = (rsel ^ gc) + RPP*u
    if constexpr (TO_COLUMNS) {
#pragma unroll
        for (int u = 0; u < U; ++u)
#pragma unroll
            for (int p = 0; p < P; ++p) {
                if constexpr (N == 128) {   // gr < E: the XOR stays inside the low 4 bits
                    float2 *b = rowb + RPP * u * N + ((jl * P + p) ^ gr);
#pragma unroll
                    for (int k2 = 0; k2 < NT; ++k2) b[E * k2] = v[u][p * NT + k2];
                } else {                    // E == 8: bit 3 of gr flips bit 0 of k2
                    const int hb = gr >> 3;
                    float2 *b = rowb + RPP * u * N + ((jl * P + p) ^ (gr & 7));
#pragma unroll
                    for (int k2 = 0; k2 < NT; ++k2) b[E * (k2 ^ hb)] = v[u][p * NT + k2];
                }
            }
        __syncthreads();
#pragma unroll
        for (int u = 0; u < U; ++u)
#pragma unroll
            for (int q = 0; q < E; ++q) v[u][q] = colb[NT * q * N + RPP * u];
        __syncthreads();
    } else {
#pragma unroll
        for (int u = 0; u < U; ++u)
#pragma unroll
            for (int q = 0; q < E; ++q) colb[NT * q * N + RPP * u] = v[u][q];
        __syncthreads();
#pragma unroll
        for (int u = 0; u < U; ++u)
#pragma unroll
            for (int p = 0; p < P; ++p) {
                if constexpr (N == 128) {
                    const float2 *b = rowb + RPP * u * N + ((jl * P + p) ^ gr);
#pragma unroll
                    for (int k2 = 0; k2 < NT; ++k2) v[u][p * NT + k2] = b[E * k2];
                } else {
                    const int hb = gr >> 3;
                    const float2 *b = rowb + RPP * u * N + ((jl * P + p) ^ (gr & 7));
#pragma unroll
                    for (int k2 = 0; k2 < NT; ++k2) v[u][p * NT + k2] = b[E * (k2 ^ hb)];
                }
            }
        __syncthreads();
    }
}

template <int N>
__device__ __forceinline__ void transpose_rk(float2 (&v)[FFTCfg<N>::U][FFTCfg<N>::E], float2 *xb) {
    transpose<N, true>(v, xb);
}
template <int N>
__device__ __forceinline__ void transpose_kr(float2 (&v)[FFTCfg<N>::U][FFTCfg<N>::E], float2 *xb) {
    transpose<N, false>(v, xb);
}

// Forward 2D DFT: R layout in, K layout out.
template <int N>
__device__ __forceinline__ void fft2_r2k(float2 (&v)[FFTCfg<N>::U][FFTCfg<N>::E], float2 *xb,
                                         const float2 *twid) {
    if constexpr (N == 256) {
        fft256_r2k(v, xb, twid);
    } else if constexpr (N == 128) {
        fft128_r2k(v, xb, twid);
    } else {
        line_pass_fwd<N>(v, xb, twid);
        transpose_rk<N>(v, xb);
        line_pass_fwd<N>(v, xb, twid);
    }
}

// Inverse 2D DFT (unnormalised): K layout in, R layout out.
template <int N>
__device__ __forceinline__ void ifft2_k2r(float2 (&v)[FFTCfg<N>::U][FFTCfg<N>::E], float2 *xb,
                                          const float2 *twid) {
    if constexpr (N == 256) {
        ifft256_k2r(v, xb, twid);
    } else if constexpr (N == 128) {
        fft128_k2r(v, xb, twid);
    } else {
        line_pass_inv<N>(v, xb, twid);
        transpose_kr<N>(v, xb);
        line_pass_inv<N>(v, xb, twid);
    }
}

// ------------------------------------------------------------- index helpers
// R layout: element (u, q) of a thread is pixel (row(u, q), col(u, q)), offset (drow(q), dcol(q))
// from element (u, 0).
// K layout: element (u, e) is frequency (ky(u, e), kx(u, e)).
// flat(u, e): register-order index (coalesced per warp), used for scratch and packed tables.
template <int N>
struct Idx;

template <>
struct Idx<128> {
    static constexpr int U = 1, E = 32;
    static __device__ __forceinline__ int row(int, int q) { return (threadIdx.x >> 5) + 16 * (q & 7); }
    static __device__ __forceinline__ int col(int, int q) { return (threadIdx.x & 31) + 32 * (q >> 3); }
    // offsets of element q from element 0 of the same u: rows and columns (compile-time)
    static __host__ __device__ __forceinline__ constexpr int drow(int q) { return 16 * (q & 7); }
    static __host__ __device__ __forceinline__ constexpr int dcol(int q) { return 32 * (q >> 3); }
    static __device__ __forceinline__ int kx(int, int e) { return (threadIdx.x & 63) + 64 * (e >> 4); }
    static __device__ __forceinline__ int ky(int, int e) { return (threadIdx.x >> 6) + 8 * (e & 15); }
    static __device__ __forceinline__ int flat(int u, int e) { return (u * E + e) * FFT_THREADS + threadIdx.x; }
    static __host__ __device__ __forceinline__ void rc_of(int t, int u, int q, int &r, int &c) {
        (void)u;
        r = (t >> 5) + 16 * (q & 7);
        c = (t & 31) + 32 * (q >> 3);
    }
    static __host__ __device__ __forceinline__ void k_of(int t, int u, int e, int &ky_, int &kx_) {
        (void)u;
        kx_ = (t & 63) + 64 * (e >> 4);
        ky_ = (t >> 6) + 8 * (e & 15);
    }
};

template <>
struct Idx<64> {
    using C = FFTCfg<64>;
    static constexpr int E = C::E, NT = C::NT, P = C::P, U = C::U;
    static __device__ __forceinline__ int row(int u, int) { return (threadIdx.x >> 3) + RPP * u; }
    static __device__ __forceinline__ int col(int, int q) { return (threadIdx.x & 7) + NT * q; }
    static __host__ __device__ __forceinline__ constexpr int drow(int) { return 0; }
    static __host__ __device__ __forceinline__ constexpr int dcol(int q) { return NT * q; }
    static __device__ __forceinline__ int kx(int u, int) { return (threadIdx.x >> 3) + RPP * u; }
    static __device__ __forceinline__ int ky(int, int e) { return ((threadIdx.x & 7) * P + e / NT) + E * (e % NT); }
    static __device__ __forceinline__ int flat(int u, int e) { return (u * E + e) * FFT_THREADS + threadIdx.x; }
    static __host__ __device__ __forceinline__ void rc_of(int t, int u, int q, int &r, int &c) {
        r = (t >> 3) + RPP * u;
        c = (t & 7) + NT * q;
    }
    static __host__ __device__ __forceinline__ void k_of(int t, int u, int e, int &ky_, int &kx_) {
        kx_ = (t >> 3) + RPP * u;
        ky_ = ((t & 7) * P + e / NT) + E * (e % NT);
    }
};

// N = 256: the CTA of cluster rank r = 2 a + b holds the polyphase component (a, b) in real
// space (pixel (2 y' + a, 2 x' + b) where the N = 128 R layout has (y', x')) and a quarter of
// the spectrum in Fourier space (slot 8 (2p + q) + j: (ky' + 128 p, kx' + 128 q) where the
// N = 128 K layout has (ky', kx') at slot 8 r + j); register-order flat indices are CTA-major
// (r * 16384 + the N = 128 flat index).
template <>
struct Idx<256> {
    using B = Idx<128>;
    static constexpr int U = 1, E = 32;
    static __device__ __forceinline__ int quad() { return cluster_rank() & 3; }
    static __device__ __forceinline__ int row(int u, int q) { return 2 * B::row(u, q) + (quad() >> 1); }
    static __device__ __forceinline__ int col(int u, int q) { return 2 * B::col(u, q) + (quad() & 1); }
    static __host__ __device__ __forceinline__ constexpr int drow(int q) { return 2 * B::drow(q); }
    static __host__ __device__ __forceinline__ constexpr int dcol(int q) { return 2 * B::dcol(q); }
    static __host__ __device__ __forceinline__ void k_of(int t, int r, int e, int &ky_, int &kx_) {
        ky_ = (t >> 6) + 64 * (r & 1) + 8 * (e & 7) + 128 * (e >> 4);
        kx_ = (t & 63) + 64 * (r >> 1) + 128 * ((e >> 3) & 1);
    }
    static __device__ __forceinline__ int ky(int, int e) {
        return (threadIdx.x >> 6) + 64 * (quad() & 1) + 8 * (e & 7) + 128 * (e >> 4);
    }
    static __device__ __forceinline__ int kx(int, int e) {
        return (threadIdx.x & 63) + 64 * (quad() >> 1) + 128 * ((e >> 3) & 1);
    }
    static __device__ __forceinline__ int flat(int u, int e) { return (quad() << 14) + B::flat(u, e); }
};

// decode a register-order flat index (from any thread) to (row, col) in R layout
template <int N>
__device__ __forceinline__ void flat_to_rc(int f, int &r, int &c) {
    if constexpr (N == 256) {
        const int q = f >> 14;
        flat_to_rc<128>(f & 16383, r, c);
        r = 2 * r + (q >> 1);
        c = 2 * c + (q & 1);
    } else {
        const int t = f % FFT_THREADS, s = f / FFT_THREADS;   // s = u*E + q
        Idx<N>::rc_of(t, s / FFTCfg<N>::E, s % FFTCfg<N>::E, r, c);
    }
}
// ... and to (ky, kx) in K layout
template <int N>
__device__ __forceinline__ void flat_to_k(int f, int &ky, int &kx) {
    if constexpr (N == 256) {
        const int g = f & 16383;
        Idx<256>::k_of(g % FFT_THREADS, f >> 14, g / FFT_THREADS, ky, kx);
    } else {
        const int t = f % FFT_THREADS, s = f / FFT_THREADS;
        Idx<N>::k_of(t, s / FFTCfg<N>::E, s % FFTCfg<N>::E, ky, kx);
    }
}

}  // namespace phb
