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

// ------------------------------------------- tensor-core implicit GEMM (tcgen05)
// A 3x3 convolution as nine shifted GEMMs on the 5th-generation tensor cores:
// D[m][c] = sum_tap sum_k A_tap[m][k] B_tap[c][k], m = 128 output pixels of one image per
// CTA (UMMA M = 128), c = the output channels (UMMA N = 32 or 64; the accumulator is a
// 128 x N float32 tile in tensor memory), k = 16 reduction channels per MMA.
//
// Pixels are numbered on a padded grid of pitch Wp: output pixel (y, x) is row
// q = (y + 1) Wp + (x + 1).  A CTA stages, once per chunk of 16 reduction channels, the
// rows its 128 outputs read -- for stride 1 the input plane itself (rows q0 - Wp - 1 ..
// q0 + 128 + Wp), for stride 2 its four polyphase components in[2i + py][2j + px] (rows
// q0 - Wp - 1 .. q0 + 127 each) -- as bf16 rows of 16 channels.  Every tap then reads
// the same staged rows shifted by a constant (dy Wp + dx rows), which in the operand
// layout (K-major, no swizzle: row r at 16 r bytes, the two 8-channel halves of a row
// R * 16 bytes apart) is only a different start address of the matrix descriptor, so
// each staged value serves all nine taps.
//
// Precision: the weights are bf16 already; each float32 activation is split into bf16
// hi + bf16 lo and both parts are multiplied (two MMAs per tap into the same
// accumulator), so the products keep ~16 mantissa bits of the activation and the
// results match the FP32 kernels' float32-activation / bf16-weight / float32-accumulate
// definition to ~1e-5.  Chunks are double buffered (the CTA stages chunk c + 1 while the
// tensor cores run chunk c; tcgen05.commit arrives on an mbarrier per buffer), and every
// wait is bounded.
//
// MODE 0: forward, stride 1 or 2 (out = conv(in, w) + bias, optional ReLU).
// MODE 1: data gradient at stride 1 (din[ci][Y][X] = sum w[co][ci][ky][kx] dout[co][Y+1-ky][X+1-kx]:
//         the tap offsets mirrored and the channel roles exchanged).
// MODE 2: data gradient at stride 2, one output parity class (py, px) per CTA (blockIdx.x % 4):
//         din[ci][2Y + py][2X + px] = sum over the class's taps of w[co][ci][ky][kx]
//         dout[co][Y + dy][X + dx], ky = 1 (dy = 0) for py = 0 and ky = 0 (dy = 1) or 2 (dy = 0)
//         for py = 1, the same for x: a convolution of dout with 1, 2 or 4 taps on the
//         dout grid (pitch Wo + 1, halo row and column after the image).
namespace tc {
constexpr int BM = 128;                 // output pixels (padded-grid rows) per CTA
constexpr int CC = 16;                  // reduction channels per chunk (one MMA K)
constexpr int THREADS = 256;
constexpr long long WAIT_LIMIT = 1ll << 22;   // try_wait attempts before a wait is abandoned
__host__ __device__ constexpr int pitch(int S, int Wo) { return S == 1 ? Wo + 2 : Wo + 1; }
// staged rows per phase
__host__ __device__ constexpr int rows(int S, int Wp) { return S == 1 ? BM + 2 * Wp + 2 : BM + Wp + 1; }
__host__ __device__ constexpr int phases(int S, int MODE = 0) { return S == 2 && MODE == 0 ? 4 : 1; }
template <int NT> struct B_ { static constexpr int BYTES = 9 * NT * CC * 2; };
// bytes of one stage: A (phases x rows x 16 channels x bf16, hi and lo) + B (9 taps x NT x 16)
__host__ __device__ constexpr int a_bytes(int S, int Wp, int MODE = 0) { return phases(S, MODE) * rows(S, Wp) * CC * 2; }
}  // namespace tc

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// shared-memory matrix descriptor: K-major, no swizzle, sm_100 descriptor version 1;
// rows 16 bytes apart (SBO 128 bytes per 8-row group), the two K halves `lbo` bytes apart
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)(128u >> 4) << 32) | ((uint64_t)1 << 46);
}
// instruction descriptor of kind::f16: D float32, A and B bf16, both K-major, M x N
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}
__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
    const uint32_t z = 0;
    asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
                 :: "r"(tmem_d), "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(z), "r"(z), "r"(z), "r"(z));
}
__device__ __forceinline__ void umma_commit(uint64_t *mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 :: "r"(smem_u32(mbar)) : "memory");
}
__device__ __forceinline__ bool mbar_wait(uint64_t *mbar, uint32_t parity, long long limit = tc::WAIT_LIMIT) {
    const uint32_t addr = smem_u32(mbar);
    for (long long i = 0; i < limit; ++i) {
        uint32_t done;
        asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                     "selp.u32 %0, 1, 0, p;\n\t}\n" : "=r"(done) : "r"(addr), "r"(parity) : "memory");
        if (done) return true;
    }
    return false;
}
// Failure-detection probe of the bounded wait above: one thread waits on an mbarrier of
// arrival count 1 that nothing completes (arrive == 0; the wait gives up after `limit`
// attempts) or that its own arrival completed first (arrive == 1).  out[0] = 1 if the
// wait saw phase 0 complete, 0 if it gave up.
__global__ void k_wait_probe(int arrive, long long limit, int32_t *out) {
    __shared__ uint64_t mbar;
    const uint32_t addr = smem_u32(&mbar);
    if (threadIdx.x == 0) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(addr) : "memory");
    __syncthreads();
    if (threadIdx.x == 0) {
        if (arrive) {
            uint64_t state;
            asm volatile("mbarrier.arrive.shared::cta.b64 %0, [%1];" : "=l"(state) : "r"(addr) : "memory");
        }
        out[0] = mbar_wait(&mbar, 0, limit) ? 1 : 0;
    }
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// named barrier `id` over `nthreads` threads (a multiple of 32) that also ANDs `v` over them
__device__ __forceinline__ bool bar_and(int id, int nthreads, bool v) {
    uint32_t r;
    asm volatile("{\n\t.reg .pred p, q;\n\tsetp.ne.u32 p, %1, 0;\n\tbar.red.and.pred q, %2, %3, p;\n\t"
                 "selp.u32 %0, 1, 0, q;\n\t}\n" : "=r"(r) : "r"((uint32_t)v), "r"(id), "r"(nthreads) : "memory");
    return r != 0;
}

__device__ __forceinline__ uint32_t pack_bf16(__nv_bfloat16 a, __nv_bfloat16 b) {
    return (uint32_t)__bfloat16_as_ushort(a) | ((uint32_t)__bfloat16_as_ushort(b) << 16);
}

// split 8 float32 values into bf16 hi and lo rows
__device__ __forceinline__ void split_row(const float (&vals)[8], uint4 &hi, uint4 &lo) {
    uint32_t h[4], l[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const __nv_bfloat16 h0 = __float2bfloat16_rn(vals[2 * j]), h1 = __float2bfloat16_rn(vals[2 * j + 1]);
        h[j] = pack_bf16(h0, h1);
        l[j] = pack_bf16(__float2bfloat16_rn(vals[2 * j] - __bfloat162float(h0)),
                         __float2bfloat16_rn(vals[2 * j + 1] - __bfloat162float(h1)));
    }
    hi = make_uint4(h[0], h[1], h[2], h[3]);
    lo = make_uint4(l[0], l[1], l[2], l[3]);
}

// src (Nb, Cr, Hs, Ws) -> out (Nb, Ncol, Ho, Wo); tiles of 128 padded-grid rows, T per image
template <int NT, int S, int MODE>
__global__ void __launch_bounds__(tc::THREADS) k_conv_tc(const float *src, const __nv_bfloat16 *w, const float *bias,
                                                         float *out, int Cr, int Ncol, int Hs, int Ws, int Ho, int Wo,
                                                         int Ci_w, int relu) {
    using namespace tc;
    static_assert(MODE == 0 || (MODE == 1 && S == 1) || (MODE == 2 && S == 2), "mode / stride");
    extern __shared__ __align__(1024) unsigned char tsm[];
    const int Wp = pitch(S, Wo), Hp = Ho + (S == 1 ? 2 : 1), R = rows(S, Wp);
    const int ABYTES = a_bytes(S, Wp, MODE);           // per stage, one part (hi or lo)
    unsigned char *Ahi = tsm, *Alo = tsm + 2 * ABYTES, *Bs = tsm + 4 * ABYTES;
    uint64_t *mbar = reinterpret_cast<uint64_t *>(Bs + 2 * B_<NT>::BYTES);
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(mbar + 2);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int T = (Hp * Wp + BM - 1) / BM;             // tiles per image
    const int tile = MODE == 2 ? (int)(blockIdx.x >> 2) : (int)blockIdx.x;
    const int cls = MODE == 2 ? (int)(blockIdx.x & 3) : 0, cpy = cls >> 1, cpx = cls & 1;   // MODE 2 parity class
    const int ntaps = MODE == 2 ? (1 + cpy) * (1 + cpx) : 9;
    const int n = tile / T, q0 = (tile % T) * BM;
    const int lo_row = MODE == 2 ? q0 : q0 - (Wp + 1);   // padded-grid row of staged row 0

    if (warp == 0) {   // tensor-memory accumulator: NT columns x 128 lanes of float32
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     :: "r"(smem_u32(tmem_slot)), "r"((uint32_t)NT) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_u32(&mbar[0])) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_u32(&mbar[1])) : "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    constexpr uint32_t IDESC = umma_idesc_bf16(BM, NT);
    const int nchunks = (Cr + CC - 1) / CC;
    const float *srcn = src + (size_t)n * Cr * Hs * Ws;
    bool ok = true;

    for (int c = 0; c < nchunks; ++c) {
        const int sb = c & 1;
        if (c >= 2) {   // chunk c - 2 has left this buffer (the decision is uniform over the CTA)
            const bool done = mbar_wait(&mbar[sb], (uint32_t)(((c >> 1) - 1) & 1));
            if (!__syncthreads_and(done)) {
                ok = false;
                break;
            }
        }
        const int ch0 = c * CC;
        unsigned char *ah = Ahi + sb * ABYTES, *al = Alo + sb * ABYTES;
        // A: per phase, R rows x two 8-channel halves; unit (phase, half, row) at
        // ((phase * 2 + half) * R + row) * 16 bytes.  Consecutive threads take consecutive
        // rows, so every channel plane is read in coalesced runs.
        const int units = phases(S, MODE) * 2 * R;
        for (int L = tid; L < units; L += THREADS) {
            const int row = L % R, ph_half = L / R, half = ph_half & 1, ph = ph_half >> 1;
            const int qg = lo_row + row, qy = qg / Wp, qx = qg - qy * Wp;   // qg may be negative: then outside
            // source pixel of this staged row
            int sy, sx;
            bool in;
            if constexpr (MODE == 2) {   // the dout grid itself, halo after the image
                sy = qy;
                sx = qx;
                in = qy < Hs && qx < Ws;
            } else if constexpr (S == 1) {
                sy = qy - 1;
                sx = qx - 1;
                in = qg >= 0 && qy >= 1 && qy <= Hs && qx >= 1 && qx <= Ws;
            } else {
                sy = 2 * (qy - 1) + (ph >> 1);
                sx = 2 * (qx - 1) + (ph & 1);
                in = qg >= 0 && qy >= 1 && qx >= 1 && sy < Hs && sx < Ws;
            }
            float vals[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const int ch = ch0 + 8 * half + j;
                vals[j] = (in && ch < Cr) ? __ldg(srcn + ((size_t)ch * Hs + sy) * Ws + sx) : 0.f;
            }
            uint4 hi, lo;
            split_row(vals, hi, lo);
            *reinterpret_cast<uint4 *>(ah + L * 16) = hi;
            *reinterpret_cast<uint4 *>(al + L * 16) = lo;
        }
        // B: per tap, NT rows x two 8-channel halves; unit (tap, half, col) at ((tap * 2 + half) * NT + col) * 16
        unsigned char *bsb = Bs + sb * B_<NT>::BYTES;
        for (int L = tid; L < ntaps * 2 * NT; L += THREADS) {
            const int col = L % NT, tap_half = L / NT, half = tap_half & 1, slot = tap_half >> 1;
            // MODE 2: slot -> the class's (ky, kx): ky = 1 for py = 0, 0 / 2 for py = 1
            const int tap = MODE == 2 ? (cpy ? 2 * (slot / (1 + cpx)) : 1) * 3 + (cpx ? 2 * (slot % (1 + cpx)) : 1)
                                      : slot;
            uint32_t wv[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                __nv_bfloat16 e[2];
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int ch = ch0 + 8 * half + 2 * j + h;
                    e[h] = __float2bfloat16_rn(0.f);
                    if (ch < Cr && col < Ncol) {
                        // forward: w[co = col][ci = ch][tap]; data gradient: w[co = ch][ci = col][tap]
                        // (its A operand is shifted by the mirrored tap offset)
                        e[h] = MODE == 0 ? w[((size_t)col * Ci_w + ch) * 9 + tap] : w[((size_t)ch * Ci_w + col) * 9 + tap];
                    }
                }
                wv[j] = pack_bf16(e[0], e[1]);
            }
            *reinterpret_cast<uint4 *>(bsb + L * 16) = make_uint4(wv[0], wv[1], wv[2], wv[3]);
        }
        // generic-proxy writes -> visible to the tensor cores (async proxy)
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
            const uint32_t a_hi = smem_u32(ah), a_lo = smem_u32(al), b0 = smem_u32(bsb);
            const uint32_t lbo_a = (uint32_t)R * 16, lbo_b = (uint32_t)NT * 16;
#pragma unroll 1
            for (int tap = 0; tap < ntaps; ++tap) {
                const int ky = tap / 3, kx = tap % 3;
                int ph = 0, start;
                if constexpr (MODE == 2) {
                    // class slot `tap`: (ky, kx) as staged in B; dout row Y + (ky == 0), column X + (kx == 0)
                    const int kyc = cpy ? 2 * (tap / (1 + cpx)) : 1, kxc = cpx ? 2 * (tap % (1 + cpx)) : 1;
                    start = (kyc == 0 ? Wp : 0) + (kxc == 0 ? 1 : 0);
                } else if constexpr (S == 1) {
                    // output row m reads padded row q0 + m + (ky - 1) Wp + (kx - 1) (mirrored for the data gradient)
                    const int dy = MODE == 0 ? ky - 1 : 1 - ky, dx = MODE == 0 ? kx - 1 : 1 - kx;
                    start = Wp + 1 + dy * Wp + dx;
                } else {
                    // input row 2y + ky - 1: phase (ky + 1) & 1 at phase row y - (ky == 0)
                    const int py = (ky + 1) & 1, px = (kx + 1) & 1, dy = ky == 0 ? -1 : 0, dx = kx == 0 ? -1 : 0;
                    ph = 2 * py + px;
                    start = Wp + 1 + dy * Wp + dx;
                }
                const uint32_t aoff = (uint32_t)((ph * 2 * R + start) * 16);
                const uint64_t db = umma_desc(b0 + (uint32_t)(tap * 2 * NT * 16), lbo_b);
                umma_bf16(tmem, umma_desc(a_hi + aoff, lbo_a), db, IDESC, (c > 0 || tap > 0) ? 1u : 0u);
                umma_bf16(tmem, umma_desc(a_lo + aoff, lbo_a), db, IDESC, 1u);
            }
            umma_commit(&mbar[sb]);
        }
    }
    if (ok) ok = mbar_wait(&mbar[(nchunks - 1) & 1], (uint32_t)(((nchunks - 1) >> 1) & 1));   // all MMAs done
    ok = __syncthreads_and(ok);
    if (!ok) {   // a wait gave up: let the issued MMAs drain (bounded) before the memory is released
        mbar_wait(&mbar[0], 0);
        mbar_wait(&mbar[1], 0);
        __syncthreads();
    }
    tc_fence_after();
    // accumulator -> registers: warp w reads lanes 32 (w % 4) .. +31, columns of half w / 4
    {
        const int qd = warp & 3, halfc = warp >> 2;
        const int m = 32 * qd + lane, qg = q0 + m, qy = qg / Wp, qx = qg - qy * Wp;
        // the padded grid's first row and column are halo (MODE 2: its last ones)
        const int y = MODE == 2 ? qy : qy - 1, x = MODE == 2 ? qx : qx - 1;
        constexpr int COLS = NT / 2;
        uint32_t r[COLS];
#pragma unroll
        for (int c16 = 0; c16 < COLS / 16; ++c16) {
            const uint32_t taddr = tmem + ((uint32_t)(32 * qd) << 16) + (uint32_t)(halfc * COLS + 16 * c16);
            uint32_t *d = r + 16 * c16;
            asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
                         "%12, %13, %14, %15}, [%16];"
                         : "=r"(d[0]), "=r"(d[1]), "=r"(d[2]), "=r"(d[3]), "=r"(d[4]), "=r"(d[5]), "=r"(d[6]),
                           "=r"(d[7]), "=r"(d[8]), "=r"(d[9]), "=r"(d[10]), "=r"(d[11]), "=r"(d[12]), "=r"(d[13]),
                           "=r"(d[14]), "=r"(d[15])
                         : "r"(taddr));
        }
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (y >= 0 && y < Ho && x >= 0 && x < Wo) {   // a real output pixel (not a halo row / column)
#pragma unroll
            for (int j = 0; j < COLS; ++j) {
                const int col = halfc * COLS + j;
                if (col >= Ncol) break;
                float v = ok ? __uint_as_float(r[j]) : __int_as_float(0x7fc00000);
                if constexpr (MODE == 0) {
                    v += bias[col];
                    if (relu) v = fmaxf(v, 0.f);
                }
                if constexpr (MODE == 2)   // din is (2 Ho) x (2 Wo): pixel (2y + py, 2x + px)
                    out[(((size_t)n * Ncol + col) * (2 * Ho) + 2 * y + cpy) * (2 * Wo) + 2 * x + cpx] = v;
                else
                    out[(((size_t)n * Ncol + col) * Ho + y) * Wo + x] = v;
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem), "r"((uint32_t)NT) : "memory");
    }
}

// ------------------------------- weight gradient on the tensor cores (stride 1)
// dw[co][ci][ky][kx] = sum_{n,y,x} dout[n][co][y][x] in[n][ci][y + ky - 1][x + kx - 1]
// as GEMMs that reduce over pixels: for tap t = (ky, kx)
//   D_t[r][co] = sum_k X[k + off_t][r] G[k][co],
// k running over the rows of the padded pixel grid of pitch Wp = W + 2 (halo rows of G are
// zero, so only real output pixels contribute), X the input activations on the same grid
// (zero outside the image), off_t = (ky - 1) Wp + (kx - 1).  Both operands are staged
// MN-major (a 16-byte row holds 8 channels of one pixel; consecutive pixels are
// consecutive rows), so the tap shift is again only the start address of the A
// descriptor: one staged chunk serves all three taps of a kernel row.
//
// Precision: the UMMA M = 128 rows of D are the input channels twice, r = c from the bf16
// hi part of X and r = 64 + c from its lo part (the two halves of the A operand's 16
// channel blocks); G is split the same way and both parts are multiplied (two MMAs per
// tap and K step).  D[c] + D[64 + c] is then (X_hi + X_lo)(G_hi + G_lo), the float32
// product to ~2^-17, accumulated in float32 tensor memory.
//
// A CTA runs the three taps of one kernel row ky = blockIdx.y (3 NT tensor-memory columns,
// NT = 32 or 64 output channels) and stages only the 130 rows they read.  CTAs stride over
// the (image, 128-row tile) chunks, double buffered, and add their D to dw once at the end.
// (Layers with at most 16 output channels stay on the FP32 kernel k_conv_bwd_w: the
// narrowest MMA, N = 16, would carry at most 16 useful columns per tap.)
namespace wg {
constexpr int BM = 128;            // padded-grid rows (the K extent) per chunk
constexpr int THREADS = 256;
constexpr int MB = 16;             // 8-channel blocks of A: 8 hi (channels 0..63), 8 lo
constexpr int ROWS = BM + 2;        // staged rows of X per plane: the 128 + 2 that three kx taps read
constexpr int PLANE = MB * ROWS * 16;
// X planes per stage: stride 1 one; stride 2 the two column parities of the kernel row's input rows
__host__ __device__ constexpr int planes(int S) { return S == 1 ? 1 : 2; }
__host__ __device__ constexpr int a_bytes(int S) { return planes(S) * PLANE; }
__host__ __device__ constexpr int b_bytes(int NT) { return 2 * (NT / 8) * BM * 16; }
__host__ __device__ constexpr int tmem_cols(int c) { return c <= 32 ? 32 : c <= 64 ? 64 : c <= 128 ? 128 : c <= 256 ? 256 : 512; }
__host__ __device__ constexpr int smem_bytes(int NT, int S) { return 2 * a_bytes(S) + 2 * b_bytes(NT) + 64; }
}  // namespace wg

// shared-memory matrix descriptor with both strides given: no swizzle, sm_100 version 1
__device__ __forceinline__ uint64_t umma_desc_mn(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | ((uint64_t)1 << 46);
}
// kind::f16 instruction descriptor with A and B MN-major (transpose bits 15 and 16)
__host__ __device__ constexpr uint32_t umma_idesc_bf16_mn(int M, int N) {
    return umma_idesc_bf16(M, N) | (1u << 15) | (1u << 16);
}

template <int NT, int S>
__global__ void __launch_bounds__(wg::THREADS) k_conv_wgrad_tc(const float *in, const float *dout, float *dw, int Ci,
                                                              int Co, int Hi, int Wi, int Ho, int Wo, int chunks) {
    using namespace wg;
    constexpr int TAPS = 3;
    constexpr int NB = NT / 8;                              // 8-channel blocks of B (per part)
    constexpr uint32_t TCOLS = (uint32_t)tmem_cols(TAPS * NT);
    static_assert(TAPS * NT <= 256, "two CTAs per SM must fit the 512 tensor-memory columns");
    extern __shared__ __align__(1024) unsigned char tsm[];
    // output pixel (y, x) is padded-grid row (y + 1) Wp + (x + 1) (halo first; stride 1 also last)
    const int Wp = S == 1 ? Wo + 2 : Wo + 1, Hp = S == 1 ? Ho + 2 : Ho + 1, R = ROWS;
    const int T = (Hp * Wp + BM - 1) / BM;                  // chunks per image
    constexpr int PL = planes(S), ABYTES = a_bytes(S);
    constexpr int BBYTES = b_bytes(NT);
    unsigned char *As = tsm, *Bs = tsm + 2 * ABYTES;
    uint64_t *mbar = reinterpret_cast<uint64_t *>(Bs + 2 * BBYTES);
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(mbar + 2);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int ky_cta = (int)blockIdx.y;
    // stride 1: input row y + ky - 1 is padded row q + (ky - 1) Wp; stride 2: input row 2y + ky - 1
    // is row y - (ky == 0) of the input's row-parity plane rp = (ky + 1) & 1
    const int rp = (ky_cta + 1) & 1;
    const int row_off = (S == 1 ? ky_cta - 1 : (ky_cta == 0 ? -1 : 0)) * Wp - 1;   // staged row 0, minus q0
    const int cbi = (Ci + 7) / 8, cbo = (Co + 7) / 8;               // live channel blocks of X and G

    // channel blocks beyond Ci / Co stay zero in both stages (never staged)
    for (int L = tid; L < 2 * PL * MB * R; L += THREADS) {
        const int blk = (L % (MB * R)) / R;
        if ((blk & 7) >= cbi) *reinterpret_cast<uint4 *>(As + (size_t)L * 16) = make_uint4(0u, 0u, 0u, 0u);
    }
    for (int L = tid; L < 2 * 2 * NB * BM; L += THREADS) {
        const int blk = (L % (2 * NB * BM)) / BM;
        if ((blk % NB) >= cbo) *reinterpret_cast<uint4 *>(Bs + (size_t)L * 16) = make_uint4(0u, 0u, 0u, 0u);
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     :: "r"(smem_u32(tmem_slot)), "r"(TCOLS) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_u32(&mbar[0])) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_u32(&mbar[1])) : "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    constexpr uint32_t IDESC = umma_idesc_bf16_mn(BM, NT);
    bool ok = true;
    int it = 0;

    // Warp 0 issues the MMAs of chunk `it` while warps 1..7 stage chunk it + 1 into the
    // other buffer: the staging warps wait (bounded) on that buffer's mbarrier, agree on
    // the outcome at a named barrier, and meet warp 0 at the block barrier after staging.
    constexpr int PRODUCERS = THREADS - 32;
    for (int c = blockIdx.x; c < chunks; c += gridDim.x, ++it) {
        const int sb = it & 1;
        const int n = c / T, q0 = (c % T) * BM;
        unsigned char *a = As + sb * ABYTES, *bsb = Bs + sb * BBYTES;
        bool good = true;
        if (warp != 0) {
            if (it >= 2) good = mbar_wait(&mbar[sb], (uint32_t)(((it >> 1) - 1) & 1));   // chunk it - 2 left it
            good = bar_and(1, PRODUCERS, good);
        }
        if (warp != 0 && good) {
            const int p = tid - 32;
            const float *inn = in + (size_t)n * Ci * Hi * Wi;
            const float *gn = dout + (size_t)n * Co * Ho * Wo;
            // A: unit (plane, block, row) at plane * PLANE + (block * R + row) * 16 (hi) and
            // plane * PLANE + ((block + 8) * R + row) * 16 (lo)
            for (int L = p; L < PL * cbi * R; L += PRODUCERS) {
                const int pl = L / (cbi * R), rem = L - pl * (cbi * R), row = rem % R, blk = rem / R;
                const int qg = q0 + row_off + row;
                const int qy = qg >= 0 ? qg / Wp : -1, qx = qg - qy * Wp;
                const int sy = S == 1 ? qy - 1 : 2 * (qy - 1) + rp, sx = S == 1 ? qx - 1 : 2 * (qx - 1) + pl;
                const bool inb = qg >= 0 && qy >= 1 && qx >= 1 && sy < Hi && sx < Wi;
                float vals[8];
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    const int ch = 8 * blk + j;
                    vals[j] = (inb && ch < Ci) ? __ldg(inn + ((size_t)ch * Hi + sy) * Wi + sx) : 0.f;
                }
                uint4 hi, lo;
                split_row(vals, hi, lo);
                *reinterpret_cast<uint4 *>(a + (size_t)pl * PLANE + (size_t)(blk * R + row) * 16) = hi;
                *reinterpret_cast<uint4 *>(a + (size_t)pl * PLANE + (size_t)((blk + 8) * R + row) * 16) = lo;
            }
            // B: unit (block, row) at (block * BM + row) * 16 (hi) and ((block + NB) * BM + row) * 16 (lo)
            for (int L = p; L < cbo * BM; L += PRODUCERS) {
                const int row = L % BM, blk = L / BM;
                const int qg = q0 + row, qy = qg / Wp, qx = qg - qy * Wp;
                const bool inb = qy >= 1 && qy <= Ho && qx >= 1 && qx <= Wo;
                float vals[8];
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    const int ch = 8 * blk + j;
                    vals[j] = (inb && ch < Co) ? __ldg(gn + ((size_t)ch * Ho + (qy - 1)) * Wo + (qx - 1)) : 0.f;
                }
                uint4 hi, lo;
                split_row(vals, hi, lo);
                *reinterpret_cast<uint4 *>(bsb + (size_t)(blk * BM + row) * 16) = hi;
                *reinterpret_cast<uint4 *>(bsb + (size_t)((blk + NB) * BM + row) * 16) = lo;
            }
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        }
        if (!__syncthreads_and(good)) {
            ok = false;
            break;
        }
        if (tid == 0) {
            tc_fence_after();
            // descriptors advance by 16 staged rows (256 bytes, 16 in the address field) per K step
            const uint32_t sbo_a = (uint32_t)R * 16, sbo_b = (uint32_t)BM * 16;
            const uint64_t dbh = umma_desc_mn(smem_u32(bsb), 128u, sbo_b);
            const uint64_t dbl = umma_desc_mn(smem_u32(bsb) + (uint32_t)(NB * BM * 16), 128u, sbo_b);
#pragma unroll 1
            for (int tap = 0; tap < TAPS; ++tap) {
                // staged row of k = 0 for tap kx: stride 1 row kx; stride 2 column x - (kx == 0) of the
                // column-parity plane (kx + 1) & 1
                const int pl = S == 1 ? 0 : (tap + 1) & 1, start = S == 1 ? tap : (tap == 0 ? 0 : 1);
                const uint64_t da = umma_desc_mn(smem_u32(a) + (uint32_t)(pl * PLANE + start * 16), 128u, sbo_a);
                const uint32_t d = tmem + (uint32_t)(tap * NT);
#pragma unroll
                for (int ks = 0; ks < BM / 16; ++ks) {
                    umma_bf16(d, da + (uint64_t)(16 * ks), dbh + (uint64_t)(16 * ks), IDESC, (it > 0 || ks > 0) ? 1u : 0u);
                    umma_bf16(d, da + (uint64_t)(16 * ks), dbl + (uint64_t)(16 * ks), IDESC, 1u);
                }
            }
            umma_commit(&mbar[sb]);
        }
    }
    if (ok && it > 0) ok = mbar_wait(&mbar[(it - 1) & 1], (uint32_t)(((it - 1) >> 1) & 1));   // all MMAs done
    ok = __syncthreads_and(ok);
    if (!ok) {   // a wait gave up: let issued MMAs drain (bounded) before the memory is reused
        mbar_wait(&mbar[0], 0);
        mbar_wait(&mbar[1], 0);
        __syncthreads();
    }
    tc_fence_after();
    // D -> shared scratch [128 rows][TAPS][NT] (the operand buffers are free now): warp w reads
    // lanes 32 (w % 4) .. +31, column half w / 4 of every tap
    float *scr = reinterpret_cast<float *>(tsm);
    if (it > 0) {
        const int qd = warp & 3, halfc = warp >> 2;
        const int r = 32 * qd + lane;
        constexpr int HC = NT / 2;
#pragma unroll 1
        for (int tap = 0; tap < TAPS; ++tap) {
#pragma unroll
            for (int c8 = 0; c8 < HC / 8; ++c8) {
                const uint32_t taddr = tmem + ((uint32_t)(32 * qd) << 16) + (uint32_t)(tap * NT + halfc * HC + 8 * c8);
                uint32_t d[8];
                asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                             : "=r"(d[0]), "=r"(d[1]), "=r"(d[2]), "=r"(d[3]), "=r"(d[4]), "=r"(d[5]), "=r"(d[6]),
                               "=r"(d[7])
                             : "r"(taddr));
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
                for (int j = 0; j < 8; ++j)
                    scr[((size_t)r * TAPS + tap) * NT + halfc * HC + 8 * c8 + j] = __uint_as_float(d[j]);
            }
        }
    }
    __syncthreads();
    if (it > 0) {
        // dw[co][ci][ky][kx] += D[ci] + D[64 + ci]; consecutive threads take consecutive taps
        const int tap0 = 3 * ky_cta;
        for (int L = tid; L < Co * Ci * TAPS; L += THREADS) {
            const int tap = L % TAPS, ci = (L / TAPS) % Ci, co = L / (TAPS * Ci);
            const float v = ok ? scr[((size_t)ci * TAPS + tap) * NT + co] + scr[((size_t)(64 + ci) * TAPS + tap) * NT + co]
                               : __int_as_float(0x7fc00000);
            atomicAdd(dw + ((size_t)co * Ci + ci) * 9 + tap0 + tap, v);
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem), "r"(TCOLS) : "memory");
    }
}

// db[co] += sum_{n, pixel} dout[n][co][pixel]: one CTA per (channel, batch slice)
__global__ void __launch_bounds__(256) k_bias_grad(const float *dout, float *db, int Nb, int Co, int P, int n_per) {
    __shared__ float red[8];
    const int co = blockIdx.x, n0 = blockIdx.y * n_per, n1 = min(Nb, n0 + n_per);
    float s = 0.f;
    for (int n = n0; n < n1; ++n) {
        const float *g = dout + ((size_t)n * Co + co) * P;
        for (int p = threadIdx.x; p < P; p += blockDim.x) s += g[p];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        float t = 0.f;
        for (int k = 0; k < 8; ++k) t += red[k];
        atomicAdd(db + co, t);
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

// the tensor-core form serves GEMM widths (output channels) of 32 and 64
template <int NT, int S, int MODE>
static int launch_conv_tc_n(const float *src, const __nv_bfloat16 *w, const float *bias, float *out, int Nb, int Cr,
                            int Ncol, int Hs, int Ws, int Ho, int Wo, int Ci_w, int relu, cudaStream_t st) {
    const int Wp = tc::pitch(S, Wo), Hp = Ho + (S == 1 ? 2 : 1);
    const int smem = 4 * tc::a_bytes(S, Wp, MODE) + 2 * tc::B_<NT>::BYTES + 64;
    if (smem > 200 * 1024) return PHB_ERR_UNSUPPORTED;   // wider images than this network uses
    const long long tiles = (long long)Nb * ((Hp * Wp + tc::BM - 1) / tc::BM) * (MODE == 2 ? 4 : 1);
    if (tiles > 0x7fffffffll) return PHB_ERR_UNSUPPORTED;
    auto k = k_conv_tc<NT, S, MODE>;
    if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess)
        return record_cuda(cudaGetLastError());
    k<<<(unsigned)tiles, tc::THREADS, smem, st>>>(src, w, bias, out, Cr, Ncol, Hs, Ws, Ho, Wo, Ci_w, relu);
    return check_launch();
}

template <int S, int MODE>
static int launch_conv_tc(const float *src, const __nv_bfloat16 *w, const float *bias, float *out, int Nb, int Cr,
                          int Ncol, int Hs, int Ws, int Ho, int Wo, int Ci_w, int relu, cudaStream_t st) {
    return Ncol <= 32 ? launch_conv_tc_n<32, S, MODE>(src, w, bias, out, Nb, Cr, Ncol, Hs, Ws, Ho, Wo, Ci_w, relu, st)
                      : launch_conv_tc_n<64, S, MODE>(src, w, bias, out, Nb, Cr, Ncol, Hs, Ws, Ho, Wo, Ci_w, relu, st);
}

static bool tc_width(int n) { return n == 32 || n == 64; }

// tensor-core weight gradient (stride 1 or 2, Ci <= 64, 17 <= Co <= 64): 3 CTAs (kernel rows)
// per group of chunks, one wave of resident CTAs striding over the (image, 128-row tile) chunks
template <int NT, int S>
static int launch_wgrad_tc(const float *in, const float *dout, float *dw, int Nb, int Ci, int Co, int Hi, int Wi,
                           cudaStream_t st) {
    const int Ho = Hi / S, Wo = Wi / S;
    const int Wp = S == 1 ? Wo + 2 : Wo + 1, Hp = S == 1 ? Ho + 2 : Ho + 1;
    constexpr int smem = wg::smem_bytes(NT, S);
    constexpr int scratch = wg::BM * 3 * NT * (int)sizeof(float);   // epilogue, over the operand buffers
    static_assert(scratch <= smem - 64, "epilogue scratch must fit the operand buffers");
    static_assert(smem <= 227 * 1024, "shared memory per CTA");
    const long long chunks = (long long)Nb * ((Hp * Wp + wg::BM - 1) / wg::BM);
    if (chunks > 0x7fffffffll) return PHB_ERR_UNSUPPORTED;
    int dev = 0, sms = 0;
    int rc = record_cuda(cudaGetDevice(&dev));
    if (!rc) rc = record_cuda(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    if (rc) return rc;
    const int per_sm = 2 * (smem + 1024) <= 227 * 1024 ? 2 : 1;
    const int groups = 3;
    long long gk = (long long)sms * per_sm / groups;   // one wave: every CTA resident at once
    if (gk > chunks) gk = chunks;
    if (gk < 1) gk = 1;
    auto k = k_conv_wgrad_tc<NT, S>;
    if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess)
        return record_cuda(cudaGetLastError());
    k<<<dim3((unsigned)gk, (unsigned)groups), wg::THREADS, smem, st>>>(in, dout, dw, Ci, Co, Hi, Wi, Ho, Wo,
                                                                         (int)chunks);
    return check_launch();
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
    if (tc_width(Co) && Wo <= 64) {   // tensor cores (tcgen05): 32 or 64 output channels
        return stride == 1 ? launch_conv_tc<1, 0>(in, w, bias, out, Nb, Ci, Co, Hi, Wi, Ho, Wo, Ci, relu, st)
                           : launch_conv_tc<2, 0>(in, w, bias, out, Nb, Ci, Co, Hi, Wi, Ho, Wo, Ci, relu, st);
    }
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
    if (tc_width(Ci) && Wi <= 64) {   // tensor cores: the GEMM width is the input-channel count
        if (stride == 1) return launch_conv_tc<1, 1>(dout, w, nullptr, din, Nb, Co, Ci, Ho, Wo, Hi, Wi, Ci, 0, st);
        // stride 2: four parity classes on the dout grid (Ho x Wo)
        return launch_conv_tc<2, 2>(dout, w, nullptr, din, Nb, Co, Ci, Ho, Wo, Ho, Wo, Ci, 0, st);
    }
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
    cudaStream_t st = (cudaStream_t)stream;
    if (Ci <= 64 && Co > 16 && Co <= 64) {   // tensor cores (tcgen05), bias gradient beside
        k_bias_grad<<<dim3((unsigned)Co, (unsigned)((Nb + 15) / 16)), 256, 0, st>>>(dout, db, Nb, Co, Ho * Wo, 16);
        int rc = check_launch();
        if (rc) return rc;
        if (stride == 1)
            return Co <= 32 ? launch_wgrad_tc<32, 1>(in, dout, dw, Nb, Ci, Co, Hi, Wi, st)
                            : launch_wgrad_tc<64, 1>(in, dout, dw, Nb, Ci, Co, Hi, Wi, st);
        return Co <= 32 ? launch_wgrad_tc<32, 2>(in, dout, dw, Nb, Ci, Co, Hi, Wi, st)
                        : launch_wgrad_tc<64, 2>(in, dout, dw, Nb, Ci, Co, Hi, Wi, st);
    }
    dim3 grid((unsigned)((Co + 7) / 8), (unsigned)Ci, (unsigned)((Nb + per - 1) / per));
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

int phb_wait_probe(int32_t arrive, int64_t limit, int32_t *out, void *stream) {
    if (!out || (arrive != 0 && arrive != 1) || limit < 1 || limit > tc::WAIT_LIMIT) return PHB_ERR_INVALID_ARG;
    k_wait_probe<<<1, 32, 0, (cudaStream_t)stream>>>(arrive, (long long)limit, out);
    return check_launch();
}

}  // extern "C"
