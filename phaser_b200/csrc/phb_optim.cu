// Gradient-engine updates with optax semantics, applied on the device.
//
// The reference's gradient engine (phaser/engines/gradient/run.py:156-349,
// phaser/engines/gradient/solvers.py:48-138) turns jax's gradient into the
// descent direction d = -conj(grad) / scale and feeds it to optax chains:
//   sgd     trace(momentum, nesterov) -> scale_by_learning_rate(lr, flip_sign=False)
//   adam    scale_by_adam(b1, b2, eps, eps_root, nesterov) -> scale_by_learning_rate(lr)
//   polyak  scale_by_learning_rate(scaling) -> scale_by_polyak(max_lr, f_min, eps)
// and adds the result to the parameter (run.py:107-124).  Here g is the
// gradient dL/dRe + i dL/dIm produced by the adjoint kernel, so d = grad_scale * g
// with grad_scale = -1/B (probe) or -1/(B * sum|probe|^2) (object, positions).
#include "phb_common.cuh"
#include "phb_runtime.h"

namespace phb {

__global__ void k_sq_norm(const float *x, int64_t n, float scale, double *out) {
    double acc = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float v = x[i] * scale;
        acc += (double)v * (double)v;
    }
    warp_atomic_sum(out, acc);
}

// one element = 1 float (real parameters) or 2 floats (complex parameters)
template <bool CPLX>
__global__ void k_optim(const phb_optim o) {
    const double bc1 = 1.0 - pow((double)o.b1, (double)o.count);
    const double bc2 = 1.0 - pow((double)o.b2, (double)o.count);
    const double bc1n = 1.0 - pow((double)o.b1, (double)(o.count + 1));
    float polyak_step = 0.f;
    if (o.kind == PHB_OPTIM_POLYAK) {
        // stochastic Polyak step size (Loizou et al., AISTATS 2021), capped at max_lr
        const double q = *o.polyak_sq_norm + (double)o.polyak_eps;
        polyak_step = q <= 0x1p-52 ? 0.f
                                   : (float)fmin((*o.polyak_loss - (double)o.polyak_f_min) / q, (double)o.polyak_max_lr);
    }
    bool bad = false;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < o.n; i += (int64_t)gridDim.x * blockDim.x) {
        float2 d = CPLX ? reinterpret_cast<const float2 *>(o.grad)[i] : make_float2(o.grad[i], 0.f);
        d = cscale(d, o.grad_scale);
        float2 out;
        if (o.kind == PHB_OPTIM_SGD) {
            if (o.momentum != 0.f) {   // optax.trace
                float2 t = CPLX ? reinterpret_cast<float2 *>(o.state1)[i] : make_float2(o.state1[i], 0.f);
                t = cadd(d, cscale(t, o.momentum));
                if (CPLX) reinterpret_cast<float2 *>(o.state1)[i] = t;
                else o.state1[i] = t.x;
                out = o.nesterov ? cadd(d, cscale(t, o.momentum)) : t;
            } else {
                out = d;
            }
            out = cscale(out, o.lr);
        } else if (o.kind == PHB_OPTIM_ADAM) {   // optax.scale_by_adam (|d|^2 for complex d)
            float2 mu = CPLX ? reinterpret_cast<float2 *>(o.state1)[i] : make_float2(o.state1[i], 0.f);
            float nu = o.state2[i];
            mu = cadd(cscale(mu, o.b1), cscale(d, 1.f - o.b1));
            nu = o.b2 * nu + (1.f - o.b2) * cabs2(d);
            if (CPLX) reinterpret_cast<float2 *>(o.state1)[i] = mu;
            else o.state1[i] = mu.x;
            o.state2[i] = nu;
            float2 mh;
            if (o.nesterov)
                mh = cadd(cscale(mu, (float)(o.b1 / bc1n)), cscale(d, (float)((1.0 - o.b1) / bc1)));
            else
                mh = cscale(mu, (float)(1.0 / bc1));
            const float nh = (float)(nu / bc2);
            out = cscale(mh, o.lr / (sqrtf(nh + o.eps_root) + o.eps));
        } else {   // polyak: step * (scaling * d)
            out = cscale(d, o.polyak_scaling * polyak_step);
        }
        if (o.update_out) {
            if (CPLX) reinterpret_cast<float2 *>(o.update_out)[i] = out;
            else o.update_out[i] = out.x;
        } else if (CPLX) {
            float2 *p = reinterpret_cast<float2 *>(o.param) + i;
            const float2 v = cadd(*p, out);
            *p = v;
            bad |= !finite2(v);
        } else {
            const float v = o.param[i] + out.x;
            o.param[i] = v;
            bad |= !isfinite(v);
        }
    }
    if (bad && o.status) atomicCAS(o.status, -1, o.status_code);
}

// param (n, 2) += upd - mean(upd) (run.py:115-118: position updates keep the scan centred)
__global__ void __launch_bounds__(1024) k_add_centred(float *param, const float *upd, int64_t n) {
    __shared__ double red[2][32];
    double sy = 0.0, sx = 0.0;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
        sy += upd[2 * i];
        sx += upd[2 * i + 1];
    }
    for (int o = 16; o > 0; o >>= 1) {
        sy += __shfl_xor_sync(0xffffffffu, sy, o);
        sx += __shfl_xor_sync(0xffffffffu, sx, o);
    }
    if ((threadIdx.x & 31) == 0) {
        red[0][threadIdx.x >> 5] = sy;
        red[1][threadIdx.x >> 5] = sx;
    }
    __syncthreads();
    if (threadIdx.x < 32) {
        double a = threadIdx.x < (blockDim.x >> 5) ? red[0][threadIdx.x] : 0.0;
        double c = threadIdx.x < (blockDim.x >> 5) ? red[1][threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) {
            a += __shfl_xor_sync(0xffffffffu, a, o);
            c += __shfl_xor_sync(0xffffffffu, c, o);
        }
        if (threadIdx.x == 0) {
            red[0][0] = a;
            red[1][0] = c;
        }
    }
    __syncthreads();
    const float my = (float)(red[0][0] / (double)n), mx = (float)(red[1][0] / (double)n);
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
        param[2 * i] += upd[2 * i] - my;
        param[2 * i + 1] += upd[2 * i + 1] - mx;
    }
}

}  // namespace phb

using namespace phb;

static inline unsigned optim_grid(int64_t n) {
    int64_t g = (n + 255) / 256;
    if (g > 148 * 8) g = 148 * 8;
    return (unsigned)(g < 1 ? 1 : g);
}

extern "C" {

int phb_sq_norm_f32(const float *x, int64_t n, float scale, double *out, void *stream) {
    if (!x || !out || n < 0) return PHB_ERR_INVALID_ARG;
    if (n == 0) return PHB_OK;
    k_sq_norm<<<optim_grid(n), 256, 0, (cudaStream_t)stream>>>(x, n, scale, out);
    return check_launch();
}

int phb_optimizer_update(const phb_optim *o, void *stream) {
    if (!o || !o->grad || o->n < 0 || (!o->param && !o->update_out)) return PHB_ERR_INVALID_ARG;
    if (o->kind < PHB_OPTIM_SGD || o->kind > PHB_OPTIM_POLYAK) return PHB_ERR_INVALID_ARG;
    if (o->kind == PHB_OPTIM_SGD && o->momentum != 0.f && !o->state1) return PHB_ERR_INVALID_ARG;
    if (o->kind == PHB_OPTIM_ADAM && (!o->state1 || !o->state2 || o->count < 1)) return PHB_ERR_INVALID_ARG;
    if (o->kind == PHB_OPTIM_POLYAK && (!o->polyak_sq_norm || !o->polyak_loss)) return PHB_ERR_INVALID_ARG;
    if (o->n == 0) return PHB_OK;
    if (o->complex_elems) k_optim<true><<<optim_grid(o->n), 256, 0, (cudaStream_t)stream>>>(*o);
    else k_optim<false><<<optim_grid(o->n), 256, 0, (cudaStream_t)stream>>>(*o);
    return check_launch();
}

int phb_add_centred(float *param, const float *update, int64_t n, void *stream) {
    if (!param || !update || n < 1) return PHB_ERR_INVALID_ARG;
    k_add_centred<<<1, 1024, 0, (cudaStream_t)stream>>>(param, update, n);
    return check_launch();
}

}  // extern "C"
