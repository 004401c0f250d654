/*
 * phaser_b200 -- C ABI of the B200 (sm_100a) multislice ptychography backend.
 *
 * Conventions for every entry point:
 *   - all array arguments are DEVICE pointers owned by the caller; nothing
 *     here allocates device memory (scratch comes in through `workspace`);
 *   - complex arrays are interleaved float pairs (C99 `float _Complex`,
 *     numpy complex64), row-major, C-contiguous;
 *   - work is enqueued on `stream` (a cudaStream_t, passed as void*) and the
 *     call returns without synchronising;
 *   - the return value is a status code (PHB_OK == 0); no exception or abort
 *     crosses this boundary.  `phb_status_string` names a code.
 *
 * The reference citations are paths inside the phaser source tree.
 */
#ifndef PHASER_B200_H
#define PHASER_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ status */
#define PHB_OK                 0
#define PHB_ERR_INVALID_ARG    1   /* null pointer, bad size, misaligned workspace */
#define PHB_ERR_UNSUPPORTED    2   /* shape the kernels do not implement (e.g. N not 64/128/256) */
#define PHB_ERR_CUDA           3   /* a CUDA launch or runtime call failed */
#define PHB_ERR_NONFINITE      4   /* NaN/inf found in the object or probe */
#define PHB_ERR_OUTSIDE        5   /* probe positions completely outside the object */
#define PHB_ERR_SCRATCH_LIMIT  6   /* problem too large for phb_solver_group_static's fixed scratch */

const char *phb_status_string(int status);
int phb_version(void);
/* Last CUDA error text seen by this library on the calling thread ("" if none). */
const char *phb_last_cuda_error(void);

/* ------------------------------------------------------------- cutouts (a1-a4)
 * Integer cutout starts and sub-pixel shifts for scan positions.
 * Replaces ObjectSampling._pos_to_object_idx + numpy.round
 * (phaser/utils/object.py:291-301, 493-495) and get_subpx_shifts (324-331).
 * idx = (pos - corner)/sampling - (n - 1)/2 in float64, rounded half-to-even,
 * bit-exact with the reference.  `group` (B) selects rows of `scan` (n_pos x 2,
 * float32, (y, x)); pass NULL to take rows 0..B-1.  `subpx` may be NULL. */
int phb_cutout_starts(const float *scan, const int64_t *group, int64_t B,
                      double corner_y, double corner_x, double samp_y, double samp_x,
                      int64_t cut_y, int64_t cut_x,
                      int64_t *starts /* B x 2 */, float *subpx /* B x 2 or NULL */,
                      void *stream);

/* Gather cutouts of every slice: out[b, s, i, j] = obj[s, i + y0_b, j + x0_b],
 * out-of-bounds pixels read `fill`.  Replaces ObjectCutout.get
 * (phaser/utils/object.py:501-519; GPU form phaser/utils/_cuda_kernels.py:51-75). */
int phb_cutout_get_c64(const void *obj, int64_t S, int64_t H, int64_t W,
                       const int64_t *starts, int64_t B, int64_t cut_y, int64_t cut_x,
                       float fill_re, float fill_im, void *out, void *stream);
int phb_cutout_get_f32(const float *obj, int64_t S, int64_t H, int64_t W,
                       const int64_t *starts, int64_t B, int64_t cut_y, int64_t cut_x,
                       float fill, float *out, void *stream);

/* Scatter-add views (B, S, cut_y, cut_x) into obj (S, H, W); out-of-bounds
 * pixels are dropped.  fp32 atomics, so the summation order is not fixed.
 * Replaces ObjectCutout.add (phaser/utils/object.py:540-557;
 * phaser/utils/_cuda_kernels.py:78-107). */
int phb_cutout_add_c64(void *obj, int64_t S, int64_t H, int64_t W,
                       const int64_t *starts, int64_t B, int64_t cut_y, int64_t cut_x,
                       const void *views, void *stream);
int phb_cutout_add_f32(float *obj, int64_t S, int64_t H, int64_t W,
                       const int64_t *starts, int64_t B, int64_t cut_y, int64_t cut_x,
                       const float *views, void *stream);

/* Overwrite cutouts (last writer wins where views overlap, as in the reference).
 * Replaces ObjectCutout.set (phaser/utils/object.py:521-538). */
int phb_cutout_set_c64(void *obj, int64_t S, int64_t H, int64_t W,
                       const int64_t *starts, int64_t B, int64_t cut_y, int64_t cut_x,
                       const void *views, void *stream);

/* --------------------------------------------------------------------- FFT (a5)
 * Batched 2D FFT with phaser's convention: centred real space, orthonormal.
 * inverse == 0: out = fft2(in)  = fft2(ifftshift(in)) / N   (phaser/utils/num.py:460-468)
 * inverse == 1: out = ifft2(in) = fftshift(ifft2(in)) / N   (phaser/utils/num.py:434-442)
 * N in {64, 128, 256}; `in` and `out` may alias. */
int phb_fft2_c64(const void *in, void *out, int64_t batch, int64_t N, int inverse, void *stream);

/* ------------------------------------------------------------- constraints (a17)
 * In-place amplitude clamp: a *= min(|a|, amplitude) / |a|.
 * Replaces clamp_amplitude (phaser/engines/common/regularizers.py:36-42). */
int phb_clamp_amplitude_c64(void *arr, int64_t n, float amplitude, void *stream);

/* In-place Fourier filter of `batch` N x N tiles: a = ifft2(fft2(a) * mask), mask
 * (N, N) float32 with the zero frequency in the corner.  Replaces
 * LimitProbeSupport.apply_iter (phaser/engines/common/regularizers.py:45-64). */
int phb_fourier_mask_c64(void *arr, int64_t batch, int64_t N, const float *mask, void *stream);

/* ------------------------------------------------------ the multislice engine
 * The LSQ-ML / ePIE / gradient mini-batch step
 * (phaser/engines/conventional/solvers.py:132-504,
 *  phaser/engines/gradient/run.py:357-438).
 *
 * One `phb_engine` describes a reconstruction resident on the device; the
 * caller fills it once (see phb_engine_workspace_bytes for the scratch) and
 * passes it to the per-group / per-iteration calls. */

#define PHB_SOLVER_LSQML 0
#define PHB_SOLVER_EPIE  1
#define PHB_SOLVER_GRAD  2      /* gradient-engine loss + adjoint */

#define PHB_NOISE_AMPLITUDE 0   /* also 'anscombe' (offset 0.375) */
#define PHB_NOISE_POISSON   1   /* loss/gradient only (no wave update, as in the reference) */

#define PHB_FLAG_UPDATE_OBJECT   1
#define PHB_FLAG_UPDATE_PROBE    2
#define PHB_FLAG_UPDATE_POSITION 4
#define PHB_FLAG_UPDATE_TILT   32   /* gradient solver: per-position tilt gradient (needs phb_engine.tilt) */
#define PHB_FLAG_CALC_ERROR      8

#define PHB_STATUS_INTERNAL (1 << 30)   /* flag bit in phb_step.status: kernel aborted its program */
/* flag bit in phb_step.status, set only by the bounds-checking build of the library
 * (compiled with -DPHB_BOUNDS_CHECK=1: libphaser_b200_bounds.so): a group index outside
 * [0, n_pos); the position is skipped instead of read or written out of bounds */
#define PHB_STATUS_BOUNDS (1 << 29)

typedef struct phb_engine {
    /* sizes */
    int32_t N;            /* probe / detector side: 64, 128 or 256 (256: no ePIE) */
    int32_t M;            /* incoherent probe modes, 1..8 */
    int32_t S;            /* object slices */
    int32_t B_max;        /* largest group the workspace was sized for */
    int64_t H, W;         /* object slice shape */
    int64_t n_pos;        /* scan positions */
    /* geometry (float64, as the reference computes cutout indices) */
    double corner_y, corner_x, samp_y, samp_x;
    /* state, updated in place */
    void  *object;        /* (S, H, W) complex64 */
    void  *probe;         /* (M, N, N) complex64, real space, centred */
    float *scan;          /* (n_pos, 2) float32 (y, x) */
    const float *tilt;    /* (n_pos, 2) float32 mrad, or NULL */
    /* data */
    const void  *patterns;    /* (n_pos, N, N) float32, or uint16 counts when pattern_u16 != 0;
                                 zero frequency in the corner */
    const float *pattern_mask;/* (N, N) float32 */
    const void  *propagators; /* (S-1, N, N) complex64 (band-limited, untilted) or NULL when S == 1 */
    const float *thicknesses; /* (S) slice thicknesses, used for tilt ramps; NULL if no tilt */
    const float *ky, *kx;     /* (N) fftfreq of the probe sampling, float32 */
    /* noise model */
    int32_t noise;        /* PHB_NOISE_* */
    float noise_eps, noise_offset, noise_var;
    /* workspace: phb_engine_workspace_bytes() bytes, 256-byte aligned */
    void *workspace;
    size_t workspace_bytes;
    /* solver bookkeeping outputs (accumulated over the iteration) */
    float *new_obj_mag;   /* (N, N) float32 or NULL */
    float *new_probe_mag; /* (S, H, W) float32 or NULL */
    /* resident pattern format: 0 = float32, 1 = uint16 detector counts (half the HBM
       footprint and read traffic; the kernels convert each count to float32 exactly,
       as the reference's cast to float32 does, phaser/execute.py:176-177) */
    int32_t pattern_u16;
} phb_engine;

typedef struct phb_step {
    int32_t solver;       /* PHB_SOLVER_* */
    int32_t flags;        /* PHB_FLAG_* */
    float beta_object, beta_probe;
    float illum_reg_object, illum_reg_probe, gamma;
    float *pos_update;    /* (n_pos, 2) float32: this group's rows are written; may be NULL */
    float *errors;        /* (n_pos) float32: per-position error of this group; may be NULL */
    float *loss;          /* (n_pos) float32: gradient-engine per-position loss; may be NULL */
    void  *grad_object;   /* gradient solver: (S, H, W) complex64 accumulator, NULL otherwise */
    void  *grad_probe;    /* gradient solver: (M, N, N) complex64 accumulator */
    float *grad_pos;      /* gradient solver: (n_pos, 2) float32 dL/d(y, x) */
    int32_t *status;      /* device int, sticky, -1 = fine: the first group index that produced NaN/inf,
                             or PHB_STATUS_INTERNAL | group index if a kernel aborted (internal error),
                             or PHB_STATUS_BOUNDS | group index (bounds-checking build only) */
    int32_t group_index;  /* index of this group within the iteration (for `status`) */
    const float *group_patterns; /* optional (B, N, N): this group's patterns in group order, read
                                    instead of patterns[group[b]] (host-streamed data) */
    void *event_begin;    /* optional cudaEvent_t recorded just before / after the fused kernel */
    void *event_end;
    float grad_pos_scale; /* gradient solver: grad_pos = grad_pos_scale * dL/d(y, x) (0 means 1) */
    double *group_loss;   /* gradient solver: optional device double, += the group's summed loss */
    int32_t b_begin, b_end; /* with PHB_FLAG_PARTIAL: the rows [b_begin, b_end) of the group this call runs */
    float *grad_tilt;     /* gradient solver with PHB_FLAG_UPDATE_TILT: (n_pos, 2) dL/d(tilt y, tilt x) [1/mrad] */
    float grad_tilt_scale;/* grad_tilt = grad_tilt_scale * dL/dtilt (0 means 1) */
} phb_step;

/* Bytes of workspace the engine needs for groups of up to B_max positions. */
size_t phb_engine_workspace_bytes(int32_t N, int32_t M, int32_t S, int32_t B_max,
                                  int64_t H, int64_t W);

/* Validate the descriptor and prepare derived tables in the workspace
 * (K-ordered propagators, mask, twiddles, probe spectrum). */
int phb_engine_init(const phb_engine *e, void *stream);

/* Refresh the cached probe spectrum after the caller changed `probe`
 * (e.g. by a constraint or by rescaling). */
int phb_engine_probe_changed(const phb_engine *e, void *stream);

/* Presolve pass of LSQ-ML / ePIE (solvers.py:132-167, 387-412) or the gradient
 * engine (gradient/run.py:413-438) over one group: accumulates per-position
 * measured/model intensity into rescale_num/rescale_den (B, float64, must be
 * zeroed by the caller).  LSQ-ML also adds the group illumination into
 * new_probe_mag and |prod O|^2 into new_obj_mag.  `gradient_form` != 0 selects
 * the gradient engine's variant (last slice transmitted, unmasked patterns). */
int phb_presolve_group(const phb_engine *e, const int64_t *group, int32_t B, int32_t solver,
                       int32_t gradient_form, double *rescale_num, double *rescale_den,
                       void *stream);

/* Forward model of one group (the gradient engine's form, gradient/run.py:357-400:
 * subpixel-shifted probe, multislice propagation, last slice transmitted, far field):
 * writes sum over modes of |fft2(exit wave)|^2 into intensity (B, N, N) float32, zero
 * frequency in the corner -- the layout of measured patterns. */
int phb_simulate_group(const phb_engine *e, const int64_t *group, int32_t B, float *intensity, void *stream);

/* One mini-batch of the chosen solver: LSQ-ML (solvers.py:171-290), ePIE
 * (solvers.py:415-504) or the gradient engine's loss and adjoint
 * (gradient/run.py:357-405 under jax.value_and_grad).  Updates object/probe in
 * place (LSQ-ML, ePIE) or accumulates gradients (GRAD). */
/* Data-parallel split of a mini-batch over ranks (one process per GPU): with
 * PHB_FLAG_PARTIAL in st->flags, phb_solver_group runs only rows [b_begin, b_end)
 * of the group and leaves its share in the workspace accumulators.  The caller then
 * sums, over all ranks, the float32 byte range [out4[0], out4[0] + out4[1]) and the
 * float64 byte range [out4[2], out4[2] + out4[3]) of the workspace
 * (phb_engine_reduce_layout) -- one all-reduce each -- and calls
 * phb_solver_group_finish with the same step, which applies the updates (identical
 * on every rank).  No counterpart in the reference (single process). */
#define PHB_FLAG_PARTIAL 16
int phb_engine_reduce_layout(int32_t N, int32_t M, int32_t S, int32_t B_max, int64_t H, int64_t W, int64_t *out4);
int phb_solver_group_finish(const phb_engine *e, const phb_step *st, const int64_t *group, int32_t B, void *stream);

int phb_solver_group(const phb_engine *e, const phb_step *st, const int64_t *group, int32_t B,
                     void *stream);

/* Allocation-free form of phb_solver_group.  It has no counterpart in the reference.
 *
 * For callers that cannot allocate device memory at the point where they run a
 * reconstruction step: e.g. a plugin inside an acquisition or instrument-control
 * process whose device memory is budgeted and owned by the host application, or
 * code running under an allocator that forbids foreign allocations.  Such callers
 * pass the same inputs and outputs as to phb_solver_group; `e->workspace` and
 * `e->workspace_bytes` are ignored.  The scratch is a fixed 64 MiB array that is
 * part of this library (every GPU that loads the library holds it until the
 * process exits); a problem whose phb_engine_workspace_bytes(N, M, S, B, H, W)
 * exceeds 64 MiB is rejected with PHB_ERR_SCRATCH_LIMIT.
 *
 * Each call rebuilds its tables from the inputs and clears every accumulator,
 * so calls are independent; no cudaMalloc, cudaFree or allocating library
 * routine is called.  All calls share the one array: calls whose work overlaps
 * on the GPU (other streams, other threads) race and corrupt each other -- order
 * them on one stream.  The first call on a device looks up the array's device
 * address (cudaGetSymbolAddress); make that first call before any stream
 * capture.  Besides that, EVERY call copies the propagator check's result to
 * the host and waits for its stream to finish before it launches the step, so
 * no call can be recorded under stream capture (CUDA graphs).
 * PHB_FLAG_PARTIAL is refused with PHB_ERR_UNSUPPORTED: a partial share left in
 * the library's array could not be summed over ranks by the caller, and the
 * next call clears it. */
int phb_solver_group_static(const phb_engine *e, const phb_step *st, const int64_t *group, int32_t B,
                            void *stream);

/* ------------------------------------------------------ gradient-engine updates
 * optax semantics of phaser/engines/gradient/solvers.py:88-138 on device arrays:
 * d = grad_scale * grad; SGD (optax.trace momentum / Nesterov, then lr), Adam
 * (optax.scale_by_adam, |d|^2 second moment for complex d, then lr) or Polyak
 * (scale_by_learning_rate(scaling) then scale_by_polyak(max_lr, f_min, eps): the
 * stochastic Polyak step min((loss - f_min) / (q + eps), max_lr), or 0 when
 * q + eps <= 2^-52, with q = *polyak_sq_norm = sum |scaling d|^2 over all of the
 * solver's parameters and loss = *polyak_loss, both device float64); the update
 * is added to `param`, or written to `update_out` when that is non-NULL. */
#define PHB_OPTIM_SGD    0
#define PHB_OPTIM_ADAM   1
#define PHB_OPTIM_POLYAK 2

typedef struct phb_optim {
    int32_t kind, nesterov;
    float *param;             /* n elements (complex pairs when complex_elems) */
    const float *grad;        /* same layout as param */
    float *state1;            /* SGD trace / Adam first moment, same layout; NULL if unused */
    float *state2;            /* Adam second moment: n reals */
    float *update_out;        /* optional: write the update instead of adding it */
    int64_t n;
    int32_t complex_elems;
    float grad_scale, lr, momentum, b1, b2, eps, eps_root;
    int64_t count;            /* Adam: step count including this update (>= 1) */
    const double *polyak_sq_norm;
    const double *polyak_loss;
    float polyak_scaling, polyak_max_lr, polyak_f_min, polyak_eps;
    int32_t *status;          /* optional: set to status_code (if still -1) when an updated */
    int32_t status_code;      /* parameter value is NaN or inf (run.py:281 check_finite) */
} phb_optim;

int phb_optimizer_update(const phb_optim *o, void *stream);

/* *out += sum over x[0:n] of (scale * x)^2 (float64 accumulation). */
int phb_sq_norm_f32(const float *x, int64_t n, float scale, double *out, void *stream);

/* param (n x 2) += update - mean(update): position updates keep the scan centred
 * (phaser/engines/gradient/run.py:115-118). */
int phb_add_centred(float *param, const float *update, int64_t n, void *stream);

/* ------------------------------------------------------------- constraints
 * RegularizeLayers (phaser/engines/common/regularizers.py:86-132): for every object
 * pixel, O <- weight * exp(convolve1d(log O, taps, axis=0, mode='nearest'))
 * + (1 - weight) * O over the S slices; `taps` (n_taps odd, device float32) are the
 * normalised Gaussian the reference builds.  S <= 96. */
int phb_regularize_layers_c64(void *obj, int64_t S, int64_t H, int64_t W, const float *taps, int32_t n_taps,
                              float weight, void *stream);

/* ObjLowPass / ObjGaussian (regularizers.py:135-192): per slice
 * O <- ifft2(filter * fft2(O)) with phaser's centred transforms (the centring
 * shifts cancel), `filter` (H, W) float32 in numpy.fft.fftfreq order on the
 * device, any H and W.  `scratch`: phb_object_filter_scratch_bytes(S, H, W). */
size_t phb_object_filter_scratch_bytes(int64_t S, int64_t H, int64_t W);
int phb_object_filter_c64(void *obj, int64_t S, int64_t H, int64_t W, const float *filter, void *scratch,
                          void *stream);

/* RemovePhaseRamp (regularizers.py:67-83, phaser/utils/image.py:30-55): per slice,
 * the least-squares plane p0 + p1 x + p2 y of angle(O) over the region rows
 * [y0, y1) and columns [x0, x1) is removed from the phase; |O| is kept.
 * `sums`: device float64 scratch of 3 S values. */
int phb_remove_phase_ramp_c64(void *obj, int64_t S, int64_t H, int64_t W, int64_t y0, int64_t y1, int64_t x0,
                              int64_t x1, double *sums, void *stream);

/* UnstructuredGaussian for per-position (n, 2) values such as tilts
 * (regularizers.py:430-497, 'tilt_gaussian'): nearest-position image on the object
 * grid, blurred with `filter` (H, W) (exp(-2 pi^2 sigma^2 k^2), fftfreq order), sampled
 * back at each position's rounded pixel, blended with `weight`.
 * `scratch`: phb_smooth_positions_scratch_bytes(H, W). */
size_t phb_smooth_positions_scratch_bytes(int64_t H, int64_t W);
int phb_smooth_position_values(float *vals, const float *scan, int64_t n, int64_t H, int64_t W, double corner_y,
                               double corner_x, double samp_y, double samp_x, const float *filter, float weight,
                               void *scratch, void *stream);

/* Cost regularisers of the gradient engine on the object (regularizers.py:195-351):
 * obj_l1 sum|O-1|, obj_l2 sum|O-1|^2, obj_phase_l1 sum|angle O|, obj_tikh
 * sum|diff_x O|^2 + |diff_y O|^2, obj_tv sum sqrt(|g_y|^2 + |g_x|^2 + tv_eps)
 * (forward differences, zero at the far edge), layers_tikh sum|diff_z O|^2,
 * layers_tv sum|diff_z O|; each weighted by its cost, all by `scale` (the
 * group's share B / n_pos).  Adds the total to *loss (device float64) and, if
 * `grad` (S, H, W complex64) is non-NULL, dL/dRe + i dL/dIm to it. */
typedef struct phb_obj_reg {
    float l1, l2, phase_l1, tikh, tv, tv_eps, layers_tikh, layers_tv, scale;
} phb_obj_reg;

int phb_object_regularizers(const void *obj, int64_t S, int64_t H, int64_t W, const phb_obj_reg *reg, void *grad,
                            double *loss, void *stream);

/* Fourier-space cost regularisers of the gradient engine.
 * Probe (regularizers.py:354-426, scale 1): with R = fft2(P) (M, N, N), N = 64 / 128:
 * probe_phase_tikh sum |diff angle R|^2, probe_recip_tikh sum |diff fftshift R|^2,
 * probe_recip_tv sum sqrt(|g_y|^2 + |g_x|^2 + tv_eps) of fftshift R.  Adds the value to
 * *loss and, if `grad` is non-NULL, dL/dRe + i dL/dIm of P to it.
 * Object (regularizers.py:233-253): obj_recip_l1 cost * sum |fft2(prod_s O_s)| (any H, W;
 * `cost` already includes the group scale B / n_pos). */
typedef struct phb_probe_reg {
    float phase_tikh, recip_tikh, recip_tv, tv_eps;
} phb_probe_reg;

size_t phb_probe_regularizers_scratch_bytes(int32_t M, int32_t N);
int phb_probe_regularizers(const void *probe, int32_t M, int32_t N, const phb_probe_reg *reg, void *grad,
                           double *loss, void *scratch, void *stream);
size_t phb_object_recip_l1_scratch_bytes(int64_t S, int64_t H, int64_t W);
int phb_object_recip_l1(const void *obj, int64_t S, int64_t H, int64_t W, float cost, void *grad, double *loss,
                        void *scratch, void *stream);

/* ---------------------------------------------------- learned warm start
 * A small convolutional network (no counterpart in the reference) predicts the
 * object patch under the probe from each diffraction pattern; the stitched
 * prediction seeds the iterative solvers.  Activations NCHW float32, weights
 * (Co, Ci, 3, 3) bfloat16, accumulation float32, padding 1, stride 1 or 2
 * (Ho = Hi / stride).  The caller zeroes dw / db before phb_conv3x3_bwd_weight,
 * which accumulates into them. */
int phb_conv3x3_fwd(const float *in, const void *w_bf16, const float *bias, float *out, int32_t Nb, int32_t Ci,
                    int32_t Hi, int32_t Wi, int32_t Co, int32_t stride, int32_t relu, void *stream);
/* Failure-detection probe of the bounded mbarrier waits of the tensor-core kernels
 * (each gives up after 2^22 attempts; the CTA then writes NaN outputs, drains its
 * MMAs and frees its tensor memory).  One thread waits on a shared-memory mbarrier
 * that nothing completes (arrive = 0) or that one arrival completes first
 * (arrive = 1), for at most `limit` attempts (1 .. 2^22); out[0] (device int32) = 1 if
 * the wait saw the phase complete, 0 if it gave up. */
int phb_wait_probe(int32_t arrive, int64_t limit, int32_t *out, void *stream);
int phb_conv3x3_bwd_data(const float *dout, const void *w_bf16, float *din, int32_t Nb, int32_t Ci, int32_t Hi,
                         int32_t Wi, int32_t Co, int32_t stride, void *stream);
int phb_conv3x3_bwd_weight(const float *in, const float *dout, float *dw, float *db, int32_t Nb, int32_t Ci,
                           int32_t Hi, int32_t Wi, int32_t Co, int32_t stride, void *stream);
int phb_relu_bwd(float *grad, const float *y, int64_t n, void *stream);   /* grad *= (y > 0) */
int phb_upsample2(const float *in, float *out, int64_t planes, int32_t H, int32_t W, void *stream);
int phb_upsample2_bwd(const float *gout, float *gin, int64_t planes, int32_t H, int32_t W, void *stream);
/* *loss += mean (pred - target)^2 (float64), grad = d/dpred (either may be NULL) */
int phb_mse(const float *pred, const float *target, float *grad, int64_t n, double *loss, void *stream);
int phb_to_bf16(const float *x, void *y, int64_t n, void *stream);
/* network input: log(1 + I) of each pattern (rows `index`, or 0..B-1 when NULL) over the
 * crop x crop detector window centred on zero frequency, binned bin x bin, mirrored through
 * zero frequency (k -> -k) when flip != 0, scaled to a maximum of 1: (B, crop/bin, crop/bin) */
int phb_pattern_features(const float *patterns, const int64_t *index, int32_t B, int32_t N, int32_t crop,
                         int32_t bin, int32_t flip, float *out, void *stream);
/* training targets: centred P x P patch of the projected object `proj` (H, W) under each
 * position's cutout (exact reference cutout start), as (Re - 1, Im): (B, 2, P, P) */
int phb_patch_targets(const void *proj, int64_t H, int64_t W, const float *scan, const int64_t *index, int32_t B,
                      double corner_y, double corner_x, double samp_y, double samp_x, int32_t N, int32_t P,
                      float *out, void *stream);
/* stitching: accumulate predicted (B, 2, P, P) patches, each pixel weighted by window (P x P,
 * NULL = 1), into acc (H, W complex) and wgt (H, W); then obj = acc / wgt where covered, 1 elsewhere */
int phb_stitch_patches(const float *pred, const float *scan, const int64_t *index, int32_t B, double corner_y,
                       double corner_x, double samp_y, double samp_x, int32_t N, int32_t P, const float *window,
                       void *acc, float *wgt, int64_t H, int64_t W, void *stream);
int phb_stitch_finish(const void *acc, const float *wgt, void *obj, int64_t n, void *stream);
/* product over the S slices of an (S, HW) complex64 object */
int phb_project_slices(const void *obj, int64_t S, int64_t HW, void *out, void *stream);

/* ---- state preparation in front of the engines (phaser/execute.py:334-402) ----
 * Resampling of a stack of batch (H, W) planes onto (Ho, Wo): output pixel (i, j) is
 * the bilinear interpolation, at (my * i + oy, mx * j + ox), of the input extended by
 * cval beyond its edges -- scipy.ndimage.affine_transform with a diagonal matrix,
 * order 1, mode 'grid-constant' (phaser/utils/image.py:151-195), as called by
 * Sampling.resample (num.py:713-733) and ObjectSampling.resample (object.py:430-467).
 * recip != 0 reads the input through fftshift and writes through ifftshift
 * (Sampling.resample_recip, num.py:735-750) for patterns and masks stored with the
 * zero frequency in the corner. */
int phb_resample_c64(const void *in, int64_t batch, int32_t H, int32_t W, void *out, int32_t Ho, int32_t Wo,
                     double my, double mx, double oy, double ox, float cval_re, float cval_im, int32_t recip,
                     void *stream);
int phb_resample_f32(const float *in, int64_t batch, int32_t H, int32_t W, float *out, int32_t Ho, int32_t Wo,
                     double my, double mx, double oy, double ox, float cval, int32_t recip, void *stream);
/* Reslicing along z (resample_slices, phaser/utils/object.py:56-157): out[i] =
 * exp(new_t[i] * (wa[i] L(ja[i]) + wb[i] L(jb[i]))) per pixel, with L(k) =
 * log(obj[k-1]) / old_t[k-1] for 1 <= k <= S_old and the padding slice for k = 0 and
 * k = S_old + 1 (pad_mode 0 vacuum = 0, 1 edge = L(1) / L(S_old), 2 average = nanmean
 * of L over the slices).  Tables are host arrays of S_new entries (S_old, S_new <= 128);
 * the caller computes them from the slice centres (_interp1d, object.py:160-185). */
int phb_resample_slices_c64(const void *obj, int32_t S_old, int64_t HW, const float *old_t, void *out,
                            int32_t S_new, const float *new_t, const int32_t *ja, const int32_t *jb,
                            const float *wa, const float *wb, int32_t pad_mode, void *stream);

/* Per-iteration position update (phaser/engines/conventional/run.py:95-110 with
 * phaser/engines/common/position_correction.py): subtract mean, momentum or
 * steepest-descent step with norm clipping, subtract mean, scan += update, and
 * count positions completely outside the object (-> *n_outside, device int). */
int phb_position_update(float *scan, float *pos_update, float *momentum_state, int64_t n_pos,
                        int32_t use_momentum, float step_size, float max_step /* <= 0: none */,
                        float momentum, double obj_min_y, double obj_min_x,
                        double obj_max_y, double obj_max_x, int32_t *n_outside, void *stream);

/* Count positions completely outside the object (-> *n_outside, device int): the
 * check of phaser/utils/object.py:288-289 on the device, for the gradient engine's
 * position updates (phaser/engines/gradient/run.py:330-349), so an iteration needs no
 * host copy of the scan. */
int phb_count_outside(const float *scan, int64_t n_pos, double obj_min_y, double obj_min_x, double obj_max_y,
                      double obj_max_x, int32_t *n_outside, void *stream);

/* Start of an iteration: *status = -1, errors[0:n] = NaN. */
int phb_iteration_reset(int32_t *status, float *errors, int64_t n, void *stream);

/* End of an iteration: out[0] = *status, out[1] = *n_outside (or 0 if NULL),
 * out[2] = nanmean(errors[0:n]) (NaN if none), out[3] = number of non-NaN errors;
 * `out` is 4 float64 (device memory, or host memory the device can write). */
int phb_iteration_report(const int32_t *status, const int32_t *n_outside, const float *errors, int64_t n,
                         double *out, void *stream);

/* Kernel launches issued by this library since it was loaded (all streams). */
int64_t phb_kernel_launches(void);

/* FP32 CUDA-core throughput of the current device, measured (no counterpart in the
 * reference: the denominator of the FP32-pipe roofline fraction).  Eight independent
 * FMA chains per thread, 64 warps per SM, `iters` FMAs per chain; one untimed launch,
 * then one launch timed with CUDA events on `stream`.  Synchronises on `stream`.
 * *tflops = FLOP / time (2 FLOP per FMA), *ms the timed launch (may be NULL). */
int phb_fp32_peak(int32_t iters, double *tflops, float *ms, void *stream);

/* cudaEvent_t helpers for callers without a CUDA runtime binding. */
int phb_event_create(void **event);
int phb_event_destroy(void *event);
int phb_event_record(void *event, void *stream);
int phb_event_elapsed_ms(void *start, void *end, float *ms);   /* synchronises on `end` */

/* nanmean of `values` (n float32) into *out (float64); count of non-NaN into *count. */
int phb_nanmean(const float *values, int64_t n, double *out, int64_t *count, void *stream);

/* isfinite over a complex64 array: sets *status to `code` if any element is NaN/inf. */
int phb_check_finite_c64(const void *arr, int64_t n, int32_t *status, int32_t code, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* PHASER_B200_H */
