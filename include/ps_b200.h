/*
 * ps_b200.h -- C ABI of the B200 PeriodSearch fit engine.
 *
 * Drop-in replacement for the reference's GPU boundary (start_CUDA.h:2-16 of
 * PeriodSearch): CUDAPrepare / CUDAPrecalc / CUDAStart / CUDAUnprepare.  The
 * reference reads part of its input from process globals (globals.h:6-22:
 * l_curves, l_points, in_rel, weight, normal, d_area, d_sphere, n_coef); here
 * those travel explicitly in ps_curves / ps_shape.  Nothing in this ABI exits
 * the process: every entry point returns a ps_status and ps_last_error()
 * describes the most recent failure.
 *
 * Array conventions (all arrays 0-based, owned by the caller, only read):
 *   ndata        number of real data points (the reference's ndata without
 *                the 3 convexity pseudo-points it appends)
 *   tim[i]       JD - jd0 of point i, days
 *   ee[3*i+k]    unit vector to the observer, ee0[3*i+k] to the Sun
 *   brightness[i], sig[i] (per-curve mean brightness), sigr2[i] = 1/sig^2,
 *   weight[i]    per-point weight
 *   ia[p]        1-based fitted mask, p = 1..ma (ma = n_coef + 8), ia[0] unused
 *   ia_par[k]    k = 0..2: fitted flags of the three phase-function parameters
 *   cg_first[k]  k = 0..n_coef-1: initial shape coefficients (ellfit output)
 *   d_sphere[f*n_coef + k]  Laplace basis value of coefficient k at facet f
 *   normal[3*f+k], d_area[f]  facet normals and areas of the Gaussian image
 */
#ifndef PS_B200_H
#define PS_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum ps_status {
    PS_OK = 0,
    PS_ERR_ARG = 1,          /* invalid argument or size beyond a limit */
    PS_ERR_CUDA = 2,         /* CUDA runtime error (message in ps_last_error) */
    PS_ERR_NOT_PREPARED = 3, /* call ps_gpu_prepare first */
    PS_ERR_CANCELLED = 4,    /* progress callback asked to stop */
    PS_ERR_ALLOC = 5         /* device or host allocation failed */
} ps_status;

#define PS_N_POLES 10
#define PS_MAX_PAR 96        /* ma <= 89 (lmax <= 8) */
#define PS_MAX_FAC 1024

/* Device-status bits accumulated over calls (ps_gpu_status). */
#define PS_DEVSTAT_SINGULAR 1   /* a Gauss-Jordan pivot was exactly zero */
#define PS_DEVSTAT_NAN_CHISQ 2  /* an evaluation produced NaN chi^2 */
#define PS_DEVSTAT_TIMEOUT 4    /* a bounded wait for a shared-memory bulk copy gave up;
                                   the CTA stopped and its remaining items are unset */

/* Quirk bits (ps_gpu_set_quirks): reproduce documented reference behaviour. */
#define PS_QUIRK_PRECALC_CONW 1 /* start_CUDA.cu:476 uploads the pointer bits of
                                   conw_r in CUDAPrecalc: the precalc rms then
                                   ignores the regularisation term */

typedef struct ps_gpu ps_gpu;

/* The lightcurve layout (globals l_curves, l_points, in_rel). */
typedef struct ps_curves {
    int32_t n_curves;            /* real curves, the pseudo-curve excluded */
    const int32_t *curve_len;    /* [n_curves] points per curve */
    const int32_t *curve_rel;    /* [n_curves] 1 = relative, 0 = calibrated */
} ps_curves;

/* The Gaussian-image shape model (globals normal, d_area, d_sphere). */
typedef struct ps_shape {
    int32_t n_coef;
    const double *normal;        /* [numfac*3] */
    const double *d_area;        /* [numfac] */
    const double *d_sphere;      /* [numfac*n_coef] */
} ps_shape;

/* One line of period_search_out (start_CUDA.cu:1200-1229). */
typedef struct ps_line {
    double period_h;     /* 24 * per_best */
    double rms;          /* dev_best */
    double chisq;        /* rms^2 * ndata */
    double dark;         /* dark-facet %, or conw_r*escl^2 on the scan's first line */
    double lambda_deg;   /* [0, 360) */
    double beta_deg;
} ps_line;

/* Result of one (frequency, pole) fit. */
typedef struct ps_fit_result {
    double dev, dark, per, lambda_deg, beta_deg, chisq;
    int32_t niter, status;
} ps_fit_result;

/* Progress callback: frequencies finished / total.  Non-zero return cancels. */
typedef int (*ps_progress_fn)(void *user, int32_t n_done, int32_t n_total);

/* Replaces CUDAPrepare (start_CUDA.h:2-4, start_CUDA.cu:207-364): opens the
   device, stores the per-point geometry and the fit constants.  cl is the
   linear Lambert coefficient (the reference uploads log(cl)). */
ps_status ps_gpu_prepare(int32_t device, const double *beta_pole, const double *lambda_pole,
                         const double *par, double cl, double alamda_start, double alamda_incr,
                         double alamda_incrr, const double *ee, const double *ee0,
                         const double *tim, double phi0, int32_t ndata, const double *weight,
                         ps_gpu **handle);

/* Replaces CUDAPrecalc (start_CUDA.h:10-12, start_CUDA.cu:400-789): fits the
   first 10 trial periods x 10 poles and doubles *conw_r while the mean dark
   facet is >= 1 %, setting *new_conw = 1 once it is below. */
ps_status ps_gpu_precalc(ps_gpu *h, double freq_start, double freq_end, double freq_step,
                         double stop_condition, int32_t n_iter_min, double *conw_r,
                         int32_t ndata, const int32_t *ia, const int32_t *ia_par,
                         int32_t *new_conw, const double *cg_first, const double *sig,
                         const double *sigr2, int32_t numfac, const double *brightness,
                         const ps_curves *curves, const ps_shape *shape);

/* Replaces CUDAStart (start_CUDA.h:6-8, start_CUDA.cu:792-1245): the full
   period scan n = n_start_from..n_max.  Instead of printing into an MFILE it
   fills lines[0..*n_lines) (one per frequency, the best of the 10 poles). */
ps_status ps_gpu_start(ps_gpu *h, int32_t n_start_from, double freq_start, double freq_end,
                       double freq_step, double stop_condition, int32_t n_iter_min,
                       double conw_r, int32_t ndata, const int32_t *ia, const int32_t *ia_par,
                       const double *cg_first, double escl, const double *sig,
                       const double *sigr2, int32_t numfac, const double *brightness,
                       const ps_curves *curves, const ps_shape *shape, ps_line *lines,
                       int32_t max_lines, int32_t *n_lines, ps_progress_fn progress,
                       void *user);

/* Replaces CUDAUnprepare (start_CUDA.h:16, start_CUDA.cu:368-385). */
void ps_gpu_unprepare(ps_gpu *h);

/* One object of a batch scan: the arguments that ps_gpu_prepare,
   ps_gpu_precalc and ps_gpu_start take for it. */
typedef struct ps_object {
    const double *beta_pole, *lambda_pole;   /* [PS_N_POLES], degrees */
    const double *par;                       /* [3] phase-function start values */
    double cl, alamda_start, alamda_incr, alamda_incrr, phi0;
    int32_t ndata;
    const double *tim, *ee, *ee0, *weight, *brightness, *sig, *sigr2;
    const int32_t *ia, *ia_par;
    const double *cg_first;
    int32_t numfac;
    ps_curves curves;
    ps_shape shape;
    double freq_start, freq_end, freq_step, stop_condition;
    int32_t n_iter_min;
    double escl;
    double conw_r;          /* conw / escl^2: the convexity-weight search starts here */
    int32_t n_start_from;   /* first frequency of the scan (>= 1) */
    int32_t max_lines;      /* lines reserved for this object in the output */
} ps_object;

/* The reference's whole flow -- convexity-weight search (CUDAPrecalc), then
   the scan (CUDAStart) -- for n_obj objects at once (no counterpart in the
   reference, which runs one object per process).  Objects of one padded
   coefficient count share one persistent FP64 launch whose device queue
   holds all their (frequency, pole) items, so uneven objects and ragged
   iteration counts even out over the CTAs; each search round is one launch
   per group, and the scans of all groups are one captured CUDA graph.
   Lines of object i go to lines[line_offset[i] .. + n_lines[i]); the final
   convexity weight to conw_r_out[i].  quirks: PS_QUIRK_* for every
   object. */
ps_status ps_gpu_scan_batch(int32_t device, int32_t n_obj, const ps_object *objs, int32_t quirks,
                            ps_line *lines, const int64_t *line_offset, int32_t *n_lines,
                            double *conw_r_out);

/* Tile layout of ps_gpu_scan_batch's groups (no reference counterpart):
   mode 1 (default) times every layout that fits in shared memory -- 32 or 16
   rows per J^T W J tile, per-curve statistics in shared memory or in the
   scratch slab -- on a one-wave, three-iteration sample of the group's own
   items and keeps the fastest (cached per group shape for the process);
   mode 2 is mode 1 with the cache cleared first; mode 0 takes the first
   layout that fits in that order.  Results do not depend on the layout. */
ps_status ps_batch_set_tuning(int32_t mode);
/* JSON description of the last ps_gpu_scan_batch's groups: padded
   coefficient count, objects, resident CTAs, candidate layouts with their
   sample times (ms; -1 where not timed), the chosen layout and whether it
   was timed, cached or the only one.  Copies at most len - 1 bytes and a
   terminating NUL into buf; returns the full length. */
int32_t ps_batch_tuning_report(char *buf, int32_t len);

/* ---- finer-grained entry points (no reference counterpart: the reference
        keeps these steps inside CUDAStart) ---- */

/* Uploads the object and scan configuration used by ps_gpu_fit_items and
   ps_gpu_eval.  conw_r_rms is the weight used in the rms (normally conw_r). */
ps_status ps_gpu_configure(ps_gpu *h, double freq_start, double freq_step, double stop_condition,
                           int32_t n_iter_min, double conw_r, double conw_r_rms, int32_t ndata,
                           const int32_t *ia, const int32_t *ia_par, const double *cg_first,
                           const double *sig, const double *sigr2, int32_t numfac,
                           const double *brightness, const ps_curves *curves,
                           const ps_shape *shape);

/* Runs n LM fits (frequency index n_freq[i] >= 1, pole index pole[i] in 0..9)
   with the configured object; results to out[i]. */
ps_status ps_gpu_fit_items(ps_gpu *h, int32_t n, const int32_t *n_freq, const int32_t *pole,
                           ps_fit_result *out);

/* As ps_gpu_fit_items, but items and results stay in device memory (pointers
   from cudaMalloc) and nothing is synchronised: the call only enqueues the
   fit kernel on the handle's stream.  Used for device-resident timing. */
ps_status ps_gpu_fit_items_device(ps_gpu *h, int32_t n, const int32_t *d_items,
                                  ps_fit_result *d_out);

/* One function evaluation (the reference's mrqcof) at the 1-based parameter
   vector a[0..ma]: chi^2, alpha (mfit x mfit row-major) and beta (mfit). */
ps_status ps_gpu_eval(ps_gpu *h, const double *a, double *chisq, double *alpha, double *beta,
                      double *area_sum);

/* Device-status bits (PS_DEVSTAT_*) accumulated since prepare. */
ps_status ps_gpu_status(ps_gpu *h, int32_t *flags);
ps_status ps_gpu_set_quirks(ps_gpu *h, int32_t quirks);

/* Arithmetic of the fit (no reference counterpart; the reference's own
   reduced-precision path is its df64 FP32-pair emulation, mreal.h:65-517).
   PS_PRECISION_FP64: FP64 throughout (default).  PS_PRECISION_MIXED: the
   facet sweep -- brightness, its parameter derivatives and the per-point
   sums -- runs in FP32, its shape-derivative products on the tensor cores
   as 3xTF32 (high x high + high x low + low x high) with FP32 accumulation,
   the reciprocal of each facet term Newton-refined and the per-point scalar
   sums flushed to FP64 every 8 facets; geometry,
   J^T W J, chi^2, the Gauss-Jordan solve and the lambda update stay FP64.
   For n_coef <= 64 (lmax <= 7).  Takes effect at the next configure (or
   precalc / start, which configure). */
#define PS_PRECISION_FP64 0
#define PS_PRECISION_MIXED 1
ps_status ps_gpu_set_precision(ps_gpu *h, int32_t precision);
/* Per-phase SM clock totals of the fit kernel (diagnostics; no reference
   counterpart).  If out is non-null it receives 12 values accumulated since
   the last call -- cycles in curv, point sort, facet sweep, curve statistics,
   J^T W J tiles (other), pseudo-points, Gauss-Jordan, the rest, tile-copy
   waits, tile staging, tile rank-k updates, then the number of evaluations --
   and the counters restart; enable = 0 switches them off. */
ps_status ps_gpu_phase_clocks(ps_gpu *h, int32_t enable, int64_t *out);
/* The CUDA stream all work of the handle runs on (a cudaStream_t). */
void *ps_gpu_stream(ps_gpu *h);
/* Fit CTAs resident per SM and SM count for the configured object. */
ps_status ps_gpu_occupancy(ps_gpu *h, int32_t *ctas_per_sm, int32_t *n_sm);

/* Allocation-free variant of ps_gpu_fit_items (no counterpart in the
   reference).  For callers that cannot call cudaMalloc: a framework whose
   own caching allocator owns the device memory (an allocation behind its back
   can fail on a full pool or fragment it), or a pipeline that forbids
   allocation once running (cudaMalloc can synchronise the device and stall
   the other streams).  Takes the
   arguments of ps_gpu_prepare + ps_gpu_configure + ps_gpu_fit_items as host
   arrays and writes host results; allocates nothing, on the device or the
   host heap.  All device data live in one file-scope 64 MiB __device__
   array per GPU.  CUDA loads modules lazily, so the array is reserved when
   the first call on a device loads the library's module there, and is held
   until the process exits; a call with n = 0 (every other argument may be
   NULL) does only that -- select the device, load the module, look up the
   array -- so a caller can reserve the 64 MiB at start-up, before its own
   allocator fills the device.  Each call looks up the array's device address
   with the device current; the first call with work also sets the kernel's
   shared-memory limit: make it before any stream capture.  Calls share the
   array and leave their data in it;
   calls that overlap on the GPU race -- serialise them.  Objects whose tables
   plus one CTA's scratch exceed 64 MiB, or with more than 200 lightcurves,
   are rejected with PS_ERR_ARG; smaller ones run on as many CTAs as the
   remaining scratch holds.  stream may be NULL (the legacy default stream);
   the call returns after the results are in out. */
ps_status ps_fit_items_noalloc(int32_t device, void *stream, const double *beta_pole,
                               const double *lambda_pole, const double *par, double cl,
                               double alamda_start, double alamda_incr, double alamda_incrr,
                               const double *ee, const double *ee0, const double *tim, double phi0,
                               const double *weight, double freq_start, double freq_step,
                               double stop_condition, int32_t n_iter_min, double conw_r,
                               double conw_r_rms, int32_t ndata, const int32_t *ia,
                               const int32_t *ia_par, const double *cg_first, const double *sig,
                               const double *sigr2, int32_t numfac, const double *brightness,
                               const ps_curves *curves, const ps_shape *shape, int32_t n,
                               const int32_t *n_freq, const int32_t *pole, ps_fit_result *out);

/* ---- learned frequency screening (no counterpart in the reference, which
        fits every trial frequency) ---- */

/* Phase-folded lightcurve features of n_freq trial frequencies (1/day: 24
   times the grid's 1/hour), 88 per frequency: features[f*88 + 8*s + a] for
   statistic s of the 8 per-curve statistics (phase-dispersion ratios for 64,
   32, 16, 8 bins; shares of harmonics 1..4 in the 32-bin mean curve) and
   aggregate a over the curves (point-weighted mean, mean, std, min,
   25/50/75 % quantiles, max); features[f*88 + 64 + 8*k + s], the same 8
   statistics of fold k of all points together (k = 0 all, 1 before and 2
   after the middle of the time span).  Host arrays; at most 256
   lightcurves. */
ps_status ps_screen_features(int32_t device, int32_t n_points, const double *tim,
                             const double *brightness, const ps_curves *curves, int32_t n_freq,
                             const double *freqs, float *features);

/* Scores of n_freq trial frequencies (1/hour) from a trained screening
   network: lower = more promising.  The 88 features above, standardised per
   feature over these frequencies, pass through n_layers dense layers
   (sizes[0] = 88 .. sizes[n_layers] = 1, ReLU between them, BF16 operands,
   FP32 accumulation); params holds each layer's weights [out][in] then its
   biases [out], FP32, layer after layer. */
ps_status ps_screen_rank(int32_t device, int32_t n_points, const double *tim,
                         const double *brightness, const ps_curves *curves, int32_t n_freq,
                         const double *freqs_per_hour, int32_t n_layers, const int32_t *sizes,
                         const float *params, float *score);

/* Device-pointer kernels of the screening network (BF16 operands, FP32
   accumulation on the tensor cores).  ps_gemm_bf16: C[m][n] (+)= sum_k
   A[m*sam + k*sak] B[k*sbk + n*sbn] (+ bias[n]) (ReLU if relu), written to
   the FP32 C (row stride ldc) and/or the BF16 Cb (row stride ldcb). */
ps_status ps_gemm_bf16(int32_t M, int32_t N, int32_t K, const void *A, int64_t sam, int64_t sak,
                       const void *B, int64_t sbk, int64_t sbn, float *C, int32_t ldc,
                       int32_t accumulate, const float *bias, int32_t relu, void *Cb, int32_t ldcb,
                       void *stream);
/* dz = dh where z > 0, else 0 (FP32 dz and/or BF16 dzb). */
ps_status ps_relu_backward(int64_t n, const float *dh, const float *z, float *dz, void *dzb,
                           void *stream);
/* out[c] = sum over rows r of x[r*cols + c]. */
ps_status ps_column_sum(int32_t rows, int32_t cols, const float *x, float *out, void *stream);
/* One Adam step on FP32 weights w (bias-corrected with step >= 1); wb, if
   not null, receives the BF16 copy. */
ps_status ps_adam_step(int64_t n, float *w, const float *grad, float *m, float *v, float lr,
                       float beta1, float beta2, float eps, int32_t step, void *wb, void *stream);
ps_status ps_to_bf16(int64_t n, const float *x, void *y, void *stream);

/* Host shape setup (trifac.c, areanorm.c, sphfunc.c, ellfit.c of the
   reference): facet normals, areas, Laplace basis and the ellipsoid fit. */
ps_status ps_setup_shape(int32_t l_max, int32_t m_max, int32_t nrows, double a, double b, double c,
                         double *normal, double *d_area, double *d_sphere, double *cg_first);
int32_t ps_n_coef(int32_t l_max, int32_t m_max);

/* FP64 FMA throughput of the device in TFLOP/s (the compute roofline of the
   fit kernel; no reference counterpart). */
ps_status ps_measure_fp64_peak(int32_t device, double *tflops);
/* Test hook (no reference counterpart): one CTA waits, with the fit
   kernel's bounded wait and a limit of `polls` polls, on a bulk-copy barrier
   that nothing completes; *status = PS_DEVSTAT_TIMEOUT when the wait gave up
   (0 if it had completed).  The context stays usable. */
ps_status ps_probe_wait_timeout(int32_t polls, int32_t *status);
/* Test hook: r[i] = the fit kernel's branch-free reciprocal of d[i], on the
   current device (no reference counterpart). */
ps_status ps_probe_reciprocal(int32_t n, const double *d, double *r);
/* Test hook: the fit kernel's full-pivot Gauss-Jordan solve (the solve of
   mrqmin_1_end_opt, Start.cu:2880-3006) of the row-major n x n system a x = b,
   1 <= n <= 89, in one CTA on the current device; x = the solve's da, *err =
   its error code (0, 1 pivot bookkeeping, 2 zero pivot: x then holds the
   partial solution the fit uses). */
ps_status ps_probe_solve(int32_t n, const double *a, const double *b, double *x, int32_t *err);

const char *ps_last_error(void);
const char *ps_version(void);

#ifdef __cplusplus
}
#endif
#endif
