// engine.h -- device-side data layout of the B200 fit engine.
//
// One object's constant tables live in HBM once; every CTA of the persistent
// fit kernel reads them through L1/L2.  Per-fit state lives in shared memory
// (facet areas, the two LM matrices, parameters); the per-point derivative
// rows of one evaluation go to a per-CTA scratch slab in HBM/L2.
#pragma once
#include <cstddef>
#include <cstdint>

namespace psb {

constexpr int kMaxPar = 96;        // ma <= 89 (lmax = 8)
constexpr int kMaxFit = 90;        // mfit <= 89, rounded to even
constexpr int kPoles = 10;
constexpr int kThreads = 256;      // threads per fit CTA
constexpr int kWarps = kThreads / 32;
constexpr int kTile = 32;          // rows per JtWJ tile
constexpr int kMaxFac = 1024;

struct DevObject {
    int n_points, n_curves, n_fac, n_coef, ncp, ma, mfit, row_stride;
    int tile_rows;            // rows per J^T W J tile: 32, or 16 for the largest models
    int cstat_smem;           // 1: per-curve statistics live in shared memory (they fit)
    const double4 *facet;     // [n_fac] {nx, ny, nz, d_area}
    const double *ysh;        // [n_fac][ncp] Laplace basis, zero-padded to ncp
    const double4 *pt_a;      // [n_points] {t, ee.x, ee.y, ee.z}
    const double4 *pt_b;      // [n_points] {ee0.x, ee0.y, ee0.z, brightness}
    const double *pt_w;       // [n_points] sigr2 * weight
    const double4 *pt_rec;    // [n_points] {brightness, sigr2 * weight, curve index, relative flag}
    const int *pt_curve;      // [n_points] curve index
    const int *curve_start;   // [n_curves + 1]
    const int *curve_rel;     // [n_curves]
    const double *curve_sig;  // [n_curves] mean brightness (sigma of a relative curve)
    const int *fidx;          // [mfit] 1-based index of each fitted parameter
    const double *cg_first;   // [n_coef]
    // mixed precision (0: FP64 throughout): the facet sweep runs in FP32 with
    // 3xTF32 tensor-core products; ysh32 holds the basis split into TF32
    // high and low parts, chunk by chunk: [chunk][hi | lo][chunk_facets][ncp]
    int mixed;
    const float *ysh32;
};

struct DevParams {
    double phi0, par[3], lcl, alamda_start, alamda_incr, alamda_incrr;
    double beta_pole[kPoles], lambda_pole[kPoles];
    double iter_diff_max, conw_r, conw_r_dev, freq_start, freq_step;
    int n_iter_max, n_iter_min;
    // optional per-phase SM clock totals [kPhaseSlots] (nullptr: off)
    unsigned long long *phase_cycles;
};

constexpr int kPhaseSlots = 12;  // 11 phases + evaluation count

struct FitItem {
    int n_freq;   // 1-based frequency index
    int pole;     // 0-based pole index
};

struct FitOut {
    double dev, dark, per, lambda_deg, beta_deg, chisq;
    int niter, status;
};

// Result of one stand-alone evaluation (parity hook).
struct EvalOut {
    double *alpha;   // [mfit*mfit]
    double *beta;    // [mfit]
    double *chisq;   // [1]
    double *area;    // [1] sum of facet areas
    const double *a; // [ma+1] parameter vector (1-based)
};

enum StatusBits : int {
    kStatusSingular = 1,
    kStatusNanChisq = 2,
    kStatusTimeout = 4,   // a bounded wait on a bulk copy gave up
};

// Bytes of dynamic shared memory one fit CTA needs.
size_t fit_smem_bytes(int n_fac, int mfit, int ncp, int n_curves, int row_stride, int tile_rows, int cstat_smem,
                      int mixed);
// Largest padded coefficient count the mixed-precision sweep is built for.
constexpr int kMaxMixedNcp = 64;
// Facets per basis chunk of the facet sweep for a padded coefficient count.
int chunk_facets_of(int ncp);
// Doubles of scratch one CTA needs (derivative rows + per-curve statistics).
size_t fit_scratch_doubles(const DevObject &o);
// Padded coefficient count the kernels are compiled for.
int padded_ncoef(int n_coef);

// Launches the persistent fit kernel over n_items items.  queue must point to
// one zeroed int.  Returns a cudaError_t value.
int launch_fits(const DevObject &o, const DevParams &p, const FitItem *items, int n_items,
                int *queue, FitOut *out, double *scratch, size_t scratch_per_cta, int n_ctas,
                int *status, void *stream);
// One evaluation at ev.a, 1 CTA.  rows_out (optional): [n_points][row_stride].
int launch_eval(const DevObject &o, const DevParams &p, EvalOut ev, double *scratch,
                void *stream);
// CTAs per SM the fit kernel reaches for this object.
int fit_ctas_per_sm(const DevObject &o);

// Many objects of one padded coefficient count in one persistent launch (FP64
// kernel).  env carries the largest sizes of the objects (the shared-memory
// layout: n_fac, mfit, n_curves, row_stride) and the common tile_rows and
// cstat_smem; d_objs / d_prms are the objects' tables and constants on the
// device, and an item's pole field is pole | object << 8.
// prepare_batch_kernel sets the kernel's shared-memory limit (once, before
// launching or capturing); launch_fits_batch only enqueues the launch.
int prepare_batch_kernel(const DevObject &env);
int fit_batch_ctas_per_sm(const DevObject &env);
int launch_fits_batch(const DevObject &env, const DevObject *d_objs, const DevParams *d_prms, const FitItem *items,
                      int n_items, int *queue, FitOut *out, double *scratch, size_t scratch_per_cta, int n_ctas,
                      int *status, void *stream);

}  // namespace psb
