/*
 * ps_oracle.h -- CPU FP64 oracle for the PeriodSearch convex-inversion hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference
 * algorithm (PeriodSearch, period_search_BOINC.cpp + start_CUDA.cu + Start.cu
 * and the host setup files trifac.c / areanorm.c / sphfunc.c / ellfit.c /
 * ludcmp.c / lubksb.c).  It is the checker for the CUDA product path and the
 * timed CPU baseline; nothing in the product links or calls it.
 *
 * Parity pin: the host-setup restatement (trifac/areanorm/sphfunc/ellfit) is
 * checked bit-for-bit against the reference's own C sources compiled by
 * oracle/Makefile into oracle/_ref.  The LM fit itself exists in the reference
 * only as CUDA code (Start.cu); the fit restatement is pinned against the
 * reference GPU build run on the same inputs where that build is available,
 * otherwise by the validator envelope (see the repository's DESIGN notes).
 *
 * Conventions (mirroring the reference):
 *   parameter vector a[1..ma] (1-based): 1..nc shape coefficients, nc+1 beta'
 *   (pi/2 - beta), nc+2 lambda, nc+3 omega [rad/day], nc+4..nc+6 phase function
 *   (A, D, k), ma-1 = ln(Lambert weight), ma = Lommel-Seeliger weight.
 *   ma = nc + 8.  ia[1..ma] marks fitted parameters.
 */
#ifndef PS_ORACLE_H
#define PS_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PSO_MAX_PAR 128      /* ma <= 89 for lmax = 8 */
#define PSO_N_POLES 10
#define PSO_TINY 1e-8        /* constants.h:16 */
#define PSO_MAX_N_ITER 60    /* constants.h:12 */

/* Quirk bits: reproduce documented reference-GPU behaviour instead of the
   Numerical-Recipes-correct one. */
#define PSO_QUIRK_PRECALC_CONW 1  /* start_CUDA.cu:476 uploads the pointer bits of
                                     conw_r, so the precalc rms uses conw_r ~ 0 */

/* One object, after parsing and host setup.  All arrays owned by the caller. */
typedef struct pso_model {
    int n_points;          /* real data points, pseudo-points excluded */
    int n_curves;          /* real lightcurves, pseudo-curve excluded */
    const int *curve_len;  /* [n_curves] */
    const int *curve_rel;  /* [n_curves] 1 = relative (renormalised), 0 = calibrated */
    const double *tim;     /* [n_points] JD - jd0 */
    const double *ee;      /* [n_points*3] unit vector to the observer (xyz) */
    const double *ee0;     /* [n_points*3] unit vector to the Sun (xyz) */
    const double *bright;  /* [n_points] */
    const double *sig;     /* [n_points] per-curve mean brightness */
    const double *sigr2;   /* [n_points] 1/(sig*sig) as the host computed it */
    const double *weight;  /* [n_points] */
    int n_fac;
    int n_coef;
    const double *normal;  /* [n_fac*3] */
    const double *d_area;  /* [n_fac] */
    const double *dsph;    /* [n_fac*n_coef]: dsph[f*n_coef + k-1] = Y_k(facet f) */
    const double *cg_first;/* [n_coef] */
    /* fit constants */
    double phi0;           /* rad */
    double par[3];         /* initial phase-function parameters */
    double lcl;            /* ln(initial Lambert coefficient) */
    double alamda_start, alamda_incr, alamda_incrr;
    double beta_pole[PSO_N_POLES], lambda_pole[PSO_N_POLES];  /* degrees */
    int ia[PSO_MAX_PAR + 1];  /* 1-based fitted-parameter mask, length ma+1 */
    int n_iter_max, n_iter_min;
    double iter_diff_max;
    double conw_r;         /* regularisation weight for the pseudo-point sigma */
    double conw_r_dev;     /* weight used in the rms (== conw_r unless quirked) */
} pso_model;

typedef struct pso_fit_result {
    double dev;            /* final rms (dev_new) */
    double dark;           /* dark-facet percentage */
    double per;            /* period [days] = 2 pi / omega */
    double lambda_deg;
    double beta_deg;
    double chisq;          /* final Chisq */
    int niter;
    int status;            /* bit 0: singular pivot met, bit 1: NaN chisq met */
} pso_fit_result;

typedef struct pso_line {
    double period_h, rms, chisq, dark, lambda_deg, beta_deg;
    int valid;
} pso_line;

/* ---- host setup (period_search_BOINC.cpp:782-837 and L1 files) ---- */
int pso_n_coef(int l_max, int m_max);
/* Builds normals, areas, the Laplace-series basis dsph and the ellipsoid fit
   cg_first for the given triangulation.  Arrays sized n_fac = 8 nrows^2 and
   n_coef.  Returns 0 on success. */
int pso_setup_shape(int l_max, int m_max, int nrows, double a, double b, double c,
                    double *normal, double *d_area, double *dsph, double *cg_first);

/* ---- kernels of the fit ---- */
/* One mrqcof evaluation at a[1..ma]: chi^2, alpha (mfit x mfit, full
   symmetric, row-major) and beta (mfit).  Optional rows[n_points+3][ma+1]
   receives the raw (un-renormalised) derivative rows with ymod in column ma,
   in parameter order (column p-1 = d/da_p). area_sum receives sum(Areag). */
double pso_eval(const pso_model *m, const double *a, double *alpha, double *beta,
                double *rows, double *area_sum);

/* Full LM fit of one (frequency, pole) item. */
void pso_fit(const pso_model *m, double freq_start, double freq_step, int n_freq,
             int pole, pso_fit_result *res);
/* Runs n items (frequency index n_freq[i] 1-based, pole[i] 0-based) on
   n_threads threads. */
void pso_fit_batch(const pso_model *m, double freq_start, double freq_step,
                   const int *n_freq, const int *pole, int n, pso_fit_result *res,
                   int n_threads);

/* CUDAPrecalc restated: 10 test periods x 10 poles, dark-facet average.
   Returns new conw_r through *conw_r and sets *new_conw. */
void pso_precalc(pso_model *m, double freq_start, double freq_step,
                 double *conw_r, int *new_conw, int quirks, int n_threads);

/* CUDAStart restated: one line per frequency n = n_start..n_max. */
int pso_scan(const pso_model *m, double freq_start, double freq_end, double freq_step,
             int n_start, pso_line *lines, int max_lines, int n_threads);

/* Whole application: reads period_search_in, writes period_search_out. */
int pso_run_file(const char *in_path, const char *out_path, int quirks, int n_threads,
                 int max_freq);

/* GJ solve with full pivoting (the reference's mrqmin_1_end_opt pivot rule).
   a is n x n row-major (destroyed), b (n) becomes the solution.  Returns 0,
   1 (pivot bookkeeping error) or 2 (zero pivot; b holds the partial result). */
int pso_gauss_solve(double *a, int n, double *b);

#ifdef __cplusplus
}
#endif
#endif
