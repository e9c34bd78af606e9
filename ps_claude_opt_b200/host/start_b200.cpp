// start_b200.cpp -- the binding a PeriodSearch maintainer adds: it replaces
// the reference's start_CUDA.cu and implements the reference's own four GPU
// entry points (start_CUDA.h:2-16 -- CUDAPrepare, CUDAPrecalc, CUDAStart,
// CUDAUnprepare) on the B200 engine's C ABI (include/ps_b200.h).  The
// reference's main (period_search_BOINC.cpp:171-907) is built unchanged
// against this file and linked with -lps_b200.
//
// What it converts: the reference passes 1-based arrays (betaPole[1..10],
// par[1..3], ia_par[1..3], brightness/sig/sigr2/weight[1..ndata+3]),
// component-major geometry ee[3][MAX_N_OBS+1], and reads the lightcurve
// layout and shape tables from process globals (globals.h:6-22: l_curves,
// l_points, in_rel, normal, d_area, d_sphere, n_coef, weight), with the
// convexity pseudo-curve appended as curve l_curves
// (period_search_BOINC.cpp:587-592).  The C ABI takes 0-based arrays,
// point-major geometry, explicit ps_curves / ps_shape, and ndata without the
// three pseudo-points.  CUDAStart prints the lines the engine returns in the
// reference's format (start_CUDA.cu:1220-1227).
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "constants.h"
#include "globals.h"
#include "mfile.h"
#include "ps_b200.h"

namespace {

ps_gpu *g_ps = nullptr;

// The lightcurve layout without the pseudo-curve, and the shape tables.
struct Tables {
    std::vector<int32_t> len, rel;
    std::vector<double> nor, dsph;
    ps_curves curves;
    ps_shape shape;
};

void fill_tables(Tables &t, int numfac)
{
    for (int i = 1; i < l_curves; ++i) {
        t.len.push_back(l_points[i]);
        t.rel.push_back(in_rel[i]);
    }
    t.nor.resize(3 * (size_t)numfac);
    t.dsph.resize((size_t)numfac * n_coef);
    for (int f = 0; f < numfac; ++f) {
        for (int k = 0; k < 3; ++k) t.nor[3 * f + k] = normal[k][f];
        for (int k = 0; k < n_coef; ++k) t.dsph[(size_t)f * n_coef + k] = d_sphere[k + 1][f];
    }
    t.curves = {(int32_t)t.len.size(), t.len.data(), t.rel.data()};
    t.shape = {n_coef, t.nor.data(), d_area, t.dsph.data()};
}

}  // namespace

int CUDAPrepare(int dev, double *beta_pole, double *lambda_pole, double *par, double cl, double a_start,
                double a_incr, double a_incrr, double ee[][MAX_N_OBS + 1], double ee0[][MAX_N_OBS + 1],
                double *tim, double phi0, int /*checkex*/, int ndata)
{
    // ndata here excludes the pseudo-points (period_search_BOINC.cpp:638)
    std::vector<double> e(3 * (size_t)ndata), e0(3 * (size_t)ndata);
    for (int i = 0; i < ndata; ++i)
        for (int k = 0; k < 3; ++k) {
            e[3 * (size_t)i + k] = ee[k][i];
            e0[3 * (size_t)i + k] = ee0[k][i];
        }
    const ps_status s = ps_gpu_prepare(dev, beta_pole + 1, lambda_pole + 1, par + 1, cl, a_start, a_incr,
                                       a_incrr, e.data(), e0.data(), tim, phi0, ndata, weight + 1, &g_ps);
    if (s != PS_OK) std::fprintf(stderr, "ps_gpu_prepare: %s\n", ps_last_error());
    return s == PS_OK;
}

int CUDAPrecalc(int /*dev*/, double f_start, double f_end, double f_step, double stop, int n_iter_min,
                double *conw_r, int ndata, int *ia, int *ia_par, int *new_conw, double *cg_first, double *sig,
                double *sigr2, int numfac, double *brightness)
{
    Tables t;
    fill_tables(t, numfac);
    // ndata here includes the 3 pseudo-points (period_search_BOINC.cpp:662-671)
    const ps_status s = ps_gpu_precalc(g_ps, f_start, f_end, f_step, stop, n_iter_min, conw_r, ndata - 3, ia,
                                       ia_par + 1, new_conw, cg_first, sig + 1, sigr2 + 1, numfac,
                                       brightness + 1, &t.curves, &t.shape);
    if (s != PS_OK) {
        std::fprintf(stderr, "ps_gpu_precalc: %s\n", ps_last_error());
        std::exit(2);
    }
    return 1;
}

int CUDAStart(int /*dev*/, int n_start_from, double f_start, double f_end, double f_step, double stop,
              int n_iter_min, double conw_r, int ndata, int *ia, int *ia_par, double *cg_first, MFILE &mf,
              double escl, double *sig, double *sigr2, int numfac, double *brightness)
{
    Tables t;
    fill_tables(t, numfac);
    const int n_max = (int)((f_start - f_end) / f_step) + 1;
    std::vector<ps_line> lines(n_max > 0 ? n_max : 1);
    int32_t n_lines = 0;
    const ps_status s = ps_gpu_start(g_ps, n_start_from, f_start, f_end, f_step, stop, n_iter_min, conw_r,
                                     ndata - 3, ia, ia_par + 1, cg_first, escl, sig + 1, sigr2 + 1, numfac,
                                     brightness + 1, &t.curves, &t.shape, lines.data(), (int32_t)lines.size(),
                                     &n_lines, nullptr, nullptr);
    if (s != PS_OK) {
        std::fprintf(stderr, "ps_gpu_start: %s\n", ps_last_error());
        std::exit(2);
    }
    for (int i = 0; i < n_lines; ++i) {
        const ps_line &l = lines[i];
        // round() before %4.0f, as the reference prints the pole
        mf.printf("%.8f  %.6f  %.6f %4.1f %4.0f %4.0f\n", l.period_h, l.rms, l.chisq, l.dark,
                  std::round(l.lambda_deg), std::round(l.beta_deg));
    }
    return 1;
}

void CUDAUnprepare(void)
{
    ps_gpu_unprepare(g_ps);
    g_ps = nullptr;
}
