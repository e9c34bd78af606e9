// ref_setup_shim.cpp -- TEST INFRASTRUCTURE ONLY.
//
// Links the reference's own host-setup sources (trifac.c, areanorm.c,
// sphfunc.c, ellfit.c, ludcmp.c, lubksb.c, memory.c, compiled in place by
// oracle/Makefile) into oracle/_ref/libref_setup.so, so that the oracle's
// C restatement of the shape setup can be compared bit-for-bit with the
// reference.  This file only provides the globals those sources expect
// (globals.h) and the vertex-direction loop that the reference keeps inline
// in main() (period_search_BOINC.cpp:790-823).
#include <cmath>
#include <cstring>

#include "constants.h"
#include "declarations.h"

int l_max, m_max, n_iter, last_call, n_coef, num_fac, l_curves, n_ph_par,
    l_points[MAX_LC + 1], in_rel[MAX_LC + 1], deallocate, max_l_points;
double o_chi_square, chi_square, a_lambda, a_lamda_incr, a_lamda_incrr, a_lamda_start, phi_0, scale,
    area[MAX_N_FAC + 1], d_area[MAX_N_FAC + 1], sclnw[MAX_LC + 1], y_out[MAX_N_OBS + 1],
    f_c[MAX_LM + 1][MAX_N_FAC + 1], f_s[MAX_LM + 1][MAX_N_FAC + 1],
    t_c[MAX_N_FAC + 1][MAX_LM + 1], t_s[MAX_N_FAC + 1][MAX_LM + 1],
    d_sphere[MAX_N_PAR + 1][MAX_N_FAC + 1], d_g[MAX_N_FAC + 1][MAX_N_PAR + 1],
    normal[3][MAX_N_FAC + 1], bl_matrix[4][4], pleg[MAX_LM + 1][MAX_LM + 1][MAX_N_FAC + 1],
    d_bl_matrix[3][4][4], weight[MAX_N_OBS + 1];

// Returns 0 on success; arrays are laid out like the oracle's
// (normal[f*3+i], d_area[f], dsph[f*n_coef + k-1], cg[k-1]).
extern "C" int ref_setup_shape(int lmax, int mmax, int nrows, double a, double b, double c,
                               double *normal_out, double *darea_out, double *dsph_out,
                               double *cg_out)
{
    int nfac = 8 * nrows * nrows;
    if (nfac > MAX_N_FAC || lmax > MAX_LM) return 1;
    l_max = lmax;
    m_max = mmax;
    int nc = 0;
    for (int m = 0; m <= m_max; m++)
        for (int l = m; l <= l_max; l++) {
            nc++;
            if (m != 0) nc++;
        }
    double *t = vector_double(MAX_N_FAC);
    double *f = vector_double(MAX_N_FAC);
    double *at = vector_double(MAX_N_FAC);
    double *af = vector_double(MAX_N_FAC);
    int **ifp = matrix_int(MAX_N_FAC, 4);
    double *cg = vector_double(MAX_N_PAR);
    double dth = PI / (2 * nrows);
    int k = 1;
    t[1] = 0;
    f[1] = 0;
    for (int i = 1; i <= nrows; i++) {
        double dph = PI / (2 * i);
        for (int j = 0; j <= 4 * i - 1; j++) {
            k++;
            t[k] = i * dth;
            f[k] = j * dph;
        }
    }
    for (int i = nrows - 1; i >= 1; i--) {
        double dph = PI / (2 * i);
        for (int j = 0; j <= 4 * i - 1; j++) {
            k++;
            t[k] = PI - i * dth;
            f[k] = j * dph;
        }
    }
    int ndir = k + 1;
    t[ndir] = PI;
    f[ndir] = 0;
    trifac(nrows, ifp);
    areanorm(t, f, ndir, nfac, ifp, at, af);
    sphfunc(nfac, at, af);
    ellfit(cg, a, b, c, nfac, nc, at, af);
    for (int i = 0; i < nfac; i++) {
        for (int q = 0; q < 3; q++) normal_out[i * 3 + q] = normal[q][i];
        darea_out[i] = d_area[i];
        for (int kk = 1; kk <= nc; kk++) dsph_out[i * nc + kk - 1] = d_sphere[kk][i];
    }
    for (int i = 0; i < nc; i++) cg_out[i] = cg[i];
    deallocate_vector(t);
    deallocate_vector(f);
    deallocate_vector(at);
    deallocate_vector(af);
    deallocate_vector(cg);
    deallocate_matrix_int(ifp, MAX_N_FAC);
    return 0;
}
