/*
 * ps_oracle.c -- CPU FP64 oracle for the PeriodSearch LM-fit hot path.
 *
 * TEST INFRASTRUCTURE ONLY (checker and timed CPU baseline).  The product
 * (ps_claude_opt_b200/csrc) never links or calls this file.
 *
 * Every function names the reference file:line it restates.  Reference paths
 * are relative to the PeriodSearch project root.  Where the reference GPU
 * code is defective (calibrated curves, ia[1]=1 off-by-one) this file follows
 * the Numerical-Recipes mrqcof/mrqmin semantics the GPU code was derived from.
 *
 * Build for parity with -O2 -ffp-contract=off (no FMA contraction) so that
 * results are identical on every x86-64 host of the same image.
 */
#define _GNU_SOURCE
#include "ps_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define PSO_PI 3.14159265358979323846
#define DEG2RAD (PSO_PI / 180)
#define RAD2DEG (180 / PSO_PI)
#define MAX_LM 15

/* ------------------------------------------------------------------------ */
/* Host setup                                                               */
/* ------------------------------------------------------------------------ */

/* Coefficient count of the Laplace series: period_search_BOINC.cpp:782-788 */
int pso_n_coef(int l_max, int m_max)
{
    int n = 0;
    for (int m = 0; m <= m_max; m++)
        for (int l = m; l <= l_max; l++) {
            n++;
            if (m != 0) n++;
        }
    return n;
}

/* Vertex directions of the Gaussian-image triangulation:
   period_search_BOINC.cpp:790-823.  t/f are 1-based, length ndir+1. */
static int vertex_dirs(int nrows, double *t, double *f)
{
    double dth = PSO_PI / (2 * nrows);
    int k = 1;
    t[1] = 0;
    f[1] = 0;
    for (int i = 1; i <= nrows; i++) {
        double dph = PSO_PI / (2 * i);
        for (int j = 0; j <= 4 * i - 1; j++) {
            k++;
            t[k] = i * dth;
            f[k] = j * dph;
        }
    }
    for (int i = nrows - 1; i >= 1; i--) {
        double dph = PSO_PI / (2 * i);
        for (int j = 0; j <= 4 * i - 1; j++) {
            k++;
            t[k] = PSO_PI - i * dth;
            f[k] = j * dph;
        }
    }
    int ndir = k + 1;
    t[ndir] = PSO_PI;
    f[ndir] = 0;
    return ndir;
}

/* Facet vertex triplets: trifac.c:11-83.  ifp[(i)*4 + 1..3], i = 1..nfac. */
static void triangulate(int nrows, int *ifp)
{
    int rows = 2 * nrows + 1, cols = 4 * nrows + 1;
    int *nod = (int *)calloc((size_t)rows * cols, sizeof(int));
#define NOD(i, j) nod[(i) * cols + (j)]
    int nnod = 1;
    NOD(0, 0) = nnod;
    for (int i = 1; i <= nrows; i++)
        for (int j = 0; j <= 4 * i - 1; j++) {
            nnod++;
            NOD(i, j) = nnod;
            if (j == 0) NOD(i, 4 * i) = nnod;
        }
    for (int i = nrows - 1; i >= 1; i--)
        for (int j = 0; j <= 4 * i - 1; j++) {
            nnod++;
            NOD(2 * nrows - i, j) = nnod;
            if (j == 0) NOD(2 * nrows - i, 4 * i) = nnod;
        }
    NOD(2 * nrows, 0) = nnod + 1;

    int ntri = 0;
#define TRI(a_, b_, c_) do { ntri++; ifp[ntri * 4 + 1] = (a_); ifp[ntri * 4 + 2] = (b_); ifp[ntri * 4 + 3] = (c_); } while (0)
    for (int j1 = 1; j1 <= nrows; j1++)
        for (int j3 = 1; j3 <= 4; j3++) {
            int j0 = (j3 - 1) * j1;
            TRI(NOD(j1 - 1, j0 - (j3 - 1)), NOD(j1, j0), NOD(j1, j0 + 1));
            for (int j2 = j0 + 1; j2 <= j0 + j1 - 1; j2++) {
                TRI(NOD(j1, j2), NOD(j1 - 1, j2 - (j3 - 1)), NOD(j1 - 1, j2 - 1 - (j3 - 1)));
                TRI(NOD(j1 - 1, j2 - (j3 - 1)), NOD(j1, j2), NOD(j1, j2 + 1));
            }
        }
    for (int j1 = nrows + 1; j1 <= 2 * nrows; j1++)
        for (int j3 = 1; j3 <= 4; j3++) {
            int j0 = (j3 - 1) * (2 * nrows - j1);
            TRI(NOD(j1, j0), NOD(j1 - 1, j0 + 1 + (j3 - 1)), NOD(j1 - 1, j0 + (j3 - 1)));
            for (int j2 = j0 + 1; j2 <= j0 + (2 * nrows - j1); j2++) {
                TRI(NOD(j1, j2), NOD(j1 - 1, j2 + (j3 - 1)), NOD(j1, j2 - 1));
                TRI(NOD(j1, j2), NOD(j1 - 1, j2 + 1 + (j3 - 1)), NOD(j1 - 1, j2 + (j3 - 1)));
            }
        }
#undef TRI
#undef NOD
    free(nod);
}

/* LU decomposition with implicit pivoting: ludcmp.c:10-96 (NR).  a is 1-based
   n x n stored as a[(i)*(n+1)+j]. */
static int lu_decompose(double *a, int n, int *indx)
{
    int N1 = n + 1, imax = -999;
    double *vv = (double *)malloc(sizeof(double) * (size_t)N1);
#define A(i, j) a[(i) * N1 + (j)]
    for (int i = 1; i <= n; i++) {
        double big = 0.0, temp;
        for (int j = 1; j <= n; j++)
            if ((temp = fabs(A(i, j))) > big) big = temp;
        if (big == 0.0) { free(vv); return 4; }
        vv[i] = 1.0 / big;
    }
    for (int j = 1; j <= n; j++) {
        for (int i = 1; i < j; i++) {
            double sum = A(i, j);
            for (int k = 1; k < i; k++) sum -= A(i, k) * A(k, j);
            A(i, j) = sum;
        }
        double big = 0.0, dum;
        for (int i = j; i <= n; i++) {
            double sum = A(i, j);
            for (int k = 1; k < j; k++) sum -= A(i, k) * A(k, j);
            A(i, j) = sum;
            if ((dum = vv[i] * fabs(sum)) >= big) {
                big = dum;
                imax = i;
            }
        }
        if (j != imax) {
            for (int k = 1; k <= n; k++) {
                dum = A(imax, k);
                A(imax, k) = A(j, k);
                A(j, k) = dum;
            }
            vv[imax] = vv[j];
        }
        indx[j] = imax;
        if (A(j, j) == 0.0) A(j, j) = 1.0e-20;
        if (j != n) {
            dum = 1.0 / (A(j, j));
            for (int i = j + 1; i <= n; i++) A(i, j) *= dum;
        }
    }
    free(vv);
    return 0;
}

/* Back substitution: lubksb.c:5-26 (NR). */
static void lu_solve(const double *a, int n, const int *indx, double *b)
{
    int N1 = n + 1, ii = 0;
    for (int i = 1; i <= n; i++) {
        int ip = indx[i];
        double sum = b[ip];
        b[ip] = b[i];
        if (ii)
            for (int j = ii; j <= i - 1; j++) sum -= A(i, j) * b[j];
        else if (sum)
            ii = i;
        b[i] = sum;
    }
    for (int i = n; i >= 1; i--) {
        double sum = b[i];
        for (int j = i + 1; j <= n; j++) sum -= A(i, j) * b[j];
        b[i] = sum / A(i, i);
    }
#undef A
}

/* Shape setup: triangulation (trifac.c), facet normals/areas (areanorm.c:11-61),
   unnormalised Laplace basis (sphfunc.c:12-88) and the ellipsoid
   log-curvature fit (ellfit.c:12-88), in the order of
   period_search_BOINC.cpp:831-837. */
int pso_setup_shape(int l_max, int m_max, int nrows, double ea, double eb, double ec,
                    double *normal, double *d_area, double *dsph, double *cg_first)
{
    if (l_max > MAX_LM || m_max > l_max || nrows < 1) return 1;
    int nfac = 8 * nrows * nrows;
    int ncoef = pso_n_coef(l_max, m_max);
    int maxdir = nfac + 8;
    double *t = (double *)calloc((size_t)maxdir, sizeof(double));
    double *f = (double *)calloc((size_t)maxdir, sizeof(double));
    int ndir = vertex_dirs(nrows, t, f);
    int *ifp = (int *)calloc((size_t)(nfac + 1) * 4, sizeof(int));
    triangulate(nrows, ifp);

    double *x = (double *)calloc((size_t)ndir + 1, sizeof(double));
    double *y = (double *)calloc((size_t)ndir + 1, sizeof(double));
    double *z = (double *)calloc((size_t)ndir + 1, sizeof(double));
    double *at = (double *)calloc((size_t)nfac + 1, sizeof(double));
    double *af = (double *)calloc((size_t)nfac + 1, sizeof(double));
    for (int i = 1; i <= ndir; i++) {
        double st = sin(t[i]);
        x[i] = st * cos(f[i]);
        y[i] = st * sin(f[i]);
        z[i] = cos(t[i]);
    }
    for (int i = 1; i <= nfac; i++) {
        double vx[4], vy[4], vz[4], c[4];
        for (int j = 2; j <= 3; j++) {
            vx[j] = x[ifp[i * 4 + j]] - x[ifp[i * 4 + 1]];
            vy[j] = y[ifp[i * 4 + j]] - y[ifp[i * 4 + 1]];
            vz[j] = z[ifp[i * 4 + j]] - z[ifp[i * 4 + 1]];
        }
        c[1] = vy[2] * vz[3] - vy[3] * vz[2];
        c[2] = vz[2] * vx[3] - vz[3] * vx[2];
        c[3] = vx[2] * vy[3] - vx[3] * vy[2];
        double clen2 = c[1] * c[1] + c[2] * c[2] + c[3] * c[3];
        double clen = sqrt(clen2);
        double n0 = c[1] / clen, n1 = c[2] / clen, n2 = c[3] / clen;
        normal[(i - 1) * 3 + 0] = n0;
        normal[(i - 1) * 3 + 1] = n1;
        normal[(i - 1) * 3 + 2] = n2;
        at[i] = acos(n2);
        af[i] = atan2(n1, n0);
        d_area[i - 1] = 0.5 * clen;
    }

    /* associated Legendre recursion coefficients (sphfunc.c:43-64) */
    static const int L1 = MAX_LM + 1;
    double *aleg = (double *)calloc((size_t)L1 * L1 * L1, sizeof(double));
#define ALEG(n, l, m) aleg[((n) * L1 + (l)) * L1 + (m)]
    ALEG(0, 0, 0) = 1;
    ALEG(1, 1, 0) = 1;
    for (int l = 1; l <= l_max; l++) ALEG(0, l, l) = ALEG(0, l - 1, l - 1) * (2 * l - 1);
    for (int m = 0; m <= m_max; m++)
        for (int l = m + 1; l <= l_max; l++) {
            int ibot;
            if ((2 * ((l - m) / 2)) == (l - m)) {
                ALEG(0, l, m) = -(l + m - 1) * ALEG(0, l - 2, m) / (1 * (l - m));
                ibot = 2;
            } else
                ibot = 1;
            if (l != 1)
                for (int n = ibot; n <= l - m; n = n + 2)
                    ALEG(n, l, m) = ((2 * l - 1) * ALEG(n - 1, l - 1, m) - (l + m - 1) * ALEG(n, l - 2, m)) / (1 * (l - m));
        }

    /* pleg[m][l][facet] (sphfunc.c:66-87), kept for ellfit */
    double *pleg = (double *)calloc((size_t)L1 * L1 * nfac, sizeof(double));
#define PLEG(m, l, i) pleg[(((size_t)(m)) * L1 + (l)) * nfac + (i)]
    for (int i = 1; i <= nfac; i++) {
        double ts[MAX_LM + 1], tc[MAX_LM + 1], fs[MAX_LM + 1], fc[MAX_LM + 1];
        ts[0] = 1;
        tc[0] = 1;
        ts[1] = sin(at[i]);
        tc[1] = cos(at[i]);
        for (int j = 2; j <= l_max; j++) {
            ts[j] = ts[1] * ts[j - 1];
            tc[j] = tc[1] * tc[j - 1];
        }
        fs[0] = 0;
        fc[0] = 1;
        for (int j = 1; j <= m_max; j++) {
            fs[j] = sin(j * af[i]);
            fc[j] = cos(j * af[i]);
        }
        int k = 0;
        for (int m = 0; m <= m_max; m++)
            for (int l = m; l <= l_max; l++) {
                double p = 0;
                int ibot = ((2 * ((l - m) / 2)) == (l - m)) ? 0 : 1;
                for (int n = ibot; n <= l - m; n = n + 2) p = p + ALEG(n, l, m) * tc[n] * ts[m];
                PLEG(m, l, i - 1) = p;
                k++;
                dsph[(size_t)(i - 1) * ncoef + (k - 1)] = fc[m] * p;
                if (m != 0) {
                    k++;
                    dsph[(size_t)(i - 1) * ncoef + (k - 1)] = fs[m] * p;
                }
            }
    }

    /* ellipsoid log-curvature fit (ellfit.c:12-88) */
    int N1 = ncoef + 1;
    double *er = (double *)calloc((size_t)nfac + 1, sizeof(double));
    double *fmat = (double *)calloc((size_t)(nfac + 1) * N1, sizeof(double));
    double *fitmat = (double *)calloc((size_t)N1 * N1, sizeof(double));
    double *fitvec = (double *)calloc((size_t)N1, sizeof(double));
    int *indx = (int *)calloc((size_t)N1, sizeof(int));
    for (int i = 1; i <= nfac; i++) {
        double st = sin(at[i]);
        double sum = pow(ea * st * cos(af[i]), 2) + pow(eb * st * sin(af[i]), 2) + pow(ec * cos(at[i]), 2);
        er[i] = 2 * (log(ea * eb * ec) - log(sum));
    }
    for (int i = 1; i <= nfac; i++) {
        int n = 0;
        for (int m = 0; m <= m_max; m++)
            for (int l = m; l <= l_max; l++) {
                n++;
                if (m != 0) {
                    fmat[i * N1 + n] = PLEG(m, l, i - 1) * cos(m * af[i]);
                    n++;
                    fmat[i * N1 + n] = PLEG(m, l, i - 1) * sin(m * af[i]);
                } else
                    fmat[i * N1 + n] = PLEG(m, l, i - 1);
            }
    }
    for (int i = 1; i <= ncoef; i++) {
        for (int j = 1; j <= ncoef; j++) {
            fitmat[i * N1 + j] = 0;
            for (int k = 1; k <= nfac; k++) fitmat[i * N1 + j] = fitmat[i * N1 + j] + fmat[k * N1 + i] * fmat[k * N1 + j];
        }
        fitvec[i] = 0;
        for (int j = 1; j <= nfac; j++) fitvec[i] = fitvec[i] + fmat[j * N1 + i] * er[j];
    }
    int rc = lu_decompose(fitmat, ncoef, indx);
    if (rc == 0) {
        lu_solve(fitmat, ncoef, indx, fitvec);
        for (int i = 1; i <= ncoef; i++) cg_first[i - 1] = fitvec[i];
    }
#undef PLEG
#undef ALEG
    free(er); free(fmat); free(fitmat); free(fitvec); free(indx);
    free(pleg); free(aleg);
    free(x); free(y); free(z); free(at); free(af);
    free(t); free(f); free(ifp);
    return rc;
}

/* ------------------------------------------------------------------------ */
/* One LM function evaluation (mrqcof)                                      */
/* ------------------------------------------------------------------------ */

typedef struct {
    double e[3], e0[3];
    double de[3][3], de0[3][3]; /* [q][xyz]: q = 0 beta', 1 lambda, 2 omega */
    double scale, ff, d2, alph;
} geo_t;

/* Rotation/phase geometry of one data point: curve1_point_geometry
   (Start.cu:2095-2195), blmatrix (Start.cu:399-417), ps_phase_mod2pi
   (Start.cu:687-692) and the exp-linear phase function.  Written with
   explicit matrices: T = Rz(phi) * B(beta', lambda). */
static void point_geometry(const pso_model *m, const double *a, int nc, int ip, geo_t *g)
{
    const double *ee = m->ee + 3 * ip, *ee0 = m->ee0 + 3 * ip;
    double t = m->tim[ip];
    double bet = a[nc + 1], lam = a[nc + 2], om = a[nc + 3];
    double A = a[nc + 4], rD = 1.0 / a[nc + 5], K = a[nc + 6];

    double cdot = ((ee[0] * ee0[0]) + ee[1] * ee0[1]) + ee[2] * ee0[2];
    double alph = acos(fmin(1.0, fmax(-1.0, cdot)));
    double ff = exp2(-1.44269504088896 * (alph * rD));
    g->alph = alph;
    g->ff = ff;
    g->scale = 1.0 + A * ff + K * alph;
    g->d2 = A * ff * alph * (rD * rD);

    double f = om * t + m->phi0;
    f = f - 2.0 * PSO_PI * round(f * (1.0 / (2.0 * PSO_PI)));
    double cf = cos(f), sf = sin(f);
    double cb = cos(bet), sb = sin(bet), cl = cos(lam), sl = sin(lam);

    double B[3][3] = {{cb * cl, cb * sl, -sb}, {-sl, cl, 0}, {sb * cl, sb * sl, cb}};
    double dBb[3][3] = {{-sb * cl, -sb * sl, -cb}, {0, 0, 0}, {cb * cl, cb * sl, -sb}};
    double dBl[3][3] = {{-cb * sl, cb * cl, 0}, {-cl, -sl, 0}, {-sb * sl, sb * cl, 0}};
    double R[3][3] = {{cf, sf, 0}, {-sf, cf, 0}, {0, 0, 1}};
    double dR[3][3] = {{-sf * t, cf * t, 0}, {-cf * t, -sf * t, 0}, {0, 0, 0}};
    double T[3][3], Tb[3][3], Tl[3][3], To[3][3];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            T[i][j] = R[i][0] * B[0][j] + R[i][1] * B[1][j] + R[i][2] * B[2][j];
            Tb[i][j] = R[i][0] * dBb[0][j] + R[i][1] * dBb[1][j] + R[i][2] * dBb[2][j];
            Tl[i][j] = R[i][0] * dBl[0][j] + R[i][1] * dBl[1][j] + R[i][2] * dBl[2][j];
            To[i][j] = dR[i][0] * B[0][j] + dR[i][1] * B[1][j] + dR[i][2] * B[2][j];
        }
    for (int i = 0; i < 3; i++) {
        g->e[i] = T[i][0] * ee[0] + T[i][1] * ee[1] + T[i][2] * ee[2];
        g->e0[i] = T[i][0] * ee0[0] + T[i][1] * ee0[1] + T[i][2] * ee0[2];
        g->de[0][i] = Tb[i][0] * ee[0] + Tb[i][1] * ee[1] + Tb[i][2] * ee[2];
        g->de0[0][i] = Tb[i][0] * ee0[0] + Tb[i][1] * ee0[1] + Tb[i][2] * ee0[2];
        g->de[1][i] = Tl[i][0] * ee[0] + Tl[i][1] * ee[1] + Tl[i][2] * ee[2];
        g->de0[1][i] = Tl[i][0] * ee0[0] + Tl[i][1] * ee0[1] + Tl[i][2] * ee0[2];
        g->de[2][i] = To[i][0] * ee[0] + To[i][1] * ee[1] + To[i][2] * ee[2];
        g->de0[2][i] = To[i][0] * ee0[0] + To[i][1] * ee0[1] + To[i][2] * ee0[2];
    }
}

/* curv: Areag[f] = Darea_f * exp(sum_k a_k Y_k(f)) (Start.cu:421-528). */
static double shape_areas(const pso_model *m, const double *a, double *area)
{
    int nf = m->n_fac, nc = m->n_coef;
    double tot = 0;
    for (int f = 0; f < nf; f++) {
        const double *y = m->dsph + (size_t)f * nc;
        double g = 0;
        for (int k = 0; k < nc; k++) g += a[k + 1] * y[k];
        area[f] = m->d_area[f] * exp(g);
        tot += area[f];
    }
    return tot;
}

/* Brightness and derivative row of one point: mrqcof_curve1_opt
   (Start.cu:2262-2535), one point at a time.  row[p-1] = d ymod / d a_p
   (un-renormalised); returns ymod = br * scale. */
#ifdef PSO_PERTURB
/* Perturbation study (test infrastructure, built only as
   _build/libps_oracle_perturb.so): every brightness term of an evaluation
   made during LM iteration < PSO_PERTURB_UNTIL is multiplied by
   1 + PSO_PERTURB_EPS * u, u uniform in [-1, 1] from a hash of (fit,
   iteration, point, term), to measure how much relative error the
   50-iteration fits tolerate before they end elsewhere. */
#include <stdint.h>
static __thread int g_iter = 0;
static __thread uint64_t g_fit = 0;
static double perturb_eps(void) { const char *e = getenv("PSO_PERTURB_EPS"); return e ? atof(e) : 0.0; }
static int perturb_until(void) { const char *e = getenv("PSO_PERTURB_UNTIL"); return e ? atoi(e) : 1000; }
static double perturb_u(uint64_t x)
{
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    x ^= x >> 31;
    return (double)(x >> 11) * (2.0 / 9007199254740992.0) - 1.0;
}
#endif

static double point_row(const pso_model *m, const double *a, const double *area, int ip,
                        double *row, double *dsh)
{
    int nf = m->n_fac, nc = m->n_coef, ma = nc + 8;
    geo_t g;
    point_geometry(m, a, nc, ip, &g);
    double cl = exp(a[ma - 1]), cls = a[ma];
    double br = 0, t1 = 0, t2 = 0, t3 = 0, t4 = 0, t5 = 0;
    for (int k = 0; k < nc; k++) dsh[k] = 0;
    for (int f = 0; f < nf; f++) {
        const double *n = m->normal + 3 * f;
        double mu = g.e[0] * n[0] + g.e[1] * n[1] + g.e[2] * n[2];
        double mu0 = g.e0[0] * n[0] + g.e0[1] * n[1] + g.e0[2] * n[2];
        if (mu > PSO_TINY && mu0 > PSO_TINY) {
            double ar = area[f];
            double dnom = mu + mu0;
            double r = 1.0 / dnom;
            double s = mu * mu0 * (cl + cls * r);
            double w = ar * s;
            br += w;
            double q0 = mu0 * r, q1 = mu * r;
            double dsmu = cls * (q0 * q0) + cl * mu0;
            double dsmu0 = cls * (q1 * q1) + cl * mu;
            double s1 = n[0] * g.de[0][0] + n[1] * g.de[0][1] + n[2] * g.de[0][2];
            double s10 = n[0] * g.de0[0][0] + n[1] * g.de0[0][1] + n[2] * g.de0[0][2];
            double s2 = n[0] * g.de[1][0] + n[1] * g.de[1][1] + n[2] * g.de[1][2];
            double s20 = n[0] * g.de0[1][0] + n[1] * g.de0[1][1] + n[2] * g.de0[1][2];
            double s3 = n[0] * g.de[2][0] + n[1] * g.de[2][1];
            double s30 = n[0] * g.de0[2][0] + n[1] * g.de0[2][1];
            t1 += ar * (dsmu * s1 + dsmu0 * s10);
            t2 += ar * (dsmu * s2 + dsmu0 * s20);
            t3 += ar * (dsmu * s3 + dsmu0 * s30);
            t4 += ar * mu * mu0;
            t5 += ar * mu * mu0 * r;
            const double *y = m->dsph + (size_t)f * nc;
            for (int k = 0; k < nc; k++) dsh[k] += w * y[k];
        }
    }
    double sc = g.scale;
#ifdef PSO_PERTURB
    double eps = perturb_eps();
    if (eps > 0 && g_iter < perturb_until()) {
        uint64_t base = (g_fit * 1000003ull + (uint64_t)g_iter) * 65537ull + (uint64_t)ip * 131ull;
        for (int k = 0; k < nc; k++) dsh[k] *= 1.0 + eps * perturb_u(base + k);
        br *= 1.0 + eps * perturb_u(base + 900);
        t1 *= 1.0 + eps * perturb_u(base + 901);
        t2 *= 1.0 + eps * perturb_u(base + 902);
        t3 *= 1.0 + eps * perturb_u(base + 903);
        t4 *= 1.0 + eps * perturb_u(base + 904);
        t5 *= 1.0 + eps * perturb_u(base + 905);
    }
#endif
    for (int k = 0; k < nc; k++) row[k] = sc * dsh[k];
    row[nc + 0] = sc * t1;
    row[nc + 1] = sc * t2;
    row[nc + 2] = sc * t3;
    row[nc + 3] = br * g.ff;
    row[nc + 4] = br * g.d2;
    row[nc + 5] = br * g.alph;
    row[nc + 6] = sc * t4 * cl;
    row[nc + 7] = sc * t5;
    return br * sc;
}

/* NR alpha/beta update for one data point with ia compaction
   (mrqcof_curve2_opt, Start.cu:2622-2828, in its NR-consistent form). */
static void accumulate(int mfit, const int *fidx, const double *dyda, double dy, double w,
                       double *alpha, double *beta)
{
    for (int j = 0; j < mfit; j++) {
        double wt = dyda[fidx[j] - 1] * w;
        double *arow = alpha + (size_t)j * mfit;
        for (int k = 0; k <= j; k++) arow[k] += wt * dyda[fidx[k] - 1];
        beta[j] += dy * wt;
    }
}

static int fit_index(const pso_model *m, int *fidx)
{
    int ma = m->n_coef + 8, mfit = 0;
    for (int p = 1; p <= ma; p++)
        if (m->ia[p]) fidx[mfit++] = p;
    return mfit;
}

double pso_eval(const pso_model *m, const double *a, double *alpha, double *beta,
                double *rows, double *area_sum)
{
    int nf = m->n_fac, nc = m->n_coef, ma = nc + 8;
    int fidx[PSO_MAX_PAR];
    int mfit = fit_index(m, fidx);
    double *area = (double *)malloc(sizeof(double) * (size_t)nf);
    double *dsh = (double *)malloc(sizeof(double) * (size_t)nc);
    int maxlp = 3;
    for (int c = 0; c < m->n_curves; c++)
        if (m->curve_len[c] > maxlp) maxlp = m->curve_len[c];
    double *crow = (double *)malloc(sizeof(double) * (size_t)maxlp * (ma + 1));
    double dave[PSO_MAX_PAR], dyda[PSO_MAX_PAR];

    double tot = shape_areas(m, a, area);
    if (area_sum) *area_sum = tot;
    memset(alpha, 0, sizeof(double) * (size_t)mfit * mfit);
    memset(beta, 0, sizeof(double) * (size_t)mfit);
    double chisq = 0;

    int ip0 = 0;
    for (int c = 0; c < m->n_curves; c++) {
        int lp = m->curve_len[c];
        double lave = 0;
        for (int j = 0; j < lp; j++) {
            double *r = crow + (size_t)j * (ma + 1);
            r[ma] = point_row(m, a, area, ip0 + j, r, dsh);
            lave += r[ma];
            if (rows) memcpy(rows + (size_t)(ip0 + j) * (ma + 1), r, sizeof(double) * (size_t)(ma + 1));
        }
        int rel = m->curve_rel[c];
        double rave = 0;
        if (rel) {
            /* per-curve column sums dave and 1/sum(ymod): Start.cu:2519-2533 */
            for (int k = 0; k < ma; k++) {
                double s = 0;
                for (int j = 0; j < lp; j++) s += crow[(size_t)j * (ma + 1) + k];
                dave[k] = s;
            }
            rave = 1.0 / lave;
        }
        for (int j = 0; j < lp; j++) {
            const double *r = crow + (size_t)j * (ma + 1);
            int ip = ip0 + j;
            double ymod;
            if (rel) {
                /* relative renormalisation: Start.cu:2660-2693 */
                double coef = m->sig[ip] * lp * rave;
                double coef1 = r[ma] * rave;
                for (int k = 0; k < ma; k++) dyda[k] = coef * (r[k] - coef1 * dave[k]);
                ymod = coef * r[ma];
            } else {
                for (int k = 0; k < ma; k++) dyda[k] = r[k];
                ymod = r[ma];
            }
            double w = m->sigr2[ip] * m->weight[ip];
            double dy = m->bright[ip] - ymod;
            chisq += dy * dy * w;
            accumulate(mfit, fidx, dyda, dy, w, alpha, beta);
        }
        ip0 += lp;
    }

    /* convexity regularisation pseudo-curve: mrqcof_curve1_last_opt
       (Start.cu:2539-2612), target 0, sigma 1/conw_r, weight 1 */
    for (int i = 0; i < 3; i++) {
        double ym = 0;
        for (int k = 0; k < ma; k++) dyda[k] = 0;
        for (int f = 0; f < nf; f++) {
            double w = area[f] * m->normal[3 * f + i];
            ym += w;
            const double *y = m->dsph + (size_t)f * nc;
            for (int k = 0; k < nc; k++) dyda[k] += w * y[k];
        }
        if (rows) {
            double *r = rows + (size_t)(m->n_points + i) * (ma + 1);
            memcpy(r, dyda, sizeof(double) * (size_t)ma);
            r[ma] = ym;
        }
        double w = m->conw_r * m->conw_r;
        double dy = 0 - ym;
        chisq += dy * dy * w;
        accumulate(mfit, fidx, dyda, dy, w, alpha, beta);
    }

    /* mirror the lower triangle: mrqcof_end (Start.cu:590-629) */
    for (int j = 1; j < mfit; j++)
        for (int k = 0; k < j; k++) alpha[(size_t)k * mfit + j] = alpha[(size_t)j * mfit + k];

    free(area);
    free(dsh);
    free(crow);
    return chisq;
}

/* ------------------------------------------------------------------------ */
/* LM step                                                                  */
/* ------------------------------------------------------------------------ */

/* Gauss-Jordan with full pivoting on [a | b] (gauss_errc; the live form is
   mrqmin_1_end_opt, Start.cu:2880-3006).  Pivot search: the last maximum in
   row-major order among rows/columns not yet pivoted.  The inverse is not
   needed by the caller, so already-pivoted columns are left untouched. */
int pso_gauss_solve(double *a, int n, double *b)
{
    int ipiv[PSO_MAX_PAR];
    for (int j = 0; j < n; j++) ipiv[j] = 0;
    for (int i = 0; i < n; i++) {
        double big = 0.0;
        int irow = 0, icol = 0;
        for (int j = 0; j < n; j++) {
            if (ipiv[j] == 1) continue;
            for (int k = 0; k < n; k++) {
                if (ipiv[k] == 0) {
                    double t = fabs(a[(size_t)j * n + k]);
                    if (t >= big) {
                        big = t;
                        irow = j;
                        icol = k;
                    }
                } else if (ipiv[k] > 1)
                    return 1;
            }
        }
        ipiv[icol] += 1;
        if (irow != icol) {
            for (int l = 0; l < n; l++) {
                double t = a[(size_t)irow * n + l];
                a[(size_t)irow * n + l] = a[(size_t)icol * n + l];
                a[(size_t)icol * n + l] = t;
            }
            double t = b[irow];
            b[irow] = b[icol];
            b[icol] = t;
        }
        double piv = a[(size_t)icol * n + icol];
        if (piv == 0.0) return 2;
        double pivinv = 1.0 / piv;
        a[(size_t)icol * n + icol] = 1.0;
        for (int l = 0; l < n; l++) a[(size_t)icol * n + l] *= pivinv;
        b[icol] *= pivinv;
        for (int ll = 0; ll < n; ll++) {
            if (ll == icol) continue;
            double dum = a[(size_t)ll * n + icol];
            for (int l = 0; l < n; l++) {
                double base = (l == icol) ? 0.0 : a[(size_t)ll * n + l];
                a[(size_t)ll * n + l] = base - a[(size_t)icol * n + l] * dum;
            }
            b[ll] -= b[icol] * dum;
        }
    }
    return 0;
}

/* Initial parameters of one (frequency, pole) item: CudaCalculatePreparePole
   (Start.cu:4346-4418). */
static void initial_params(const pso_model *m, double freq_start, double freq_step, int n,
                           int pole, double *a)
{
    int nc = m->n_coef, ma = nc + 8;
    for (int k = 1; k <= nc; k++) a[k] = m->cg_first[k - 1];
    double period = 1.0 / (freq_start - (n - 1) * freq_step);
    a[nc + 1] = DEG2RAD * 90 - DEG2RAD * m->beta_pole[pole];
    a[nc + 2] = DEG2RAD * m->lambda_pole[pole];
    a[nc + 3] = (24.0 * 2.0 * PSO_PI) / period;
    a[nc + 4] = m->par[0];
    a[nc + 5] = m->par[1];
    a[nc + 6] = m->par[2];
    a[ma - 1] = m->lcl;
    a[ma] = 1;
}

/* The LM loop of one fit: CudaCalculateIter1Begin (Start.cu:4421-4462),
   mrqmin_1_end_opt, the two mrqcof evaluations, mrqmin_2_end
   (Start.cu:300-392), CudaCalculateIter2 (Start.cu:5129-5248) and
   CudaCalculateFinishPole (Start.cu:5056-5125). */
void pso_fit(const pso_model *m, double freq_start, double freq_step, int n_freq,
             int pole, pso_fit_result *res)
{
    int nf = m->n_fac, nc = m->n_coef, ma = nc + 8;
    int fidx[PSO_MAX_PAR];
    int mfit = fit_index(m, fidx);
    size_t msz = (size_t)mfit * mfit;
    double *alpha = (double *)calloc(msz, sizeof(double));
    double *covar = (double *)calloc(msz, sizeof(double));
    double *beta = (double *)calloc((size_t)mfit, sizeof(double));
    double *da = (double *)calloc((size_t)mfit, sizeof(double));
    double *area = (double *)malloc(sizeof(double) * (size_t)nf);
    double a[PSO_MAX_PAR + 1], atry[PSO_MAX_PAR + 1];
    memset(atry, 0, sizeof(atry));
    initial_params(m, freq_start, freq_step, n_freq, pole, a);
#ifdef PSO_PERTURB
    g_fit = (uint64_t)n_freq * 16 + (uint64_t)pole;
#endif

    double alamda = -1, chisq = 0, ochisq = 0;
    int niter = 0, status = 0;
    double iter_diff = 1e40, dev_old = 1e30, dev_new = 0, chck = 0, area_last = 0;
    int ndata = m->n_points + 3;

    for (;;) {
        int go = ((niter < m->n_iter_max) && (iter_diff > m->iter_diff_max)) || (niter < m->n_iter_min);
        if (!go) break;
#ifdef PSO_PERTURB
        g_iter = niter;
#endif
        int first = 0;
        if (alamda < 0) {
            alamda = m->alamda_start;
            first = 1;
        }
        if (first) {
            ochisq = pso_eval(m, a, alpha, beta, NULL, &area_last);
            for (int l = 1; l <= ma; l++) atry[l] = a[l];
        }
        /* damped normal matrix and solve */
        double ccc = 1 + alamda;
        for (int j = 0; j < mfit; j++) {
            for (int k = 0; k < mfit; k++) covar[(size_t)j * mfit + k] = alpha[(size_t)j * mfit + k];
            covar[(size_t)j * mfit + j] = alpha[(size_t)j * mfit + j] * ccc;
            da[j] = beta[j];
        }
        int err = pso_gauss_solve(covar, mfit, da);
        if (err == 0 || err == 2) {
            if (err == 2) status |= 1;
            for (int j = 0; j < mfit; j++) atry[fidx[j]] = a[fidx[j]] + da[j];
        }
        chisq = pso_eval(m, atry, covar, da, NULL, &area_last);
        if (isnan(chisq)) status |= 2;
        if (chisq < ochisq) {
            memcpy(beta, da, sizeof(double) * (size_t)mfit);
            alamda *= m->alamda_incrr;
            memcpy(alpha, covar, sizeof(double) * msz);
            for (int l = 1; l <= ma; l++) a[l] = atry[l];
        } else {
            alamda = m->alamda_incr * alamda;
            chisq = ochisq;
        }
        niter++;
        if (niter == 1 || chisq < ochisq) {
            ochisq = chisq;
            area_last = shape_areas(m, a, area);
            double r0 = 0, r1 = 0, r2 = 0;
            for (int f = 0; f < nf; f++) {
                r0 += area[f] * m->normal[3 * f + 0];
                r1 += area[f] * m->normal[3 * f + 1];
                r2 += area[f] * m->normal[3 * f + 2];
            }
            double aa = r0 * r0 + r1 * r1 + r2 * r2;
            double rchisq = chisq - aa * (m->conw_r_dev * m->conw_r_dev);
            dev_new = sqrt(rchisq / (ndata - 3));
            chck = sqrt(aa);
            double diff = dev_old - dev_new;
            if (diff > 1e-10) {
                iter_diff = diff;
                dev_old = dev_new;
            }
        }
    }

    double dd = chck * 100.0 * (1.0 / area_last);
    if (isnan(dd)) dd = 1.0;
    double la = RAD2DEG * a[nc + 2];
    res->dev = dev_new;
    res->dark = dd;
    res->per = 2 * PSO_PI / a[nc + 3];
    res->lambda_deg = la + (la < 0 ? 360 : 0);
    res->beta_deg = 90 - RAD2DEG * a[nc + 1];
    res->chisq = chisq;
    res->niter = niter;
    res->status = status;
    free(alpha); free(covar); free(beta); free(da); free(area);
}

/* ------------------------------------------------------------------------ */
/* Threaded batches                                                         */
/* ------------------------------------------------------------------------ */

typedef struct {
    const pso_model *m;
    double fs, fstep;
    const int *n_freq, *pole;
    int n;
    pso_fit_result *res;
    int next;
    pthread_mutex_t mu;
} batch_t;

static void *batch_worker(void *p)
{
    batch_t *b = (batch_t *)p;
    for (;;) {
        pthread_mutex_lock(&b->mu);
        int i = b->next++;
        pthread_mutex_unlock(&b->mu);
        if (i >= b->n) break;
        pso_fit(b->m, b->fs, b->fstep, b->n_freq[i], b->pole[i], &b->res[i]);
    }
    return NULL;
}

void pso_fit_batch(const pso_model *m, double freq_start, double freq_step,
                   const int *n_freq, const int *pole, int n, pso_fit_result *res,
                   int n_threads)
{
    batch_t b;
    b.m = m;
    b.fs = freq_start;
    b.fstep = freq_step;
    b.n_freq = n_freq;
    b.pole = pole;
    b.n = n;
    b.res = res;
    b.next = 0;
    pthread_mutex_init(&b.mu, NULL);
    if (n_threads < 1) n_threads = 1;
    if (n_threads > 256) n_threads = 256;
    pthread_t th[256];
    for (int i = 0; i < n_threads; i++) pthread_create(&th[i], NULL, batch_worker, &b);
    for (int i = 0; i < n_threads; i++) pthread_join(th[i], NULL);
    pthread_mutex_destroy(&b.mu);
}

/* Best pole of one frequency: NaN-safe, the earliest pole wins ties
   (start_CUDA.cu:1200-1229). */
static int best_pole(const pso_fit_result *r)
{
    int best = -1;
    for (int p = 0; p < PSO_N_POLES; p++)
        if (best < 0 || (!isnan(r[p].dev) && !(r[p].dev >= r[best].dev))) best = p;
    return best;
}

void pso_precalc(pso_model *m, double freq_start, double freq_step,
                 double *conw_r, int *new_conw, int quirks, int n_threads)
{
    const int max_test_periods = 10; /* start_CUDA.cu:420 */
    int n = max_test_periods * PSO_N_POLES;
    int nf[100], pl[100];
    pso_fit_result res[100];
    for (int i = 0; i < n; i++) {
        nf[i] = 1 + i / PSO_N_POLES;
        pl[i] = i % PSO_N_POLES;
    }
    m->conw_r = *conw_r;
    m->conw_r_dev = (quirks & PSO_QUIRK_PRECALC_CONW) ? 0.0 : *conw_r;
    pso_fit_batch(m, freq_start, freq_step, nf, pl, n, res, n_threads);
    double sum_dark = 0;
    for (int t = 0; t < max_test_periods; t++) {
        int b = best_pole(res + t * PSO_N_POLES);
        sum_dark = sum_dark + res[t * PSO_N_POLES + b].dark;
    }
    double ave = sum_dark / max_test_periods;
    if (ave < 1.0) *new_conw = 1;
    if (ave >= 1.0) *conw_r = *conw_r * 2;
}

int pso_scan(const pso_model *m, double freq_start, double freq_end, double freq_step,
             int n_start, pso_line *lines, int max_lines, int n_threads)
{
    int n_max = (int)((freq_start - freq_end) / freq_step) + 1;
    int nfreq = n_max - n_start + 1;
    if (nfreq > max_lines) nfreq = max_lines;
    if (nfreq <= 0) return 0;
    int n = nfreq * PSO_N_POLES;
    int *nf = (int *)malloc(sizeof(int) * (size_t)n);
    int *pl = (int *)malloc(sizeof(int) * (size_t)n);
    pso_fit_result *res = (pso_fit_result *)malloc(sizeof(pso_fit_result) * (size_t)n);
    for (int i = 0; i < n; i++) {
        nf[i] = n_start + i / PSO_N_POLES;
        pl[i] = i % PSO_N_POLES;
    }
    pso_fit_batch(m, freq_start, freq_step, nf, pl, n, res, n_threads);
    for (int q = 0; q < nfreq; q++) {
        const pso_fit_result *r = res + q * PSO_N_POLES;
        int b = best_pole(r);
        lines[q].period_h = 24 * r[b].per;
        lines[q].rms = r[b].dev;
        lines[q].chisq = r[b].dev * r[b].dev * m->n_points;
        lines[q].dark = r[b].dark;
        lines[q].lambda_deg = r[b].lambda_deg;
        lines[q].beta_deg = r[b].beta_deg;
        lines[q].valid = 1;
    }
    free(nf); free(pl); free(res);
    return nfreq;
}

/* ------------------------------------------------------------------------ */
/* Whole application: period_search_BOINC.cpp:171-907 without BOINC          */
/* ------------------------------------------------------------------------ */

static int skip_line(FILE *f)
{
    int c;
    while ((c = fgetc(f)) != EOF && c != '\n') {}
    return c;
}

int pso_run_file(const char *in_path, const char *out_path, int quirks, int n_threads,
                 int max_freq)
{
    FILE *in = fopen(in_path, "r");
    if (!in) return 10;
    double p_start, p_coef, p_end, jd00, phi0, conw, par[3], cl, stop, lincr, lstart;
    int ia_prd, lmax, mmax, nrows, ia_par[3], ia_cl, n_iter_min, n_curves;
    int ok = 1;
    ok &= fscanf(in, "%lf %lf %lf %d", &p_start, &p_coef, &p_end, &ia_prd) == 4; skip_line(in);
    ok &= fscanf(in, "%lf", &jd00) == 1; skip_line(in);
    ok &= fscanf(in, "%lf", &phi0) == 1; skip_line(in);
    ok &= fscanf(in, "%lf", &conw) == 1; skip_line(in);
    ok &= fscanf(in, "%d %d", &lmax, &mmax) == 2; skip_line(in);
    ok &= fscanf(in, "%d", &nrows) == 1; skip_line(in);
    for (int i = 0; i < 3; i++) { ok &= fscanf(in, "%lf %d", &par[i], &ia_par[i]) == 2; skip_line(in); }
    ok &= fscanf(in, "%lf %d", &cl, &ia_cl) == 2; skip_line(in);
    ok &= fscanf(in, "%lf", &stop) == 1; skip_line(in);
    ok &= fscanf(in, "%d", &n_iter_min) == 1; skip_line(in);
    ok &= fscanf(in, "%lf", &lincr) == 1; skip_line(in);
    ok &= fscanf(in, "%lf", &lstart) == 1; skip_line(in);
    ok &= fscanf(in, "%d", &n_curves) == 1;
    if (!ok || n_curves <= 0) { fclose(in); return 11; }

    int cap = 1024, np = 0;
    int *clen = (int *)calloc((size_t)n_curves, sizeof(int));
    int *crel = (int *)calloc((size_t)n_curves, sizeof(int));
    double *tim = (double *)malloc(sizeof(double) * cap);
    double *br = (double *)malloc(sizeof(double) * cap);
    double *ee = (double *)malloc(sizeof(double) * cap * 3);
    double *ee0 = (double *)malloc(sizeof(double) * cap * 3);
    double *sig = (double *)malloc(sizeof(double) * cap);
    double *sigr2 = (double *)malloc(sizeof(double) * cap);
    double *al = (double *)calloc((size_t)n_curves, sizeof(double));
    double jd_min = 1e20, jd_max = -1e40, al0 = PSO_PI, al0_abs = PSO_PI;
    int ial0 = -1, ial0_abs = -1, onlyrel = 1;
    for (int i = 0; i < n_curves; i++) {
        int itemp;
        ok &= fscanf(in, "%d %d", &clen[i], &itemp) == 2;
        skip_line(in);
        crel[i] = 1 - itemp;
        if (crel[i] == 0) onlyrel = 0;
        double ave = 0;
        for (int j = 0; j < clen[i]; j++) {
            if (np + 1 >= cap) {
                cap *= 2;
                tim = (double *)realloc(tim, sizeof(double) * cap);
                br = (double *)realloc(br, sizeof(double) * cap);
                ee = (double *)realloc(ee, sizeof(double) * cap * 3);
                ee0 = (double *)realloc(ee0, sizeof(double) * cap * 3);
                sig = (double *)realloc(sig, sizeof(double) * cap);
                sigr2 = (double *)realloc(sigr2, sizeof(double) * cap);
            }
            double e0[3], e[3];
            ok &= fscanf(in, "%lf %lf", &tim[np], &br[np]) == 2;
            ok &= fscanf(in, "%lf %lf %lf", &e0[0], &e0[1], &e0[2]) == 3;
            ok &= fscanf(in, "%lf %lf %lf", &e[0], &e[1], &e[2]) == 3;
            if (tim[np] < jd_min) jd_min = tim[np];
            if (tim[np] > jd_max) jd_max = tim[np];
            double e0len = sqrt(e0[0] * e0[0] + e0[1] * e0[1] + e0[2] * e0[2]);
            double elen = sqrt(e[0] * e[0] + e[1] * e[1] + e[2] * e[2]);
            ave += br[np];
            for (int k = 0; k < 3; k++) {
                ee[np * 3 + k] = e[k] / elen;
                ee0[np * 3 + k] = e0[k] / e0len;
            }
            if (j == 0) {
                double cosa = (e[0] * e0[0] + e[1] * e0[1] + e[2] * e0[2]) / (elen * e0len);
                al[i] = acos(cosa);
                if (al[i] < al0) { al0 = al[i]; ial0 = np; }
                if (al[i] < al0_abs && crel[i] == 0) { al0_abs = al[i]; ial0_abs = np; }
            }
            np++;
        }
        ave /= clen[i];
        for (int j = np - clen[i]; j < np; j++) {
            sig[j] = ave;
            sigr2[j] = 1.0 / (ave * ave);
        }
    }
    if (!ok) { fclose(in); return 12; }
    /* trailing "curve# weight" pairs (period_search_BOINC.cpp:524-533) */
    double *wlc = (double *)malloc(sizeof(double) * (size_t)n_curves);
    for (int i = 0; i < n_curves; i++) wlc[i] = -1;
    for (;;) {
        int lc;
        double wv;
        if (fscanf(in, "%d", &lc) != 1) break;
        if (fscanf(in, "%lf", &wv) != 1) break;
        if (lc >= 1 && lc <= n_curves) wlc[lc - 1] = wv;
    }
    fclose(in);
    double *weight = (double *)malloc(sizeof(double) * (size_t)np);
    {
        int k = 0;
        for (int i = 0; i < n_curves; i++)
            for (int j = 0; j < clen[i]; j++) weight[k++] = (wlc[i] == -1) ? 1 : wlc[i];
    }
    double jd0 = jd00;
    if (jd0 <= 0) jd0 = (int)jd_min;
    for (int i = 0; i < np; i++) tim[i] = tim[i] - jd0;

    if (onlyrel == 0) { al0 = al0_abs; ial0 = ial0_abs; }
    double ea = 1.05, eb = 1.00, ec = 0.95;
    double rfit = sqrt(2 * sig[ial0] / (0.5 * PSO_PI * (1 + cos(al0))));
    double escl = rfit / sqrt((ea * eb + eb * ec + ea * ec) / 3);
    if (onlyrel == 0) escl *= 0.8;
    ea *= escl; eb *= escl; ec *= escl;

    int nfac = 8 * nrows * nrows, ncoef = pso_n_coef(lmax, mmax);
    double *normal = (double *)malloc(sizeof(double) * (size_t)nfac * 3);
    double *darea = (double *)malloc(sizeof(double) * (size_t)nfac);
    double *dsph = (double *)malloc(sizeof(double) * (size_t)nfac * ncoef);
    double *cgf = (double *)malloc(sizeof(double) * (size_t)ncoef);
    int rc = pso_setup_shape(lmax, mmax, nrows, ea, eb, ec, normal, darea, dsph, cgf);
    if (rc) return 13;

    pso_model m;
    memset(&m, 0, sizeof(m));
    m.n_points = np;
    m.n_curves = n_curves;
    m.curve_len = clen;
    m.curve_rel = crel;
    m.tim = tim;
    m.ee = ee;
    m.ee0 = ee0;
    m.bright = br;
    m.sig = sig;
    m.sigr2 = sigr2;
    m.weight = weight;
    m.n_fac = nfac;
    m.n_coef = ncoef;
    m.normal = normal;
    m.d_area = darea;
    m.dsph = dsph;
    m.cg_first = cgf;
    m.phi0 = phi0 * DEG2RAD;
    for (int i = 0; i < 3; i++) m.par[i] = par[i];
    m.lcl = log(cl);
    m.alamda_start = lstart;
    m.alamda_incr = lincr;
    m.alamda_incrr = (lincr != 0.0) ? 1.0 / lincr : 1.79769313486231570815e+308;
    static const double lp[10] = {0, 90, 180, 270, 60, 180, 300, 60, 180, 300};
    static const double bp[10] = {0, 0, 0, 0, 60, 60, 60, -60, -60, -60};
    for (int i = 0; i < 10; i++) { m.lambda_pole[i] = lp[i]; m.beta_pole[i] = bp[i]; }
    int ma = ncoef + 8;
    for (int i = 1; i <= ncoef; i++) m.ia[i] = 1;
    if (onlyrel) m.ia[1] = 0;
    m.ia[ncoef + 1] = 1;
    m.ia[ncoef + 2] = 1;
    m.ia[ncoef + 3] = ia_prd;
    for (int i = 0; i < 3; i++) m.ia[ncoef + 4 + i] = ia_par[i];
    m.ia[ma - 1] = ia_cl;
    m.ia[ma] = 0;
    if (stop > 1) {
        m.n_iter_max = (int)stop;
        m.iter_diff_max = 0;
        m.n_iter_min = 0;
    } else {
        m.n_iter_max = (stop < 1) ? PSO_MAX_N_ITER : 0;
        m.iter_diff_max = (stop < 1) ? stop : -1;
        m.n_iter_min = n_iter_min;
    }

    double f_start = 1 / p_start, f_end = 1 / p_end;
    double f_step = 0.5 / (jd_max - jd_min) / 24 * p_coef;

    double conw_r = conw / escl / escl;
    int new_conw = 0;
    while ((new_conw != 1) && ((conw_r * escl * escl) < 10.0))
        pso_precalc(&m, f_start, f_step, &conw_r, &new_conw, quirks, n_threads);
    m.conw_r = conw_r;
    m.conw_r_dev = conw_r;

    int n_max = (int)((f_start - f_end) / f_step) + 1;
    if (max_freq > 0 && n_max > max_freq) n_max = max_freq;
    pso_line *lines = (pso_line *)calloc((size_t)n_max + 1, sizeof(pso_line));
    int nl = pso_scan(&m, f_start, f_end, f_step, 1, lines, n_max, n_threads);
    FILE *out = fopen(out_path, "w");
    if (!out) return 14;
    for (int q = 0; q < nl; q++) {
        double dark = (q == 0) ? conw_r * escl * escl : lines[q].dark;
        fprintf(out, "%.8f  %.6f  %.6f %4.1f %4.0f %4.0f\n", lines[q].period_h, lines[q].rms,
                lines[q].chisq, dark, round(lines[q].lambda_deg), round(lines[q].beta_deg));
    }
    fclose(out);
    free(lines);
    free(normal); free(darea); free(dsph); free(cgf);
    free(clen); free(crel); free(tim); free(br); free(ee); free(ee0);
    free(sig); free(sigr2); free(al); free(wlc); free(weight);
    return 0;
}
