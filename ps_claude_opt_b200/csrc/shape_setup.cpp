// shape_setup.cpp -- host-side Gaussian-image setup of the product.
//
// Triangulated unit sphere (trifac.c:11-83), facet normals and areas
// (areanorm.c:11-61), the unnormalised Laplace-series basis (sphfunc.c:12-88)
// and the least-squares ellipsoid log-curvature fit of the initial shape
// (ellfit.c:12-88 with NR ludcmp.c / lubksb.c).  The floating-point operations
// run in the reference's order so the tables are bit-identical to it.
#include <cmath>
#include <vector>

#include "ps_b200.h"
#include "util.h"

namespace {

constexpr double kPi = 3.14159265358979323846;
constexpr int kMaxLm = 15;

// Vertex directions (theta, phi), 1-based: period_search_BOINC.cpp:790-823.
int vertex_directions(int nrows, std::vector<double> &t, std::vector<double> &f)
{
    const int nv = 4 * nrows * nrows + 2;
    t.assign(nv + 2, 0.0);
    f.assign(nv + 2, 0.0);
    const double dth = kPi / (2 * nrows);
    int k = 1;
    for (int i = 1; i <= nrows; ++i) {
        const double dph = kPi / (2 * i);
        for (int j = 0; j < 4 * i; ++j) {
            ++k;
            t[k] = i * dth;
            f[k] = j * dph;
        }
    }
    for (int i = nrows - 1; i >= 1; --i) {
        const double dph = kPi / (2 * i);
        for (int j = 0; j < 4 * i; ++j) {
            ++k;
            t[k] = kPi - i * dth;
            f[k] = j * dph;
        }
    }
    t[k + 1] = kPi;
    f[k + 1] = 0;
    return k + 1;
}

// Triangle vertex indices (1-based vertices) per facet, rows of latitude bands
// from the north pole: trifac.c.
std::vector<int> facet_vertices(int nrows)
{
    const int cols = 4 * nrows + 1;
    std::vector<int> node((2 * nrows + 1) * cols, 0);
    auto nod = [&](int i, int j) -> int & { return node[i * cols + j]; };
    int next = 1;
    nod(0, 0) = next;
    for (int i = 1; i <= nrows; ++i)
        for (int j = 0; j < 4 * i; ++j) {
            nod(i, j) = ++next;
            if (j == 0) nod(i, 4 * i) = next;
        }
    for (int i = nrows - 1; i >= 1; --i)
        for (int j = 0; j < 4 * i; ++j) {
            nod(2 * nrows - i, j) = ++next;
            if (j == 0) nod(2 * nrows - i, 4 * i) = next;
        }
    nod(2 * nrows, 0) = next + 1;

    std::vector<int> tri;
    tri.reserve(8 * nrows * nrows * 3);
    auto add = [&](int a, int b, int c) {
        tri.push_back(a);
        tri.push_back(b);
        tri.push_back(c);
    };
    for (int r = 1; r <= nrows; ++r)
        for (int q = 0; q < 4; ++q) {
            const int j0 = q * r;
            add(nod(r - 1, j0 - q), nod(r, j0), nod(r, j0 + 1));
            for (int j = j0 + 1; j <= j0 + r - 1; ++j) {
                add(nod(r, j), nod(r - 1, j - q), nod(r - 1, j - 1 - q));
                add(nod(r - 1, j - q), nod(r, j), nod(r, j + 1));
            }
        }
    for (int r = nrows + 1; r <= 2 * nrows; ++r)
        for (int q = 0; q < 4; ++q) {
            const int w = 2 * nrows - r;
            const int j0 = q * w;
            add(nod(r, j0), nod(r - 1, j0 + 1 + q), nod(r - 1, j0 + q));
            for (int j = j0 + 1; j <= j0 + w; ++j) {
                add(nod(r, j), nod(r - 1, j + q), nod(r, j - 1));
                add(nod(r, j), nod(r - 1, j + 1 + q), nod(r - 1, j + q));
            }
        }
    return tri;
}

// NR LU decomposition with implicit scaling and its back substitution
// (ludcmp.c, lubksb.c), 1-based square matrix in a flat vector.
bool lu_solve(std::vector<double> &a, int n, std::vector<double> &b)
{
    const int n1 = n + 1;
    auto A = [&](int i, int j) -> double & { return a[i * n1 + j]; };
    std::vector<double> scale(n1);
    std::vector<int> perm(n1);
    for (int i = 1; i <= n; ++i) {
        double big = 0.0, v;
        for (int j = 1; j <= n; ++j)
            if ((v = std::fabs(A(i, j))) > big) big = v;
        if (big == 0.0) return false;
        scale[i] = 1.0 / big;
    }
    int imax = -1;
    for (int j = 1; j <= n; ++j) {
        for (int i = 1; i < j; ++i) {
            double sum = A(i, j);
            for (int k = 1; k < i; ++k) sum -= A(i, k) * A(k, j);
            A(i, j) = sum;
        }
        double big = 0.0, dum;
        for (int i = j; i <= n; ++i) {
            double sum = A(i, j);
            for (int k = 1; k < j; ++k) sum -= A(i, k) * A(k, j);
            A(i, j) = sum;
            if ((dum = scale[i] * std::fabs(sum)) >= big) {
                big = dum;
                imax = i;
            }
        }
        if (j != imax) {
            for (int k = 1; k <= n; ++k) std::swap(A(imax, k), A(j, k));
            scale[imax] = scale[j];
        }
        perm[j] = imax;
        if (A(j, j) == 0.0) A(j, j) = 1.0e-20;
        if (j != n) {
            dum = 1.0 / (A(j, j));
            for (int i = j + 1; i <= n; ++i) A(i, j) *= dum;
        }
    }
    int first = 0;
    for (int i = 1; i <= n; ++i) {
        const int ip = perm[i];
        double sum = b[ip];
        b[ip] = b[i];
        if (first)
            for (int j = first; j <= i - 1; ++j) sum -= A(i, j) * b[j];
        else if (sum)
            first = i;
        b[i] = sum;
    }
    for (int i = n; i >= 1; --i) {
        double sum = b[i];
        for (int j = i + 1; j <= n; ++j) sum -= A(i, j) * b[j];
        b[i] = sum / A(i, i);
    }
    return true;
}

}  // namespace

extern "C" int32_t ps_n_coef(int32_t l_max, int32_t m_max)
{
    int n = 0;
    for (int m = 0; m <= m_max; ++m)
        for (int l = m; l <= l_max; ++l) n += (m != 0) ? 2 : 1;
    return n;
}

extern "C" ps_status ps_setup_shape(int32_t l_max, int32_t m_max, int32_t nrows, double ea, double eb,
                                    double ec, double *normal, double *d_area, double *d_sphere,
                                    double *cg_first)
{
    if (l_max < 0 || l_max > kMaxLm || m_max < 0 || m_max > l_max || nrows < 1 ||
        8 * nrows * nrows > PS_MAX_FAC || !normal || !d_area || !d_sphere || !cg_first)
        return psb_fail(PS_ERR_ARG, "ps_setup_shape: invalid arguments");
    const int nfac = 8 * nrows * nrows;
    const int nc = ps_n_coef(l_max, m_max);
    std::vector<double> t, f;
    const int ndir = vertex_directions(nrows, t, f);
    const std::vector<int> tri = facet_vertices(nrows);

    std::vector<double> x(ndir + 1), y(ndir + 1), z(ndir + 1);
    for (int i = 1; i <= ndir; ++i) {
        const double st = std::sin(t[i]);
        x[i] = st * std::cos(f[i]);
        y[i] = st * std::sin(f[i]);
        z[i] = std::cos(t[i]);
    }
    std::vector<double> at(nfac), af(nfac);
    for (int i = 0; i < nfac; ++i) {
        const int v1 = tri[3 * i], v2 = tri[3 * i + 1], v3 = tri[3 * i + 2];
        const double ax = x[v2] - x[v1], ay = y[v2] - y[v1], az = z[v2] - z[v1];
        const double bx = x[v3] - x[v1], by = y[v3] - y[v1], bz = z[v3] - z[v1];
        const double c1 = ay * bz - by * az;
        const double c2 = az * bx - bz * ax;
        const double c3 = ax * by - bx * ay;
        const double clen = std::sqrt(c1 * c1 + c2 * c2 + c3 * c3);
        normal[3 * i + 0] = c1 / clen;
        normal[3 * i + 1] = c2 / clen;
        normal[3 * i + 2] = c3 / clen;
        at[i] = std::acos(normal[3 * i + 2]);
        af[i] = std::atan2(normal[3 * i + 1], normal[3 * i + 0]);
        d_area[i] = 0.5 * clen;
    }

    // recursion coefficients of the unnormalised associated Legendre functions
    // written as polynomials in cos(theta) times sin^m(theta)
    const int L = kMaxLm + 1;
    std::vector<double> coef(L * L * L, 0.0);
    auto C = [&](int n, int l, int m) -> double & { return coef[(n * L + l) * L + m]; };
    C(0, 0, 0) = 1;
    C(1, 1, 0) = 1;
    for (int l = 1; l <= l_max; ++l) C(0, l, l) = C(0, l - 1, l - 1) * (2 * l - 1);
    for (int m = 0; m <= m_max; ++m)
        for (int l = m + 1; l <= l_max; ++l) {
            int nlow = 1;
            if (((l - m) & 1) == 0) {
                C(0, l, m) = -(l + m - 1) * C(0, l - 2, m) / (1 * (l - m));
                nlow = 2;
            }
            if (l != 1)
                for (int n = nlow; n <= l - m; n += 2)
                    C(n, l, m) = ((2 * l - 1) * C(n - 1, l - 1, m) - (l + m - 1) * C(n, l - 2, m)) / (1 * (l - m));
        }

    // basis values and the Legendre table the ellipsoid fit reuses
    std::vector<double> leg((size_t)L * L * nfac, 0.0);
    auto P = [&](int m, int l, int i) -> double & { return leg[((size_t)m * L + l) * nfac + i]; };
    for (int i = 0; i < nfac; ++i) {
        double ts[kMaxLm + 1], tc[kMaxLm + 1], fs[kMaxLm + 1], fc[kMaxLm + 1];
        ts[0] = 1;
        tc[0] = 1;
        ts[1] = std::sin(at[i]);
        tc[1] = std::cos(at[i]);
        for (int j = 2; j <= l_max; ++j) {
            ts[j] = ts[1] * ts[j - 1];
            tc[j] = tc[1] * tc[j - 1];
        }
        fs[0] = 0;
        fc[0] = 1;
        for (int j = 1; j <= m_max; ++j) {
            fs[j] = std::sin(j * af[i]);
            fc[j] = std::cos(j * af[i]);
        }
        int k = 0;
        for (int m = 0; m <= m_max; ++m)
            for (int l = m; l <= l_max; ++l) {
                double p = 0;
                for (int n = (l - m) & 1; n <= l - m; n += 2) p = p + C(n, l, m) * tc[n] * ts[m];
                P(m, l, i) = p;
                d_sphere[(size_t)i * nc + k++] = fc[m] * p;
                if (m != 0) d_sphere[(size_t)i * nc + k++] = fs[m] * p;
            }
    }

    // ellipsoid log-curvature least squares: normal equations + LU
    const int n1 = nc + 1;
    std::vector<double> er(nfac), fm((size_t)nfac * n1, 0.0), nm((size_t)n1 * n1, 0.0), rhs(n1, 0.0);
    for (int i = 0; i < nfac; ++i) {
        const double st = std::sin(at[i]);
        const double s = std::pow(ea * st * std::cos(af[i]), 2) + std::pow(eb * st * std::sin(af[i]), 2) +
                         std::pow(ec * std::cos(at[i]), 2);
        er[i] = 2 * (std::log(ea * eb * ec) - std::log(s));
        int n = 0;
        for (int m = 0; m <= m_max; ++m)
            for (int l = m; l <= l_max; ++l) {
                ++n;
                if (m != 0) {
                    fm[(size_t)i * n1 + n] = P(m, l, i) * std::cos(m * af[i]);
                    ++n;
                    fm[(size_t)i * n1 + n] = P(m, l, i) * std::sin(m * af[i]);
                } else {
                    fm[(size_t)i * n1 + n] = P(m, l, i);
                }
            }
    }
    for (int r = 1; r <= nc; ++r) {
        for (int c = 1; c <= nc; ++c) {
            double acc = 0;
            for (int i = 0; i < nfac; ++i) acc = acc + fm[(size_t)i * n1 + r] * fm[(size_t)i * n1 + c];
            nm[(size_t)r * n1 + c] = acc;
        }
        double acc = 0;
        for (int i = 0; i < nfac; ++i) acc = acc + fm[(size_t)i * n1 + r] * er[i];
        rhs[r] = acc;
    }
    if (!lu_solve(nm, nc, rhs)) return psb_fail(PS_ERR_ARG, "ps_setup_shape: singular ellipsoid fit");
    for (int k = 1; k <= nc; ++k) cg_first[k - 1] = rhs[k];
    return PS_OK;
}
