// ps_input.cpp -- period_search_in reader (see ps_input.h).
#include "ps_input.h"

#include <cmath>
#include <cstdarg>
#include <cstring>

#include "ps_b200.h"

namespace psh {

namespace {

constexpr double kPi = 3.14159265358979323846;
constexpr double kDeg2Rad = kPi / 180.0;

// One header line: the leading values, then the rest of the line (the
// reference reads each with fscanf and drops the comment with fgets).
bool header_line(std::FILE *f, const char *fmt, int want, std::string &err, const char *what, ...)
{
    va_list ap;
    va_start(ap, what);
    const int got = std::vfscanf(f, fmt, ap);
    va_end(ap);
    if (got != want) {
        err = std::string("period_search_in: cannot read ") + what;
        return false;
    }
    int c;
    while ((c = std::fgetc(f)) != EOF && c != '\n') {
    }
    return true;
}

void skip_line(std::FILE *f)
{
    int c;
    while ((c = std::fgetc(f)) != EOF && c != '\n') {
    }
}

}  // namespace

bool read_object(std::FILE *f, Object &o, std::string &err)
{
    // header (period_search_BOINC.cpp:343-387)
    if (!header_line(f, "%lf %lf %lf %d", 4, err, "period start/step/end", &o.p_start, &o.p_coef, &o.p_end,
                     &o.ia_prd))
        return false;
    if (!header_line(f, "%lf", 1, err, "epoch", &o.jd00)) return false;
    if (!header_line(f, "%lf", 1, err, "initial rotation angle", &o.phi0_deg)) return false;
    if (!header_line(f, "%lf", 1, err, "convexity weight", &o.conw)) return false;
    if (!header_line(f, "%d %d", 2, err, "Laplace series degree and order", &o.l_max, &o.m_max)) return false;
    if (!header_line(f, "%d", 1, err, "triangulation rows", &o.nrows)) return false;
    for (int k = 0; k < 3; ++k)
        if (!header_line(f, "%lf %d", 2, err, "phase-function parameter", &o.par[k], &o.ia_par[k])) return false;
    if (!header_line(f, "%lf %d", 2, err, "Lambert coefficient", &o.cl, &o.ia_cl)) return false;
    if (!header_line(f, "%lf", 1, err, "stop condition", &o.stop_condition)) return false;
    if (!header_line(f, "%d", 1, err, "minimum iterations", &o.n_iter_min)) return false;
    if (!header_line(f, "%lf", 1, err, "lambda factor", &o.lambda_incr)) return false;
    o.lambda_incrr = o.lambda_incr != 0.0 ? 1.0 / o.lambda_incr : 1.7976931348623157e308;
    if (!header_line(f, "%lf", 1, err, "initial lambda", &o.lambda_start)) return false;
    if (o.l_max < 0 || o.m_max < 0 || o.m_max > o.l_max || o.nrows < 1) {
        err = "period_search_in: bad Laplace degree/order or triangulation rows";
        return false;
    }

    // lightcurves (period_search_BOINC.cpp:389-518)
    if (std::fscanf(f, "%d", &o.n_curves) != 1 || o.n_curves < 1) {
        err = "period_search_in: cannot read the number of lightcurves";
        return false;
    }
    double al0 = kPi, al0_abs = kPi;
    int ial0 = -1, ial0_abs = -1;
    o.jd_min = 1e20;
    o.jd_max = -1e40;
    o.onlyrel = true;
    for (int i = 0; i < o.n_curves; ++i) {
        int lp = 0, calibrated = 0;
        if (std::fscanf(f, "%d %d", &lp, &calibrated) != 2 || lp < 1) {
            err = "period_search_in: bad lightcurve header " + std::to_string(i + 1);
            return false;
        }
        skip_line(f);
        const int rel = 1 - calibrated;
        o.curve_len.push_back(lp);
        o.curve_rel.push_back(rel);
        if (rel == 0) o.onlyrel = false;
        double ave = 0.0;
        for (int j = 0; j < lp; ++j) {
            double t, br, e0[3], e[3];
            if (std::fscanf(f, "%lf %lf %lf %lf %lf %lf %lf %lf", &t, &br, &e0[0], &e0[1], &e0[2], &e[0], &e[1],
                            &e[2]) != 8) {
                err = "period_search_in: bad data point " + std::to_string(j + 1) + " of lightcurve " +
                      std::to_string(i + 1);
                return false;
            }
            if (t < o.jd_min) o.jd_min = t;
            if (t > o.jd_max) o.jd_max = t;
            const double e0len = std::sqrt(e0[0] * e0[0] + e0[1] * e0[1] + e0[2] * e0[2]);
            const double elen = std::sqrt(e[0] * e[0] + e[1] * e[1] + e[2] * e[2]);
            ave += br;
            for (int k = 0; k < 3; ++k) {
                o.ee.push_back(e[k] / elen);
                o.ee0.push_back(e0[k] / e0len);
            }
            if (j == 0) {
                // solar phase angle of the curve's first point
                const double cosa = (e[0] * e0[0] + e[1] * e0[1] + e[2] * e0[2]) / (elen * e0len);
                const double a = std::acos(cosa);
                if (a < al0) {
                    al0 = a;
                    ial0 = o.n_points;
                }
                if (a < al0_abs && rel == 0) {
                    al0_abs = a;
                    ial0_abs = o.n_points;
                }
            }
            o.tim.push_back(t);
            o.brightness.push_back(br);
            ++o.n_points;
        }
        ave /= lp;
        // each curve's mean brightness is its sigma (period_search_BOINC.cpp:507-516)
        for (int j = 0; j < lp; ++j) {
            o.sig.push_back(ave);
            o.sigr2.push_back(1.0 / (ave * ave));
        }
    }

    // trailing "lightcurve weight" pairs (period_search_BOINC.cpp:520-533)
    std::vector<double> wlc(o.n_curves, -1.0);
    int lc;
    double w;
    while (std::fscanf(f, "%d %lf", &lc, &w) == 2)
        if (lc >= 1 && lc <= o.n_curves) wlc[lc - 1] = w;

    // epoch (period_search_BOINC.cpp:535-548)
    o.jd0 = o.jd00;
    if (o.jd0 <= 0) o.jd0 = static_cast<int>(o.jd_min);
    for (double &t : o.tim) t = t - o.jd0;
    o.phi0 = o.phi0_deg * kDeg2Rad;

    // per-point weights (period_search_BOINC.cpp:552-564)
    for (int i = 0; i < o.n_curves; ++i)
        for (int j = 0; j < o.curve_len[i]; ++j) o.weight.push_back(wlc[i] == -1 ? 1.0 : wlc[i]);

    // initial ellipsoid scale, calibrated data preferred (period_search_BOINC.cpp:566-585)
    if (!o.onlyrel) {
        al0 = al0_abs;
        ial0 = ial0_abs;
    }
    double a = 1.05, b = 1.00, c = 0.95;
    const double rfit = std::sqrt(2 * o.sig[ial0] / (0.5 * kPi * (1 + std::cos(al0))));
    o.escl = rfit / std::sqrt((a * b + b * c + a * c) / 3);
    if (!o.onlyrel) o.escl *= 0.8;
    a *= o.escl;
    b *= o.escl;
    c *= o.escl;
    o.conw_r = o.conw / o.escl / o.escl;

    // shape tables (trifac / areanorm / sphfunc / ellfit)
    o.n_coef = ps_n_coef(o.l_max, o.m_max);
    o.n_fac = 8 * o.nrows * o.nrows;
    if (o.n_coef + 8 > PS_MAX_PAR - 7 || o.n_fac > PS_MAX_FAC) {
        err = "period_search_in: shape model larger than the engine's limits (lmax <= 8, nrows <= 11)";
        return false;
    }
    o.normal.resize(3 * (size_t)o.n_fac);
    o.d_area.resize(o.n_fac);
    o.d_sphere.resize((size_t)o.n_fac * o.n_coef);
    o.cg_first.resize(o.n_coef);
    if (ps_setup_shape(o.l_max, o.m_max, o.nrows, a, b, c, o.normal.data(), o.d_area.data(), o.d_sphere.data(),
                       o.cg_first.data()) != PS_OK) {
        err = std::string("shape setup: ") + ps_last_error();
        return false;
    }

    // frequency grid (period_search_BOINC.cpp:839-841) and mask (:843-857)
    o.freq_start = 1 / o.p_start;
    o.freq_end = 1 / o.p_end;
    o.freq_step = 0.5 / (o.jd_max - o.jd_min) / 24 * o.p_coef;
    o.n_max = (int)((o.freq_start - o.freq_end) / o.freq_step) + 1;
    const int nc = o.n_coef, ma = o.ma();
    o.ia.assign(ma + 1, 0);
    for (int p = 1; p <= nc; ++p) o.ia[p] = 1;
    if (o.onlyrel) o.ia[1] = 0;
    o.ia[nc + 1] = 1;
    o.ia[nc + 2] = 1;
    o.ia[nc + 3] = o.ia_prd;
    for (int k = 0; k < 3; ++k) o.ia[nc + 4 + k] = o.ia_par[k];
    o.ia[ma - 1] = o.ia_cl;
    o.ia[ma] = 0;
    return true;
}

namespace {

void dump(std::FILE *out, const char *name, const double *v, size_t n)
{
    std::fprintf(out, "%s %zu", name, n);
    for (size_t i = 0; i < n; ++i) std::fprintf(out, " %a", v[i]);
    std::fputc('\n', out);
}

void dump(std::FILE *out, const char *name, const int *v, size_t n)
{
    std::fprintf(out, "%s %zu", name, n);
    for (size_t i = 0; i < n; ++i) std::fprintf(out, " %d", v[i]);
    std::fputc('\n', out);
}

}  // namespace

void dump_object(const Object &o, std::FILE *out)
{
    const double scal[] = {o.phi0, o.par[0], o.par[1], o.par[2], o.cl, o.lambda_start, o.lambda_incr,
                           o.lambda_incrr, o.stop_condition, o.conw_r, o.escl, o.jd0, o.freq_start, o.freq_end,
                           o.freq_step};
    dump(out, "scalars", scal, sizeof(scal) / sizeof(scal[0]));
    const int ints[] = {o.n_points, o.n_curves, o.n_coef, o.n_fac, o.n_iter_min, o.n_max, o.onlyrel ? 1 : 0};
    dump(out, "ints", ints, sizeof(ints) / sizeof(ints[0]));
    dump(out, "curve_len", o.curve_len.data(), o.curve_len.size());
    dump(out, "curve_rel", o.curve_rel.data(), o.curve_rel.size());
    dump(out, "ia", o.ia.data(), o.ia.size());
    dump(out, "tim", o.tim.data(), o.tim.size());
    dump(out, "brightness", o.brightness.data(), o.brightness.size());
    dump(out, "sig", o.sig.data(), o.sig.size());
    dump(out, "sigr2", o.sigr2.data(), o.sigr2.size());
    dump(out, "weight", o.weight.data(), o.weight.size());
    dump(out, "ee", o.ee.data(), o.ee.size());
    dump(out, "ee0", o.ee0.data(), o.ee0.size());
    dump(out, "normal", o.normal.data(), o.normal.size());
    dump(out, "d_area", o.d_area.data(), o.d_area.size());
    dump(out, "d_sphere", o.d_sphere.data(), o.d_sphere.size());
    dump(out, "cg_first", o.cg_first.data(), o.cg_first.size());
}

}  // namespace psh
