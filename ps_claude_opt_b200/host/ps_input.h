// ps_input.h -- period_search_in reader and per-object preparation for the
// B200 host program.
//
// Restates the host half of PeriodSearch's main (period_search_BOINC.cpp):
// the 14 header lines (:343-387), the lightcurve blocks (:389-518), the
// trailing "lightcurve weight" pairs (:520-533), the epoch (:535-548), the
// weights (:552-564), the initial ellipsoid scale (:566-585), the frequency
// grid (:839-841) and the fitted-parameter mask (:843-857).  The shape tables
// come from ps_setup_shape in the engine library.
#pragma once
#include <cstdio>
#include <string>
#include <vector>

namespace psh {

struct Object {
    // header (period_search_in lines 1-14)
    double p_start = 0, p_coef = 0, p_end = 0;
    int ia_prd = 0;
    double jd00 = 0, phi0_deg = 0, conw = 0;
    int l_max = 0, m_max = 0, nrows = 0;
    double par[3] = {0, 0, 0};
    int ia_par[3] = {0, 0, 0};
    double cl = 0;
    int ia_cl = 0;
    double stop_condition = 0;
    int n_iter_min = 0;
    double lambda_incr = 0, lambda_incrr = 0, lambda_start = 0;

    // data, 0-based, pseudo-points not included
    int n_curves = 0, n_points = 0;
    std::vector<int> curve_len, curve_rel;
    std::vector<double> tim;         // JD - jd0
    std::vector<double> brightness, sig, sigr2, weight;
    std::vector<double> ee, ee0;     // [3*i + k], unit vectors to the observer / the Sun
    double jd_min = 0, jd_max = 0, jd0 = 0;
    bool onlyrel = true;

    // derived
    double escl = 0, conw_r = 0, phi0 = 0;
    int n_coef = 0, n_fac = 0;
    std::vector<double> normal, d_area, d_sphere, cg_first;
    std::vector<int> ia;             // 1-based, ma + 1 entries
    double freq_start = 0, freq_end = 0, freq_step = 0;
    int n_max = 0;

    int ma() const { return n_coef + 8; }
};

// Reads and prepares one object.  Returns false with a message in err on a
// malformed file or a failed shape setup.
bool read_object(std::FILE *f, Object &obj, std::string &err);

// Writes every prepared quantity as "name count values..." with C99 hex
// floats (exact), for comparison with other readers of the same file.
void dump_object(const Object &obj, std::FILE *out);

}  // namespace psh
