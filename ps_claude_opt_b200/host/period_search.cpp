// period_search.cpp -- the PeriodSearch host program on the B200 engine.
//
// Reads period_search_in, runs the convexity-weight search and the period
// scan through the C ABI (ps_gpu_prepare / ps_gpu_precalc / ps_gpu_start /
// ps_gpu_unprepare, the replacements of CUDAPrepare / CUDAPrecalc / CUDAStart
// / CUDAUnprepare) and writes period_search_out, one line per trial
// frequency in the reference's format (start_CUDA.cu:1220-1227).  This is the
// flow of the reference's main (period_search_BOINC.cpp:638-872) without the
// BOINC runtime.
//
// Checkpoint/resume (period_search_BOINC.cpp:101-118, 293-313): after the
// convexity-weight search and after every chunk of frequencies the program
// flushes the output and writes "<lines> <new_conw> <conw_r>" (%d %d %.17g)
// to the state file through a temporary file and a rename.  A later run that
// finds a valid state file skips the search, keeps the first <lines> lines of
// the output (dropping any written after the last checkpoint) and continues
// from frequency <lines> + 1.
//
//   period_search [options] [input [output]]
//     -d N           CUDA device (default 0)
//     -s PATH        state file (default period_search_state)
//     --chunk N      frequencies per checkpoint (default 1024)
//     --max-freq N   stop after N frequencies of the grid
//     --quirks Q     PS_QUIRK_* bits
//     --fresh        ignore an existing state file
//     --stop-after N exit after N chunks, as an interrupted run would
//     --dump-object  print the prepared object (hex floats) and exit, no GPU
//     --precision P  fp64 (default) or mixed (FP32 facet sweep, 3xTF32
//                    tensor-core shape derivatives, FP64 elsewhere)
//     --screen MODEL fit only the frequencies a trained screening network
//                    ranks first (the top 3.4 % with one neighbour on either
//                    side, plus a 2 % audit sample), widen around a best line
//                    at the edge of a fitted run, probe its period-doubling
//                    partners, and fall back to the whole
//                    grid when the audit sample contradicts the ranking; one
//                    output line per fitted frequency, in frequency order; no
//                    checkpoints
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "ps_b200.h"
#include "ps_input.h"
#include "screen_flow.h"

namespace {

struct Options {
    int device = 0;
    std::string in = "period_search_in", out = "period_search_out", state = "period_search_state";
    int chunk = 1024, max_freq = 0, quirks = 0, stop_after = 0, precision = PS_PRECISION_FP64;
    bool fresh = false, dump = false;
    std::string screen;
};

int usage()
{
    std::fprintf(stderr,
                 "usage: period_search [-d device] [-s state] [--chunk N] [--max-freq N] [--quirks Q] [--fresh]\n"
                 "                     [--stop-after N] [--dump-object] [--precision fp64|mixed] [--screen MODEL]\n"
                 "                     [input [output]]\n");
    return 2;
}

bool parse_args(int argc, char **argv, Options &o)
{
    int pos = 0;
    for (int i = 1; i < argc; ++i) {
        const std::string a = argv[i];
        auto next = [&](int &v) {
            if (i + 1 >= argc) return false;
            v = std::atoi(argv[++i]);
            return true;
        };
        if (a == "-d") {
            if (!next(o.device)) return false;
        } else if (a == "-s") {
            if (i + 1 >= argc) return false;
            o.state = argv[++i];
        } else if (a == "--chunk") {
            if (!next(o.chunk) || o.chunk < 1) return false;
        } else if (a == "--max-freq") {
            if (!next(o.max_freq)) return false;
        } else if (a == "--quirks") {
            if (!next(o.quirks)) return false;
        } else if (a == "--stop-after") {
            if (!next(o.stop_after)) return false;
        } else if (a == "--fresh") {
            o.fresh = true;
        } else if (a == "--dump-object") {
            o.dump = true;
        } else if (a == "--precision") {
            if (i + 1 >= argc) return false;
            const std::string v = argv[++i];
            if (v == "fp64") o.precision = PS_PRECISION_FP64;
            else if (v == "mixed") o.precision = PS_PRECISION_MIXED;
            else return false;
        } else if (a == "--screen") {
            if (i + 1 >= argc) return false;
            o.screen = argv[++i];
        } else if (!a.empty() && a[0] == '-') {
            return false;
        } else if (pos == 0) {
            o.in = a;
            ++pos;
        } else if (pos == 1) {
            o.out = a;
            ++pos;
        } else {
            return false;
        }
    }
    return true;
}

// C round(): half away from zero, as the reference's round() before %4.0f.
void print_line(std::FILE *f, const ps_line &l)
{
    std::fprintf(f, "%.8f  %.6f  %.6f %4.1f %4.0f %4.0f\n", l.period_h, l.rms, l.chisq, l.dark,
                 std::round(l.lambda_deg), std::round(l.beta_deg));
}

bool write_state(const std::string &path, int nlines, int new_conw, double conw_r)
{
    const std::string tmp = path + ".tmp";
    std::FILE *f = std::fopen(tmp.c_str(), "w");
    if (!f) return false;
    std::fprintf(f, "%d %d %.17g", nlines, new_conw, conw_r);
    if (std::fclose(f) != 0) return false;
    return std::rename(tmp.c_str(), path.c_str()) == 0;
}

bool read_state(const std::string &path, int &nlines, int &new_conw, double &conw_r)
{
    std::FILE *f = std::fopen(path.c_str(), "r");
    if (!f) return false;
    const int n = std::fscanf(f, "%d %d %lf", &nlines, &new_conw, &conw_r);
    std::fclose(f);
    return n == 3 && nlines >= 0;
}

// Keeps the first nlines lines of the output file (lines written after the
// last checkpoint are dropped) and reopens it for appending.
std::FILE *reopen_output(const std::string &path, int nlines)
{
    std::string kept;
    if (std::FILE *f = std::fopen(path.c_str(), "r")) {
        int c, seen = 0;
        while (seen < nlines && (c = std::fgetc(f)) != EOF) {
            kept.push_back((char)c);
            if (c == '\n') ++seen;
        }
        std::fclose(f);
        if (seen < nlines) return nullptr;   // output shorter than the checkpoint says
    } else if (nlines > 0) {
        return nullptr;
    }
    std::FILE *f = std::fopen(path.c_str(), "w");
    if (!f) return nullptr;
    std::fwrite(kept.data(), 1, kept.size(), f);
    return f;
}

// A screening network file: "PSMLP001", int32 layer count, int32 sizes,
// then float32 weights [out][in] and biases [out] per layer.
bool read_model(const std::string &path, std::vector<int32_t> &sizes, std::vector<float> &params)
{
    std::FILE *f = std::fopen(path.c_str(), "rb");
    if (!f) return false;
    char magic[8];
    int32_t nl = 0;
    bool ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, "PSMLP001", 8) == 0 &&
              std::fread(&nl, 4, 1, f) == 1 && nl >= 1 && nl <= 16;
    if (ok) {
        sizes.resize(nl + 1);
        ok = std::fread(sizes.data(), 4, nl + 1, f) == (size_t)(nl + 1);
    }
    size_t n = 0;
    if (ok)
        for (int l = 0; l < nl; ++l) n += (size_t)sizes[l + 1] * sizes[l] + sizes[l + 1];
    if (ok) {
        params.resize(n);
        ok = std::fread(params.data(), 4, n, f) == n && std::fgetc(f) == EOF;
    }
    std::fclose(f);
    return ok;
}

int fail(const char *what)
{
    std::fprintf(stderr, "period_search: %s: %s\n", what, ps_last_error());
    return 1;
}

}  // namespace

int main(int argc, char **argv)
{
    Options opt;
    if (!parse_args(argc, argv, opt)) return usage();

    std::FILE *in = std::fopen(opt.in.c_str(), "r");
    if (!in) {
        std::fprintf(stderr, "period_search: cannot open %s\n", opt.in.c_str());
        return 1;
    }
    psh::Object obj;
    std::string err;
    const bool ok = psh::read_object(in, obj, err);
    std::fclose(in);
    if (!ok) {
        std::fprintf(stderr, "period_search: %s\n", err.c_str());
        return 1;
    }
    if (opt.dump) {
        psh::dump_object(obj, stdout);
        return 0;
    }

    // initial poles (period_search_BOINC.cpp:229-238)
    const double lambda_pole[PS_N_POLES] = {0, 90, 180, 270, 60, 180, 300, 60, 180, 300};
    const double beta_pole[PS_N_POLES] = {0, 0, 0, 0, 60, 60, 60, -60, -60, -60};

    // the host thread sleeps while the GPU works instead of spinning
    // (as the reference asks for, start_CUDA.cu:129-148); the flag only
    // takes effect before the device is first used
    cudaSetDeviceFlags(cudaDeviceScheduleBlockingSync);
    ps_gpu *h = nullptr;
    if (ps_gpu_prepare(opt.device, beta_pole, lambda_pole, obj.par, obj.cl, obj.lambda_start, obj.lambda_incr,
                       obj.lambda_incrr, obj.ee.data(), obj.ee0.data(), obj.tim.data(), obj.phi0, obj.n_points,
                       obj.weight.data(), &h) != PS_OK)
        return fail("prepare");
    if (opt.quirks) ps_gpu_set_quirks(h, opt.quirks);
    if (ps_gpu_set_precision(h, opt.precision) != PS_OK) {
        ps_gpu_unprepare(h);
        return fail("precision");
    }

    const ps_curves curves{obj.n_curves, obj.curve_len.data(), obj.curve_rel.data()};
    const ps_shape shape{obj.n_coef, obj.normal.data(), obj.d_area.data(), obj.d_sphere.data()};
    const int nc = obj.n_coef;
    const int32_t *ia_par = &obj.ia[nc + 4];

    int nlines = 0, new_conw = 0;
    double conw_r = obj.conw_r;
    const bool resume = !opt.fresh && read_state(opt.state, nlines, new_conw, conw_r);
    std::FILE *out = resume ? reopen_output(opt.out, nlines) : std::fopen(opt.out.c_str(), "w");
    if (!out) {
        std::fprintf(stderr, "period_search: cannot open %s%s\n", opt.out.c_str(),
                     resume ? " (shorter than the checkpoint)" : "");
        ps_gpu_unprepare(h);
        return 1;
    }

    if (!resume) {
        // convexity-weight search (period_search_BOINC.cpp:646-770)
        new_conw = 0;
        while (new_conw != 1 && conw_r * obj.escl * obj.escl < 10.0) {
            if (ps_gpu_precalc(h, obj.freq_start, obj.freq_end, obj.freq_step, obj.stop_condition, obj.n_iter_min,
                               &conw_r, obj.n_points, obj.ia.data(), ia_par, &new_conw, obj.cg_first.data(),
                               obj.sig.data(), obj.sigr2.data(), obj.n_fac, obj.brightness.data(), &curves,
                               &shape) != PS_OK) {
                std::fclose(out);
                ps_gpu_unprepare(h);
                return fail("precalc");
            }
        }
        std::fflush(out);
        if (!write_state(opt.state, 0, new_conw, conw_r)) std::fprintf(stderr, "period_search: checkpoint failed\n");
    }

    int n_last = obj.n_max;
    if (opt.max_freq > 0 && opt.max_freq < n_last) n_last = opt.max_freq;

    if (!opt.screen.empty()) {
        // screened scan: rank every frequency, fit the chosen ones
        std::vector<int32_t> sizes;
        std::vector<float> params;
        if (!read_model(opt.screen, sizes, params)) {
            std::fprintf(stderr, "period_search: cannot read screening model %s\n", opt.screen.c_str());
            std::fclose(out);
            ps_gpu_unprepare(h);
            return 1;
        }
        std::vector<double> freqs(n_last);
        for (int f = 0; f < n_last; ++f) freqs[f] = obj.freq_start - f * obj.freq_step;
        std::vector<float> score(n_last);
        if (ps_screen_rank(opt.device, obj.n_points, obj.tim.data(), obj.brightness.data(), &curves, n_last,
                           freqs.data(), (int32_t)sizes.size() - 1, sizes.data(), params.data(),
                           score.data()) != PS_OK) {
            std::fclose(out);
            ps_gpu_unprepare(h);
            return fail("screen");
        }
        std::vector<char> core, aud;
        psflow::screen_parts(score, 0.034, 1, 0.02, 0, core, aud);
        if (ps_gpu_configure(h, obj.freq_start, obj.freq_step, obj.stop_condition, obj.n_iter_min, conw_r, conw_r,
                             obj.n_points, obj.ia.data(), ia_par, obj.cg_first.data(), obj.sig.data(),
                             obj.sigr2.data(), obj.n_fac, obj.brightness.data(), &curves, &shape) != PS_OK) {
            std::fclose(out);
            ps_gpu_unprepare(h);
            return fail("screened scan");
        }
        psflow::Plan sc(n_last);
        std::vector<ps_line> line(n_last);
        // fits the given frequencies, all poles: keeps their lines, returns their rms
        auto fit = [&](const std::vector<int> &sel, std::vector<double> &rms) {
            std::vector<int32_t> nf, pl;
            for (int f : sel)
                for (int p = 0; p < PS_N_POLES; ++p) {
                    nf.push_back(f + 1);
                    pl.push_back(p);
                }
            std::vector<ps_fit_result> res(nf.size());
            if (ps_gpu_fit_items(h, (int32_t)nf.size(), nf.data(), pl.data(), res.data()) != PS_OK) return false;
            for (size_t q = 0; q < sel.size(); ++q) {
                const ps_fit_result *r = &res[q * PS_N_POLES];
                int best = -1;  // NaN-safe, earliest pole wins ties (start_CUDA.cu:1200-1229)
                for (int p = 0; p < PS_N_POLES; ++p)
                    if (best < 0 || (!std::isnan(r[p].dev) && !(r[p].dev >= r[best].dev))) best = p;
                const ps_fit_result &b = r[best];
                const int f = sel[q];
                line[f] = ps_line{24 * b.per, b.dev, b.dev * b.dev * obj.n_points,
                                  f == 0 ? conw_r * obj.escl * obj.escl : b.dark, b.lambda_deg, b.beta_deg};
                rms[q] = b.dev;
            }
            return true;
        };
        bool ok = psflow::run_plan(sc, core, aud, obj.freq_start, obj.freq_step, fit);
        if (ok && opt.precision == PS_PRECISION_MIXED) {
            // the candidates' final fits in FP64
            ok = ps_gpu_set_precision(h, PS_PRECISION_FP64) == PS_OK &&
                 ps_gpu_configure(h, obj.freq_start, obj.freq_step, obj.stop_condition, obj.n_iter_min, conw_r,
                                  conw_r, obj.n_points, obj.ia.data(), ia_par, obj.cg_first.data(), obj.sig.data(),
                                  obj.sigr2.data(), obj.n_fac, obj.brightness.data(), &curves, &shape) == PS_OK &&
                 psflow::polish(sc, obj.freq_start, obj.freq_step, fit);
        }
        if (!ok) {
            std::fclose(out);
            ps_gpu_unprepare(h);
            return fail("screened scan");
        }
        int n_fit = 0;
        for (int f = 0; f < n_last; ++f)
            if (sc.fitted[f]) {
                print_line(out, line[f]);
                ++n_fit;
            }
        std::fclose(out);
        std::fprintf(stderr,
                     "period_search: screened scan fitted %d of %d frequencies (first selection %d, %d edge "
                     "expansions, %d period-doubling probes%s%s; %d refitted in FP64)\n",
                     n_fit, n_last, sc.initial, sc.expansions, sc.alias_probes,
                     sc.fallback ? ", fell back to the full grid: " : "", sc.reason, sc.polished);
        ps_gpu_unprepare(h);
        return 0;
    }
    std::vector<ps_line> lines(opt.chunk);
    int chunks = 0;
    for (int n = nlines + 1; n <= n_last;) {
        const int want = std::min(opt.chunk, n_last - n + 1);
        int32_t got = 0;
        if (ps_gpu_start(h, n, obj.freq_start, obj.freq_end, obj.freq_step, obj.stop_condition, obj.n_iter_min,
                         conw_r, obj.n_points, obj.ia.data(), ia_par, obj.cg_first.data(), obj.escl, obj.sig.data(),
                         obj.sigr2.data(), obj.n_fac, obj.brightness.data(), &curves, &shape, lines.data(), want,
                         &got, nullptr, nullptr) != PS_OK) {
            std::fclose(out);
            ps_gpu_unprepare(h);
            return fail("scan");
        }
        for (int i = 0; i < got; ++i) print_line(out, lines[i]);
        std::fflush(out);
        n += got;
        nlines += got;
        if (!write_state(opt.state, nlines, new_conw, conw_r)) std::fprintf(stderr, "period_search: checkpoint failed\n");
        std::fprintf(stderr, "period_search: %d / %d frequencies\n", nlines, n_last);
        if (got < want) break;
        if (opt.stop_after > 0 && ++chunks >= opt.stop_after && n <= n_last) {
            std::fclose(out);
            ps_gpu_unprepare(h);
            return 0;
        }
    }
    std::fclose(out);
    int32_t flags = 0;
    ps_gpu_status(h, &flags);
    if (flags) std::fprintf(stderr, "period_search: device status 0x%x\n", (unsigned)flags);
    ps_gpu_unprepare(h);
    return 0;
}
