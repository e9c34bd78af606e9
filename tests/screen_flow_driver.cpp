// Test driver for ps_claude_opt_b200/host/screen_flow.h (the host program's
// screened-scan control flow): runs the flow on a synthetic rms landscape
// read from stdin and prints what it fitted, so a CPU test can compare it
// with ps_claude_opt_b200.screen (plan_scan, polish_plan).
//
// stdin:  n top halo audit seed freq_start freq_step polish
//         n scores (float), n rms values of the first pass, n FP64 rms values
// stdout: one JSON object.
#include <cstdio>
#include <vector>

#include "screen_flow.h"

static void print_list(const char *name, const std::vector<int> &v)
{
    std::printf("\"%s\": [", name);
    for (size_t i = 0; i < v.size(); ++i) std::printf("%s%d", i ? ", " : "", v[i]);
    std::printf("], ");
}

int main()
{
    int n = 0, halo = 0, do_polish = 0;
    double top = 0, audit = 0, f0 = 0, df = 0;
    unsigned long long seed = 0;
    if (std::scanf("%d %lf %d %lf %llu %lf %lf %d", &n, &top, &halo, &audit, &seed, &f0, &df, &do_polish) != 8)
        return 2;
    std::vector<float> score(n);
    std::vector<double> rms(n), rms64(n);
    for (float &x : score)
        if (std::scanf("%f", &x) != 1) return 2;
    for (double &x : rms)
        if (std::scanf("%lf", &x) != 1) return 2;
    for (double &x : rms64)
        if (std::scanf("%lf", &x) != 1) return 2;

    std::vector<char> core, aud;
    psflow::screen_parts(score, top, halo, audit, seed, core, aud);
    std::vector<std::vector<int>> calls;
    auto fit = [&](const std::vector<int> &sel, std::vector<double> &r) {
        calls.push_back(sel);
        for (size_t q = 0; q < sel.size(); ++q) r[q] = rms[sel[q]];
        return true;
    };
    auto fit64 = [&](const std::vector<int> &sel, std::vector<double> &r) {
        calls.push_back(sel);
        for (size_t q = 0; q < sel.size(); ++q) r[q] = rms64[sel[q]];
        return true;
    };
    psflow::Plan p(n);
    if (!psflow::run_plan(p, core, aud, f0, df, fit)) return 1;
    const int best_plan = psflow::best_fitted(p);
    if (do_polish && !psflow::polish(p, f0, df, fit64)) return 1;

    std::vector<int> fitted, c, a;
    for (int i = 0; i < n; ++i) {
        if (p.fitted[i]) fitted.push_back(i);
        if (core[i]) c.push_back(i);
        if (aud[i]) a.push_back(i);
    }
    std::printf("{");
    print_list("core", c);
    print_list("audit", a);
    print_list("fitted", fitted);
    std::printf("\"calls\": [");
    for (size_t k = 0; k < calls.size(); ++k) {
        std::printf("%s[", k ? ", " : "");
        for (size_t i = 0; i < calls[k].size(); ++i) std::printf("%s%d", i ? ", " : "", calls[k][i]);
        std::printf("]");
    }
    std::printf("], \"initial\": %d, \"expansions\": %d, \"alias_probes\": %d, \"fallback\": %s, "
                "\"reason\": \"%s\", \"best_plan\": %d, \"best\": %d, \"polished\": %d, \"polish_rounds\": %d}\n",
                p.initial, p.expansions, p.alias_probes, p.fallback ? "true" : "false", p.reason, best_plan,
                psflow::best_fitted(p), p.polished, p.polish_rounds);
    return 0;
}
