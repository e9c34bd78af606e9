// screen_flow.h -- control flow of the screened scan, independent of the
// device: which frequencies a screened scan fits, in which rounds, when it
// widens, probes period-doubling partners, falls back to the full grid and,
// for mixed-precision fits, which candidates it refits in FP64.  The same
// steps as ps_claude_opt_b200.screen (select_parts, plan_scan, polish_plan);
// the period_search program drives it with GPU fits, a CPU test with
// synthetic rms landscapes.
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

namespace psflow {

constexpr double kAuditMargin = 0.10;  // an audit line within 10 % of the best rms: fall back
constexpr int kEdge = 2;               // frequencies fitted each side of a best line at a run edge
constexpr int kMaxExpansions = 8;      // edge expansions before falling back
constexpr int kPolishMinima = 8;       // mixed precision: lowest local minima refitted in FP64
constexpr int kPolishRounds = 4;       // ... and rounds of FP64 refits around a moving best line

// The frequencies (0-based) a screened scan fits first: the core -- the
// lowest-scoring `top` share with `halo` neighbours each side -- and an
// `audit` share of the rest drawn by a partial Fisher-Yates shuffle from a
// 64-bit linear congruential generator (select_parts draws the same sample).
// core[i] / aud[i] mark the two sets.
inline void screen_parts(const std::vector<float> &score, double top, int halo, double audit, uint64_t seed,
                         std::vector<char> &core, std::vector<char> &aud)
{
    const int n = (int)score.size();
    std::vector<int> order(n);
    for (int i = 0; i < n; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return score[a] < score[b]; });
    const int k = std::max(1, (int)std::nearbyint(top * n));
    core.assign(n, 0);
    aud.assign(n, 0);
    for (int r = 0; r < k; ++r)
        for (int d = -halo; d <= halo; ++d)
            if (order[r] + d >= 0 && order[r] + d < n) core[order[r] + d] = 1;
    std::vector<int> rest;
    for (int i = 0; i < n; ++i)
        if (!core[i]) rest.push_back(i);
    const int na = std::min((int)rest.size(), std::max(1, (int)std::nearbyint(audit * n)));
    uint64_t x = seed * 2654435761ull + 1ull;
    for (int j = 0; j < na; ++j) {
        x = 6364136223846793005ull * x + 1442695040888963407ull;
        const uint64_t r = x >> 33;
        const int pick = j + (int)(r % (uint64_t)(rest.size() - j));
        std::swap(rest[j], rest[pick]);
        aud[rest[j]] = 1;
    }
}

// State of one screened scan over n frequencies.
struct Plan {
    std::vector<double> rms;   // best rms over the poles, where fitted
    std::vector<char> fitted;
    int initial = 0, expansions = 0, alias_probes = 0, polished = 0, polish_rounds = 0;
    bool fallback = false;
    const char *reason = "";   // why it fell back: "audit" or "edge"
    explicit Plan(int n) : rms(n, NAN), fitted(n, 0) {}
    int size() const { return (int)rms.size(); }
};

// Lowest-rms fitted frequency (NaN never wins; the first minimum wins ties), or -1.
inline int best_fitted(const Plan &p)
{
    int b = -1;
    double br = INFINITY;
    for (int i = 0; i < p.size(); ++i)
        if (p.fitted[i] && p.rms[i] < br) {
            b = i;
            br = p.rms[i];
        }
    return b;
}

// 0-based grid indices nearest the period-doubling partners (twice and half
// the frequency) of index b that lie on a grid of n frequencies
// freq_start - i freq_step.
inline std::vector<int> alias_indices(double freq_start, double freq_step, int n, int b)
{
    std::vector<int> out;
    if (freq_step <= 0) return out;
    const double fb = freq_start - b * freq_step;
    for (double t : {2.0 * fb, 0.5 * fb}) {
        // nearest grid index, halves to even like Python's round()
        const int a = (int)std::nearbyint((freq_start - t) / freq_step);
        if (a >= 0 && a < n) out.push_back(a);
    }
    return out;
}

// Fits (fit(sel, rms) fills rms[q] for each 0-based frequency sel[q], all
// poles, and returns false on failure) the frequencies of sel that the plan
// has not fitted yet, and records their rms.
template <class Fit>
bool fit_new(Plan &p, const std::vector<int> &want, Fit &fit)
{
    std::vector<int> sel;
    for (int f : want)
        if (f >= 0 && f < p.size() && !p.fitted[f]) sel.push_back(f);
    std::sort(sel.begin(), sel.end());
    sel.erase(std::unique(sel.begin(), sel.end()), sel.end());
    if (sel.empty()) return true;
    std::vector<double> r(sel.size());
    if (!fit(sel, r)) return false;
    for (size_t q = 0; q < sel.size(); ++q) {
        p.rms[sel[q]] = r[q];
        p.fitted[sel[q]] = 1;
    }
    return true;
}

inline std::vector<int> range_of(int lo, int hi)
{
    std::vector<int> v;
    for (int i = lo; i <= hi; ++i) v.push_back(i);
    return v;
}

// The screened scan (plan_scan): fit the core and the audit sample; while
// the best line has an unfitted neighbour, fit kEdge more frequencies each
// side of it (at most kMaxExpansions times, then fall back); fit the
// neighbourhoods of the best line's period-doubling partners once per best
// line, widening again if one wins; if an audit frequency farther than kEdge
// from the best line comes within kAuditMargin (relative) of its rms, fall
// back.  Falling back fits every remaining frequency, which makes the
// result the full scan's.  Returns false if a fit failed.
template <class Fit>
bool run_plan(Plan &p, const std::vector<char> &core, const std::vector<char> &aud, double freq_start,
              double freq_step, Fit &fit)
{
    const int n = p.size();
    std::vector<int> first;
    for (int f = 0; f < n; ++f)
        if (core[f] || aud[f]) first.push_back(f);
    if (!fit_new(p, first, fit)) return false;
    for (int f = 0; f < n; ++f) p.initial += p.fitted[f];
    std::vector<char> probed(n, 0);
    while (!p.fallback) {
        for (;;) {  // widen around a best line at the edge of a fitted run
            const int b = best_fitted(p);
            if (b < 0) {
                p.fallback = true;
                p.reason = "edge";
                break;
            }
            const bool open = (b > 0 && !p.fitted[b - 1]) || (b + 1 < n && !p.fitted[b + 1]);
            if (!open) break;
            if (p.expansions >= kMaxExpansions) {
                p.fallback = true;
                p.reason = "edge";
                break;
            }
            if (!fit_new(p, range_of(b - kEdge, b + kEdge), fit)) return false;
            ++p.expansions;
        }
        if (p.fallback) break;
        // probe the best line's period-doubling partners (twice and half its frequency) once
        const int b = best_fitted(p);
        if (probed[b]) break;
        probed[b] = 1;
        std::vector<int> around;
        for (int a : alias_indices(freq_start, freq_step, n, b))
            for (int i = a - kEdge; i <= a + kEdge; ++i) around.push_back(i);
        if (!fit_new(p, around, fit)) return false;
        ++p.alias_probes;
        if (best_fitted(p) == b) break;
    }
    if (!p.fallback) {
        const int b = best_fitted(p);
        for (int a = 0; a < n; ++a)
            if (aud[a] && std::abs(a - b) > kEdge && p.fitted[a] && p.rms[a] <= p.rms[b] * (1.0 + kAuditMargin)) {
                p.fallback = true;
                p.reason = "audit";
                break;
            }
    }
    if (p.fallback) return fit_new(p, range_of(0, n - 1), fit);
    return true;
}

// Mixed-precision fits: refit the candidates in FP64 (polish_plan).  In the
// first round the kPolishMinima lowest local minima of the rms over the
// fitted frequencies (an unfitted or NaN neighbour counts as higher) with
// one neighbour each side; in every round the best line and its
// period-doubling partners with kEdge neighbours each side; rounds repeat
// while they add frequencies, at most kPolishRounds times.  fit64 has fit's
// signature; refitted frequencies may include unfitted ones, which become
// fitted.  Returns false if a fit failed.
template <class Fit>
bool polish(Plan &p, double freq_start, double freq_step, Fit &fit64)
{
    const int n = p.size();
    std::vector<char> done(n, 0);
    auto key = [&](int i) {
        if (i < 0 || i >= n || !p.fitted[i] || std::isnan(p.rms[i])) return (double)INFINITY;
        return p.rms[i];
    };
    for (int round = 0; round < kPolishRounds; ++round) {
        const int b = best_fitted(p);
        if (b < 0) break;
        std::vector<char> need(n, 0);
        auto mark = [&](int lo, int hi) {
            for (int i = std::max(0, lo); i <= std::min(n - 1, hi); ++i) need[i] = 1;
        };
        mark(b - kEdge, b + kEdge);
        for (int a : alias_indices(freq_start, freq_step, n, b)) mark(a - kEdge, a + kEdge);
        if (round == 0) {
            std::vector<int> loc;
            for (int i = 0; i < n; ++i)
                if (key(i) < INFINITY && key(i) <= key(i - 1) && key(i) <= key(i + 1)) loc.push_back(i);
            std::stable_sort(loc.begin(), loc.end(), [&](int x, int y) { return key(x) < key(y); });
            for (size_t q = 0; q < loc.size() && q < (size_t)kPolishMinima; ++q) mark(loc[q] - 1, loc[q] + 1);
        }
        std::vector<int> sel;
        for (int i = 0; i < n; ++i)
            if (need[i] && !done[i]) sel.push_back(i);
        if (sel.empty()) break;
        std::vector<double> r(sel.size());
        if (!fit64(sel, r)) return false;
        for (size_t q = 0; q < sel.size(); ++q) {
            p.rms[sel[q]] = r[q];
            p.fitted[sel[q]] = 1;
            done[sel[q]] = 1;
        }
        p.polished += (int)sel.size();
        p.polish_rounds = round + 1;
    }
    return true;
}

}  // namespace psflow
