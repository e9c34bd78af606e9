// batch.cu -- ps_gpu_scan_batch: the convexity-weight search and the period
// scan of many objects on one GPU.
//
// The reference runs one object per process (period_search_BOINC.cpp:
// 638-872): a convexity-weight search of 100 fits per round
// (start_CUDA.cu:400-789) -- too few to fill 148 SMs -- and then the scan.
// Here every object gets its own handle (tables, items, results), and the
// launches of all objects go to kSlots streams: each search round launches
// every still-searching object at once, and the scans follow, so kernels of
// different objects overlap and the tail of one object's persistent launch
// is filled by the next object's CTAs.  Objects go to slots largest first,
// each to the slot with the least work so far.  A slot's launches run one
// after another and share its scratch and queue counter; every launch
// zeroes the counter on the slot's stream before it starts.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <numeric>
#include <vector>

#include "engine.h"
#include "handle.h"
#include "ps_b200.h"
#include "util.h"

namespace {

constexpr int kSlots = 4;
constexpr int kTestPeriods = 10;  // start_CUDA.cu:420

struct Slot {
    cudaStream_t stream = nullptr;
    psb::DevBuf<double> scratch;
    psb::DevBuf<int> queue;
    size_t scratch_doubles = 0;
};

struct Batch {
    std::vector<ps_gpu *> h;
    Slot slot[kSlots];
    ~Batch()
    {
        for (Slot &s : slot) {
            if (s.stream) cudaStreamSynchronize(s.stream);
            s.scratch.release();
            s.queue.release();
            if (s.stream) cudaStreamDestroy(s.stream);
        }
        for (ps_gpu *x : h) ps_gpu_unprepare(x);
    }
};

ps_status configure(ps_gpu *h, const ps_object &o, double conw_r, double conw_r_rms)
{
    return ps_gpu_configure(h, o.freq_start, o.freq_step, o.stop_condition, o.n_iter_min, conw_r, conw_r_rms,
                            o.ndata, o.ia, o.ia_par, o.cg_first, o.sig, o.sigr2, o.numfac, o.brightness, &o.curves,
                            &o.shape);
}

// Uploads the items of each job, launches all jobs on their slots and
// brings the results back.  job = (object index, items).
ps_status run_jobs(Batch &b, const std::vector<int> &slot_of, const std::vector<std::pair<int, std::vector<psb::FitItem>>> &jobs,
                   std::vector<std::vector<psb::FitOut>> &res)
{
    res.assign(jobs.size(), {});
    // everything a launch reads is on the device before the first launch
    for (Slot &s : b.slot) {
        if (s.scratch_doubles) PSB_CUDA(s.scratch.ensure(s.scratch_doubles));
        PSB_CUDA(s.queue.ensure(1));
    }
    for (const auto &j : jobs) {
        ps_gpu *h = b.h[j.first];
        PSB_CUDA(psb::upload(h->items, j.second, h->stream));
        PSB_CUDA(h->out.ensure(j.second.size()));
        PSB_CUDA(cudaStreamSynchronize(h->stream));
    }
    for (const auto &j : jobs) {
        ps_gpu *h = b.h[j.first];
        Slot &s = b.slot[slot_of[j.first]];
        const int n = (int)j.second.size();
        if (n == 0) continue;
        const int n_ctas = std::max(1, std::min(n, h->ctas_per_sm * h->n_sm));
        PSB_CUDA(cudaMemsetAsync(s.queue.ptr, 0, sizeof(int), s.stream));
        const int e = psb::launch_fits(h->obj, h->prm, h->items.ptr, n, s.queue.ptr, h->out.ptr, s.scratch.ptr,
                                       h->scratch_per_cta, n_ctas, h->status.ptr, s.stream);
        if (e) return psb_fail_cuda(e, "ps_gpu_scan_batch: fit kernel launch");
    }
    for (Slot &s : b.slot) PSB_CUDA(cudaStreamSynchronize(s.stream));
    for (size_t k = 0; k < jobs.size(); ++k) {
        ps_gpu *h = b.h[jobs[k].first];
        res[k].resize(jobs[k].second.size());
        if (!res[k].empty())
            PSB_CUDA(cudaMemcpy(res[k].data(), h->out.ptr, res[k].size() * sizeof(psb::FitOut),
                                cudaMemcpyDeviceToHost));
    }
    return PS_OK;
}

int scan_lines(const ps_object &o)
{
    const int n_max = (int)((o.freq_start - o.freq_end) / o.freq_step) + 1;
    return std::max(0, std::min(n_max - o.n_start_from + 1, (int)o.max_lines));
}

}  // namespace

extern "C" ps_status ps_gpu_scan_batch(int32_t device, int32_t n_obj, const ps_object *objs, int32_t quirks,
                                       ps_line *lines, const int64_t *line_offset, int32_t *n_lines,
                                       double *conw_r_out)
{
    if (n_obj < 0 || (n_obj > 0 && (!objs || !lines || !line_offset || !n_lines || !conw_r_out)))
        return psb_fail(PS_ERR_ARG, "ps_gpu_scan_batch: null argument");
    for (int i = 0; i < n_obj; ++i) {
        if (objs[i].n_start_from < 1 || objs[i].max_lines < 0 || line_offset[i] < 0)
            return psb_fail(PS_ERR_ARG, "ps_gpu_scan_batch: n_start_from < 1, max_lines < 0 or line_offset < 0");
        if (!(objs[i].freq_step > 0)) return psb_fail(PS_ERR_ARG, "ps_gpu_scan_batch: freq_step must be > 0");
        n_lines[i] = 0;
    }
    if (n_obj == 0) return PS_OK;

    Batch b;
    b.h.assign(n_obj, nullptr);
    for (int i = 0; i < n_obj; ++i) {
        const ps_object &o = objs[i];
        ps_status st = ps_gpu_prepare(device, o.beta_pole, o.lambda_pole, o.par, o.cl, o.alamda_start, o.alamda_incr,
                                      o.alamda_incrr, o.ee, o.ee0, o.tim, o.phi0, o.ndata, o.weight, &b.h[i]);
        if (st != PS_OK) return st;
        b.h[i]->quirks = quirks;
        // a first configure validates the object and sizes its scratch
        st = configure(b.h[i], o, o.conw_r, o.conw_r);
        if (st != PS_OK) return st;
    }
    PSB_CUDA(cudaSetDevice(device));
    for (Slot &s : b.slot) PSB_CUDA(cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking));

    // slots: largest object first, each to the least-loaded slot
    std::vector<double> cost(n_obj);
    for (int i = 0; i < n_obj; ++i) {
        const psb::DevObject &d = b.h[i]->obj;
        cost[i] = (double)(scan_lines(objs[i]) + kTestPeriods) * d.n_points * d.n_fac * d.ncp;
    }
    std::vector<int> order(n_obj), slot_of(n_obj);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return cost[x] > cost[y]; });
    double load[kSlots] = {0, 0, 0, 0};
    for (int i : order) {
        const int s = (int)(std::min_element(load, load + kSlots) - load);
        slot_of[i] = s;
        load[s] += cost[i];
        ps_gpu *h = b.h[i];
        const int n_ctas = h->ctas_per_sm * h->n_sm;
        b.slot[s].scratch_doubles = std::max(b.slot[s].scratch_doubles, h->scratch_per_cta * (size_t)n_ctas);
    }

    // convexity-weight search, all objects' rounds together
    // (period_search_BOINC.cpp:646-770, start_CUDA.cu:400-789)
    std::vector<double> conw(n_obj);
    std::vector<int> new_conw(n_obj, 0);
    for (int i = 0; i < n_obj; ++i) conw[i] = objs[i].conw_r;
    std::vector<psb::FitItem> test_items;
    for (int n = 1; n <= kTestPeriods; ++n)
        for (int pl = 0; pl < PS_N_POLES; ++pl) test_items.push_back(psb::FitItem{n, pl});
    for (;;) {
        std::vector<std::pair<int, std::vector<psb::FitItem>>> jobs;
        for (int i = 0; i < n_obj; ++i) {
            if (new_conw[i] == 1 || !(conw[i] * objs[i].escl * objs[i].escl < 10.0)) continue;
            const double rms_w = (quirks & PS_QUIRK_PRECALC_CONW) ? 0.0 : conw[i];
            ps_status st = configure(b.h[i], objs[i], conw[i], rms_w);
            if (st != PS_OK) return st;
            jobs.emplace_back(i, test_items);
        }
        if (jobs.empty()) break;
        std::vector<std::vector<psb::FitOut>> res;
        ps_status st = run_jobs(b, slot_of, jobs, res);
        if (st != PS_OK) return st;
        for (size_t k = 0; k < jobs.size(); ++k) {
            const int i = jobs[k].first;
            double sum_dark = 0.0;
            for (int t = 0; t < kTestPeriods; ++t)
                sum_dark = sum_dark + res[k][t * PS_N_POLES + psb_best_pole(&res[k][t * PS_N_POLES])].dark;
            const double ave = sum_dark / kTestPeriods;
            if (ave < 1.0) new_conw[i] = 1;
            if (ave >= 1.0) conw[i] = conw[i] * 2;
        }
    }

    // the scans (start_CUDA.cu:792-1245)
    std::vector<std::pair<int, std::vector<psb::FitItem>>> jobs;
    for (int i = 0; i < n_obj; ++i) {
        conw_r_out[i] = conw[i];
        ps_status st = configure(b.h[i], objs[i], conw[i], conw[i]);
        if (st != PS_OK) return st;
        std::vector<psb::FitItem> items;
        const int nl = scan_lines(objs[i]);
        items.reserve((size_t)nl * PS_N_POLES);
        for (int q = 0; q < nl; ++q)
            for (int pl = 0; pl < PS_N_POLES; ++pl) items.push_back(psb::FitItem{objs[i].n_start_from + q, pl});
        jobs.emplace_back(i, std::move(items));
    }
    std::vector<std::vector<psb::FitOut>> res;
    ps_status st = run_jobs(b, slot_of, jobs, res);
    if (st != PS_OK) return st;
    for (int i = 0; i < n_obj; ++i) {
        const ps_object &o = objs[i];
        const int nl = scan_lines(o);
        ps_line *out = lines + line_offset[i];
        for (int q = 0; q < nl; ++q) {
            const psb::FitOut *r = &res[i][(size_t)q * PS_N_POLES];
            const psb::FitOut &bp = r[psb_best_pole(r)];
            ps_line &L = out[q];
            L.period_h = 24 * bp.per;
            L.rms = bp.dev;
            L.chisq = bp.dev * bp.dev * o.ndata;
            L.dark = (o.n_start_from + q == 1) ? conw[i] * o.escl * o.escl : bp.dark;
            L.lambda_deg = bp.lambda_deg;
            L.beta_deg = bp.beta_deg;
        }
        n_lines[i] = nl;
    }
    return PS_OK;
}
