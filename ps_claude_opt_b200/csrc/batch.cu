// batch.cu -- ps_gpu_scan_batch: the convexity-weight search and the period
// scan of many objects on one GPU.
//
// The reference runs one object per process (period_search_BOINC.cpp:
// 638-872): a convexity-weight search of 100 fits per round
// (start_CUDA.cu:400-789) -- too few to fill 148 SMs -- and then the scan.
// Here the objects are grouped by padded coefficient count (one kernel
// instance each) and every group runs as ONE persistent launch whose device
// queue holds the (frequency, pole) items of all its objects: an item's pole
// field carries its object, and a CTA reloads the object's facet table when
// its next item belongs to another object (items are ordered by object, so
// that is rare).  Ragged iteration counts and uneven object sizes even out
// across the CTAs.  Each search round launches every group once with the
// items of the objects still searching; the scan launches of all groups are
// captured into one CUDA graph (a fork over the groups' streams and a join)
// and replayed.  The groups' launches run concurrently on their streams.
//
// Two scheduling choices are made per group:
//  * the tile layout (rows per J^T W J tile: 32, which allows the k-slice
//    mode, or 16; per-curve statistics in shared memory or in the scratch
//    slab) is picked by a small autotuner: every layout that fits in shared
//    memory is timed on a one-wave sample of the group's own items cut to
//    three LM iterations, and the fastest is kept for the group's shape
//    (cached per process); ps_batch_set_tuning(0) takes the first layout that
//    fits instead;
//  * items go into the queue largest object first (longest-processing-time
//    order by an estimate of the per-fit cost), so the most expensive fits
//    start early and the launch's tail is made of short ones.
// Neither choice changes a result: every fit runs the same arithmetic.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <numeric>
#include <string>
#include <tuple>
#include <vector>

#include "engine.h"
#include "handle.h"
#include "ps_b200.h"
#include "util.h"

namespace {

constexpr int kTestPeriods = 10;  // start_CUDA.cu:420
constexpr int kTuneIterations = 3; // LM iterations of a tuning sample fit

// Tile layouts in order of preference: {rows per J^T W J tile, per-curve
// statistics in shared memory}.
constexpr int kLayouts[4][2] = {{32, 1}, {32, 0}, {16, 1}, {16, 0}};

struct Tuning {
    std::mutex mu;
    int mode = 1;                                            // 1 autotune, 0 first layout that fits
    std::map<std::tuple<int, int, int, int, int>, int> cache;  // group shape -> layout index
    std::string report = "[]";                               // JSON of the last ps_gpu_scan_batch
};
Tuning &tuning()
{
    static Tuning t;
    return t;
}

struct Group {
    int ncp = 0;
    std::vector<int> members;          // object indices
    std::vector<int> order;            // member positions, most expensive object first
    psb::DevObject env{};              // largest sizes: the shared-memory layout
    size_t per_cta = 0;                // scratch doubles of one CTA (largest object)
    int ctas = 0;                      // resident CTAs of the batch kernel
    cudaStream_t stream = nullptr;
    cudaEvent_t join = nullptr;
    psb::DevBuf<psb::DevObject> objs;
    psb::DevBuf<psb::DevParams> prms;
    psb::DevBuf<psb::FitItem> items;
    psb::DevBuf<psb::FitOut> out;
    psb::DevBuf<double> scratch;
    psb::DevBuf<int> queue, status;
};

struct Batch {
    std::vector<ps_gpu *> h;
    std::vector<Group> groups;
    cudaStream_t origin = nullptr;
    cudaEvent_t fork = nullptr;
    ~Batch()
    {
        for (Group &g : groups) {
            if (g.stream) cudaStreamSynchronize(g.stream);
            g.objs.release();
            g.prms.release();
            g.items.release();
            g.out.release();
            g.scratch.release();
            g.queue.release();
            g.status.release();
            if (g.join) cudaEventDestroy(g.join);
            if (g.stream) cudaStreamDestroy(g.stream);
        }
        if (fork) cudaEventDestroy(fork);
        if (origin) cudaStreamDestroy(origin);
        for (ps_gpu *x : h) ps_gpu_unprepare(x);
    }
};

ps_status configure(ps_gpu *h, const ps_object &o, double conw_r, double conw_r_rms)
{
    return ps_gpu_configure(h, o.freq_start, o.freq_step, o.stop_condition, o.n_iter_min, conw_r, conw_r_rms,
                            o.ndata, o.ia, o.ia_par, o.cg_first, o.sig, o.sigr2, o.numfac, o.brightness, &o.curves,
                            &o.shape);
}

int scan_lines(const ps_object &o)
{
    const int n_max = (int)((o.freq_start - o.freq_end) / o.freq_step) + 1;
    return std::max(0, std::min(n_max - o.n_start_from + 1, (int)o.max_lines));
}

// Estimated FP64 work of one LM evaluation of an object (the facet sweep,
// the J^T W J update and the pseudo-points): the key of the queue order.
double eval_cost(const psb::DevObject &o)
{
    const double nf = o.n_fac, nc = o.n_coef, mf = o.mfit;
    return o.n_points * (10.0 * nf + 0.45 * nf * (60.0 + 2.0 * nc) + mf * (mf + 1.0)) + 8.0 * nf * nc;
}

// The group's objects (their current constants) to the device.  iter_cap > 0
// cuts every fit to that many LM iterations (tuning samples).
ps_status upload_objects(Batch &b, Group &g, int iter_cap = 0)
{
    std::vector<psb::DevObject> objs;
    std::vector<psb::DevParams> prms;
    for (int i : g.members) {
        psb::DevObject o = b.h[i]->obj;
        o.tile_rows = g.env.tile_rows;
        o.cstat_smem = g.env.cstat_smem;
        objs.push_back(o);
        psb::DevParams p = b.h[i]->prm;
        p.phase_cycles = nullptr;
        if (iter_cap > 0) {
            p.n_iter_max = iter_cap;
            p.iter_diff_max = 0;
            p.n_iter_min = 0;
        }
        prms.push_back(p);
    }
    PSB_CUDA(psb::upload(g.objs, objs, g.stream));
    PSB_CUDA(psb::upload(g.prms, prms, g.stream));
    return PS_OK;
}

// Device time of one launch of the tuning sample (one wave of the group's
// first items, round-robin over its objects, kTuneIterations iterations
// each) under the layout now in g.env.
ps_status time_layout(Batch &b, Group &g, float *ms)
{
    PSB_CUDA(cudaStreamSynchronize(g.stream));
    ps_status st = upload_objects(b, g, kTuneIterations);
    if (st != PS_OK) return st;
    std::vector<psb::FitItem> sample;
    for (int q = 0; (int)sample.size() < g.ctas && q < 64 * PS_N_POLES; ++q)
        for (size_t k = 0; k < g.members.size() && (int)sample.size() < g.ctas; ++k)
            sample.push_back(psb::FitItem{1 + q / PS_N_POLES, (q % PS_N_POLES) | (int)k << 8});
    PSB_CUDA(psb::upload(g.items, sample, g.stream));
    PSB_CUDA(g.out.ensure(sample.size()));
    PSB_CUDA(g.scratch.ensure(g.per_cta * sample.size()));
    PSB_CUDA(g.queue.ensure(1));
    PSB_CUDA(g.status.ensure(1));
    PSB_CUDA(cudaMemsetAsync(g.status.ptr, 0, sizeof(int), g.stream));
    PSB_CUDA(cudaMemsetAsync(g.queue.ptr, 0, sizeof(int), g.stream));
    const int e = psb::prepare_batch_kernel(g.env);
    if (e) return psb_fail_cuda(e, "ps_gpu_scan_batch: kernel attributes");
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    PSB_CUDA(cudaEventCreate(&t0));
    PSB_CUDA(cudaEventCreate(&t1));
    cudaError_t ce = cudaEventRecord(t0, g.stream);
    int le = 0;
    if (ce == cudaSuccess)
        le = psb::launch_fits_batch(g.env, g.objs.ptr, g.prms.ptr, g.items.ptr, (int)sample.size(), g.queue.ptr,
                                    g.out.ptr, g.scratch.ptr, g.per_cta, (int)sample.size(), g.status.ptr, g.stream);
    if (ce == cudaSuccess && !le) ce = cudaEventRecord(t1, g.stream);
    if (ce == cudaSuccess && !le) ce = cudaEventSynchronize(t1);
    if (ce == cudaSuccess && !le) ce = cudaEventElapsedTime(ms, t0, t1);
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    if (le) return psb_fail_cuda(le, "ps_gpu_scan_batch: tuning launch");
    if (ce != cudaSuccess) return psb_fail_cuda(ce, "ps_gpu_scan_batch: tuning timing");
    return PS_OK;
}

// Shared-memory layout of a group: the largest sizes of its objects and a
// tile layout that fits (beside the kernel's static object copy) -- the
// autotuner's pick, or the first that fits.  Appends the group's entry to
// the JSON report.
ps_status plan_group(Batch &b, Group &g, size_t smem_limit, std::string &report)
{
    psb::DevObject &e = g.env;
    e = b.h[g.members[0]]->obj;
    for (int i : g.members) {
        const psb::DevObject &o = b.h[i]->obj;
        e.n_fac = std::max(e.n_fac, o.n_fac);
        e.mfit = std::max(e.mfit, o.mfit);
        e.n_curves = std::max(e.n_curves, o.n_curves);
        e.row_stride = std::max(e.row_stride, o.row_stride);
        e.ma = std::max(e.ma, o.ma);
    }
    std::vector<int> fits;
    for (int l = 0; l < 4; ++l)
        if (psb::fit_smem_bytes(e.n_fac, e.mfit, e.ncp, e.n_curves, e.row_stride, kLayouts[l][0], kLayouts[l][1], 0) +
                1024 <= smem_limit)
            fits.push_back(l);
    if (fits.empty()) return psb_fail(PS_ERR_ARG, "ps_gpu_scan_batch: objects too large for shared memory");
    g.per_cta = 0;
    for (int i : g.members) g.per_cta = std::max(g.per_cta, psb::fit_scratch_doubles(b.h[i]->obj));
    // queue order: most expensive object first, ties by position
    g.order.resize(g.members.size());
    std::iota(g.order.begin(), g.order.end(), 0);
    std::stable_sort(g.order.begin(), g.order.end(), [&](int x, int y) {
        return eval_cost(b.h[g.members[x]]->obj) > eval_cost(b.h[g.members[y]]->obj);
    });

    auto set_layout = [&](int l) -> ps_status {
        e.tile_rows = kLayouts[l][0];
        e.cstat_smem = kLayouts[l][1];
        const int per_sm = psb::fit_batch_ctas_per_sm(e);
        if (per_sm < 1) return psb_fail(PS_ERR_CUDA, "ps_gpu_scan_batch: batch kernel cannot be resident");
        g.ctas = per_sm * b.h[g.members[0]]->n_sm;
        return PS_OK;
    };
    Tuning &t = tuning();
    int mode;
    {
        std::lock_guard<std::mutex> lk(t.mu);
        mode = t.mode;
    }
    const auto key = std::make_tuple(e.ncp, e.n_fac, e.mfit, e.n_curves, e.row_stride);
    int chosen = fits[0];
    const char *source = "only layout that fits";
    std::vector<float> ms(fits.size(), -1.0f);
    if (fits.size() > 1 && mode == 0) {
        source = "first that fits";
    } else if (fits.size() > 1) {
        bool cached = false;
        {
            std::lock_guard<std::mutex> lk(t.mu);
            auto it = t.cache.find(key);
            if (it != t.cache.end()) {
                chosen = it->second;
                cached = true;
            }
        }
        source = "cache";
        if (!cached) {
            source = "timed";
            float best = 0;
            for (size_t c = 0; c < fits.size(); ++c) {
                ps_status st = set_layout(fits[c]);
                if (st == PS_OK) st = time_layout(b, g, &ms[c]);
                if (st != PS_OK) return st;
                if (c == 0 || ms[c] < best) {
                    best = ms[c];
                    chosen = fits[c];
                }
            }
            std::lock_guard<std::mutex> lk(t.mu);
            t.cache[key] = chosen;
        }
    }
    ps_status st = set_layout(chosen);
    if (st != PS_OK) return st;
    char buf[256];
    std::snprintf(buf, sizeof buf,
                  "%s{\"ncp\": %d, \"objects\": %zu, \"n_fac\": %d, \"mfit\": %d, \"ctas\": %d, \"source\": \"%s\", "
                  "\"chosen\": {\"tile_rows\": %d, \"cstat_smem\": %d}, \"candidates\": [",
                  report.size() > 1 ? ", " : "", e.ncp, g.members.size(), e.n_fac, e.mfit, g.ctas, source,
                  kLayouts[chosen][0], kLayouts[chosen][1]);
    report += buf;
    for (size_t c = 0; c < fits.size(); ++c) {
        std::snprintf(buf, sizeof buf, "%s{\"tile_rows\": %d, \"cstat_smem\": %d, \"sample_ms\": %.4f}",
                      c ? ", " : "", kLayouts[fits[c]][0], kLayouts[fits[c]][1], (double)ms[c]);
        report += buf;
    }
    report += "]}";
    return PS_OK;
}

// Items of one launch per group: for member k of group g, items[k] (n_freq,
// pole) pairs.  Uploads, launches (captured into a graph when `graph`), and
// returns each member's results.
ps_status run_groups(Batch &b, const std::vector<std::vector<std::vector<psb::FitItem>>> &items, bool graph,
                     std::vector<std::vector<std::vector<psb::FitOut>>> &res)
{
    res.assign(b.groups.size(), {});
    std::vector<std::vector<int>> offset(b.groups.size());
    std::vector<int> total(b.groups.size(), 0);
    for (size_t gi = 0; gi < b.groups.size(); ++gi) {
        Group &g = b.groups[gi];
        std::vector<psb::FitItem> flat;
        offset[gi].assign(g.members.size(), 0);
        for (int k : g.order) {
            offset[gi][k] = (int)flat.size();
            for (psb::FitItem it : items[gi][k]) {
                it.pole |= k << 8;
                flat.push_back(it);
            }
        }
        total[gi] = (int)flat.size();
        if (flat.empty()) continue;
        PSB_CUDA(psb::upload(g.items, flat, g.stream));
        PSB_CUDA(g.out.ensure(flat.size()));
        PSB_CUDA(g.scratch.ensure(g.per_cta * (size_t)std::min(g.ctas, total[gi])));
        PSB_CUDA(g.queue.ensure(1));
        if (!g.status.ptr) {
            PSB_CUDA(g.status.ensure(1));
            PSB_CUDA(cudaMemsetAsync(g.status.ptr, 0, sizeof(int), g.stream));
        }
        PSB_CUDA(cudaStreamSynchronize(g.stream));  // uploads done before any capture
        const int e = psb::prepare_batch_kernel(g.env);
        if (e) return psb_fail_cuda(e, "ps_gpu_scan_batch: kernel attributes");
    }
    auto enqueue = [&](size_t gi) -> ps_status {
        Group &g = b.groups[gi];
        PSB_CUDA(cudaMemsetAsync(g.queue.ptr, 0, sizeof(int), g.stream));
        const int e = psb::launch_fits_batch(g.env, g.objs.ptr, g.prms.ptr, g.items.ptr, total[gi], g.queue.ptr,
                                             g.out.ptr, g.scratch.ptr, g.per_cta, std::min(g.ctas, total[gi]),
                                             g.status.ptr, g.stream);
        if (e) return psb_fail_cuda(e, "ps_gpu_scan_batch: fit kernel launch");
        return PS_OK;
    };
    if (graph) {
        cudaGraph_t gr = nullptr;
        cudaGraphExec_t ex = nullptr;
        PSB_CUDA(cudaStreamBeginCapture(b.origin, cudaStreamCaptureModeThreadLocal));
        ps_status st = PS_OK;
        cudaError_t ce = cudaEventRecord(b.fork, b.origin);
        for (size_t gi = 0; gi < b.groups.size() && st == PS_OK && ce == cudaSuccess; ++gi) {
            if (!total[gi]) continue;
            Group &g = b.groups[gi];
            ce = cudaStreamWaitEvent(g.stream, b.fork, 0);
            if (ce == cudaSuccess) st = enqueue(gi);
            if (st == PS_OK && ce == cudaSuccess) ce = cudaEventRecord(g.join, g.stream);
            if (st == PS_OK && ce == cudaSuccess) ce = cudaStreamWaitEvent(b.origin, g.join, 0);
        }
        const cudaError_t ee = cudaStreamEndCapture(b.origin, &gr);
        if (st != PS_OK) {
            if (gr) cudaGraphDestroy(gr);
            return st;
        }
        if (ce != cudaSuccess || ee != cudaSuccess) {
            if (gr) cudaGraphDestroy(gr);
            return psb_fail_cuda(ce != cudaSuccess ? ce : ee, "ps_gpu_scan_batch: graph capture");
        }
        ce = cudaGraphInstantiate(&ex, gr, 0);
        if (ce == cudaSuccess) ce = cudaGraphLaunch(ex, b.origin);
        if (ce == cudaSuccess) ce = cudaStreamSynchronize(b.origin);
        if (ex) cudaGraphExecDestroy(ex);
        cudaGraphDestroy(gr);
        if (ce != cudaSuccess) return psb_fail_cuda(ce, "ps_gpu_scan_batch: graph launch");
    } else {
        for (size_t gi = 0; gi < b.groups.size(); ++gi) {
            if (!total[gi]) continue;
            ps_status st = enqueue(gi);
            if (st != PS_OK) return st;
        }
        for (Group &g : b.groups) PSB_CUDA(cudaStreamSynchronize(g.stream));
    }
    for (size_t gi = 0; gi < b.groups.size(); ++gi) {
        Group &g = b.groups[gi];
        std::vector<psb::FitOut> all(total[gi]);
        if (total[gi])
            PSB_CUDA(cudaMemcpy(all.data(), g.out.ptr, sizeof(psb::FitOut) * total[gi], cudaMemcpyDeviceToHost));
        res[gi].resize(g.members.size());
        for (size_t k = 0; k < g.members.size(); ++k) {
            const int n = (int)items[gi][k].size();
            res[gi][k].assign(all.begin() + offset[gi][k], all.begin() + offset[gi][k] + n);
        }
    }
    return PS_OK;
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
        // a first configure validates the object and builds its device tables
        st = configure(b.h[i], o, o.conw_r, o.conw_r);
        if (st != PS_OK) return st;
    }
    PSB_CUDA(cudaSetDevice(device));
    cudaDeviceProp prop;
    PSB_CUDA(cudaGetDeviceProperties(&prop, device));
    PSB_CUDA(cudaStreamCreateWithFlags(&b.origin, cudaStreamNonBlocking));
    PSB_CUDA(cudaEventCreateWithFlags(&b.fork, cudaEventDisableTiming));
    std::map<int, int> by_ncp;
    for (int i = 0; i < n_obj; ++i) {
        const int ncp = b.h[i]->obj.ncp;
        if (!by_ncp.count(ncp)) {
            by_ncp[ncp] = (int)b.groups.size();
            b.groups.emplace_back();
            b.groups.back().ncp = ncp;
        }
        b.groups[by_ncp[ncp]].members.push_back(i);
    }
    std::string report = "[";
    for (Group &g : b.groups) {
        PSB_CUDA(cudaStreamCreateWithFlags(&g.stream, cudaStreamNonBlocking));
        PSB_CUDA(cudaEventCreateWithFlags(&g.join, cudaEventDisableTiming));
        ps_status st = plan_group(b, g, prop.sharedMemPerBlockOptin, report);
        if (st != PS_OK) return st;
    }
    report += "]";
    {
        std::lock_guard<std::mutex> lk(tuning().mu);
        tuning().report = report;
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
        bool any = false;
        std::vector<std::vector<std::vector<psb::FitItem>>> items(b.groups.size());
        for (size_t gi = 0; gi < b.groups.size(); ++gi) {
            Group &g = b.groups[gi];
            items[gi].resize(g.members.size());
            for (size_t k = 0; k < g.members.size(); ++k) {
                const int i = g.members[k];
                if (new_conw[i] == 1 || !(conw[i] * objs[i].escl * objs[i].escl < 10.0)) continue;
                const double rms_w = (quirks & PS_QUIRK_PRECALC_CONW) ? 0.0 : conw[i];
                ps_status st = configure(b.h[i], objs[i], conw[i], rms_w);
                if (st != PS_OK) return st;
                items[gi][k] = test_items;
                any = true;
            }
            ps_status st = upload_objects(b, g);
            if (st != PS_OK) return st;
        }
        if (!any) break;
        std::vector<std::vector<std::vector<psb::FitOut>>> res;
        ps_status st = run_groups(b, items, false, res);
        if (st != PS_OK) return st;
        for (size_t gi = 0; gi < b.groups.size(); ++gi)
            for (size_t k = 0; k < b.groups[gi].members.size(); ++k) {
                if (items[gi][k].empty()) continue;
                const int i = b.groups[gi].members[k];
                const std::vector<psb::FitOut> &r = res[gi][k];
                double sum_dark = 0.0;
                for (int t = 0; t < kTestPeriods; ++t)
                    sum_dark = sum_dark + r[t * PS_N_POLES + psb_best_pole(&r[t * PS_N_POLES])].dark;
                const double ave = sum_dark / kTestPeriods;
                if (ave < 1.0) new_conw[i] = 1;
                if (ave >= 1.0) conw[i] = conw[i] * 2;
            }
    }

    // the scans (start_CUDA.cu:792-1245), one graph over all groups
    std::vector<std::vector<std::vector<psb::FitItem>>> items(b.groups.size());
    for (size_t gi = 0; gi < b.groups.size(); ++gi) {
        Group &g = b.groups[gi];
        items[gi].resize(g.members.size());
        for (size_t k = 0; k < g.members.size(); ++k) {
            const int i = g.members[k];
            conw_r_out[i] = conw[i];
            ps_status st = configure(b.h[i], objs[i], conw[i], conw[i]);
            if (st != PS_OK) return st;
            const int nl = scan_lines(objs[i]);
            items[gi][k].reserve((size_t)nl * PS_N_POLES);
            for (int q = 0; q < nl; ++q)
                for (int pl = 0; pl < PS_N_POLES; ++pl)
                    items[gi][k].push_back(psb::FitItem{objs[i].n_start_from + q, pl});
        }
        ps_status st = upload_objects(b, g);
        if (st != PS_OK) return st;
    }
    std::vector<std::vector<std::vector<psb::FitOut>>> res;
    ps_status st = run_groups(b, items, true, res);
    if (st != PS_OK) return st;
    for (size_t gi = 0; gi < b.groups.size(); ++gi)
        for (size_t k = 0; k < b.groups[gi].members.size(); ++k) {
            const int i = b.groups[gi].members[k];
            const ps_object &o = objs[i];
            const int nl = scan_lines(o);
            ps_line *out = lines + line_offset[i];
            for (int q = 0; q < nl; ++q) {
                const psb::FitOut *r = &res[gi][k][(size_t)q * PS_N_POLES];
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

extern "C" ps_status ps_batch_set_tuning(int32_t mode)
{
    if (mode < 0 || mode > 2) return psb_fail(PS_ERR_ARG, "ps_batch_set_tuning: mode must be 0, 1 or 2");
    std::lock_guard<std::mutex> lk(tuning().mu);
    tuning().mode = mode == 0 ? 0 : 1;
    if (mode == 2) tuning().cache.clear();
    return PS_OK;
}

extern "C" int32_t ps_batch_tuning_report(char *buf, int32_t len)
{
    std::lock_guard<std::mutex> lk(tuning().mu);
    const std::string &r = tuning().report;
    if (buf && len > 0) {
        const size_t n = std::min(r.size(), (size_t)len - 1);
        std::memcpy(buf, r.data(), n);
        buf[n] = 0;
    }
    return (int32_t)r.size();
}
