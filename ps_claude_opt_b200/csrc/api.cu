// api.cu -- C ABI of the fit engine (include/ps_b200.h).
//
// Host orchestration that replaces start_CUDA.cu: object upload, the work
// list of (frequency, pole) items, one persistent-kernel launch per chunk of
// the scan, and the best-pole reduction into output lines.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "engine.h"
#include "handle.h"
#include "ps_b200.h"
#include "util.h"

namespace {

thread_local std::string g_last_error;

}  // namespace

ps_status psb_fail(ps_status code, const char *msg)
{
    g_last_error = msg ? msg : "";
    return code;
}

ps_status psb_fail_cuda(int cuda_error, const char *what)
{
    g_last_error = std::string(what) + ": " + cudaGetErrorString((cudaError_t)cuda_error);
    return PS_ERR_CUDA;
}

extern "C" const char *ps_last_error(void) { return g_last_error.c_str(); }
extern "C" const char *ps_version(void) { return "ps-b200 0.1 (sm_100a FP64 persistent LM)"; }

extern "C" ps_status ps_gpu_prepare(int32_t device, const double *beta_pole, const double *lambda_pole,
                                    const double *par, double cl, double alamda_start, double alamda_incr,
                                    double alamda_incrr, const double *ee, const double *ee0, const double *tim,
                                    double phi0, int32_t ndata, const double *weight, ps_gpu **handle)
{
    if (!handle || !beta_pole || !lambda_pole || !par || !ee || !ee0 || !tim || !weight || ndata <= 0)
        return psb_fail(PS_ERR_ARG, "ps_gpu_prepare: null argument or ndata <= 0");
    if (!(cl > 0)) return psb_fail(PS_ERR_ARG, "ps_gpu_prepare: Lambert coefficient must be > 0");
    *handle = nullptr;
    int ndev = 0;
    PSB_CUDA(cudaGetDeviceCount(&ndev));
    if (device < 0 || device >= ndev) return psb_fail(PS_ERR_ARG, "ps_gpu_prepare: no such CUDA device");
    PSB_CUDA(cudaSetDevice(device));
    cudaDeviceProp prop;
    PSB_CUDA(cudaGetDeviceProperties(&prop, device));
    ps_gpu *h = new ps_gpu();
    h->device = device;
    h->n_sm = prop.multiProcessorCount;
    cudaError_t e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete h;
        return psb_fail_cuda(e, "cudaStreamCreateWithFlags");
    }
    h->ndata = ndata;
    h->tim.assign(tim, tim + ndata);
    h->ee.assign(ee, ee + 3 * (size_t)ndata);
    h->ee0.assign(ee0, ee0 + 3 * (size_t)ndata);
    h->weight.assign(weight, weight + ndata);
    for (int i = 0; i < PS_N_POLES; ++i) {
        h->beta_pole[i] = beta_pole[i];
        h->lambda_pole[i] = lambda_pole[i];
    }
    for (int i = 0; i < 3; ++i) h->par[i] = par[i];
    h->lcl = std::log(cl);
    h->alamda_start = alamda_start;
    h->alamda_incr = alamda_incr;
    h->alamda_incrr = alamda_incrr;
    h->phi0 = phi0;
    *handle = h;
    return PS_OK;
}

extern "C" void ps_gpu_unprepare(ps_gpu *h)
{
    if (!h) return;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    h->facet.release(); h->pt_a.release(); h->pt_b.release(); h->pt_rec.release();
    h->ysh.release(); h->ysh32.release(); h->pt_w.release(); h->curve_sig.release(); h->cg_first.release();
    h->scratch.release(); h->eval_buf.release();
    h->pt_curve.release(); h->curve_start.release(); h->curve_rel.release(); h->fidx.release();
    h->queue.release(); h->status.release(); h->items.release(); h->out.release(); h->phase.release();
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
}

extern "C" ps_status ps_gpu_set_quirks(ps_gpu *h, int32_t quirks)
{
    if (!h) return psb_fail(PS_ERR_NOT_PREPARED, "ps_gpu_set_quirks: null handle");
    h->quirks = quirks;
    return PS_OK;
}

extern "C" void *ps_gpu_stream(ps_gpu *h) { return h ? (void *)h->stream : nullptr; }

extern "C" ps_status ps_gpu_set_precision(ps_gpu *h, int32_t precision)
{
    if (!h) return psb_fail(PS_ERR_NOT_PREPARED, "ps_gpu_set_precision: null handle");
    if (precision != PS_PRECISION_FP64 && precision != PS_PRECISION_MIXED)
        return psb_fail(PS_ERR_ARG, "ps_gpu_set_precision: unknown precision");
    h->precision = precision;
    h->configured = false;  // takes effect at the next configure
    return PS_OK;
}

// Rounds x to the nearest TF32 value (10 explicit mantissa bits, ties to
// even); finite inputs only.
static float tf32_round(float x)
{
    uint32_t u;
    std::memcpy(&u, &x, 4);
    const uint32_t lsb = (u >> 13) & 1u;
    u = (u + 0x0fffu + lsb) & ~0x1fffu;
    float r;
    std::memcpy(&r, &u, 4);
    return r;
}


extern "C" ps_status ps_gpu_configure(ps_gpu *h, double freq_start, double freq_step, double stop_condition,
                                      int32_t n_iter_min, double conw_r, double conw_r_rms, int32_t ndata,
                                      const int32_t *ia, const int32_t *ia_par, const double *cg_first,
                                      const double *sig, const double *sigr2, int32_t numfac,
                                      const double *brightness, const ps_curves *curves, const ps_shape *shape)
{
    if (!h) return psb_fail(PS_ERR_NOT_PREPARED, "ps_gpu_configure: null handle");
    if (!ia || !ia_par || !cg_first || !sig || !sigr2 || !brightness || !curves || !shape ||
        !curves->curve_len || !curves->curve_rel || !shape->normal || !shape->d_area || !shape->d_sphere)
        return psb_fail(PS_ERR_ARG, "ps_gpu_configure: null argument");
    if (ndata != h->ndata) return psb_fail(PS_ERR_ARG, "ps_gpu_configure: ndata differs from ps_gpu_prepare");
    const int nc = shape->n_coef, ma = nc + 8;
    if (nc < 1 || ma > 89) return psb_fail(PS_ERR_ARG, "ps_gpu_configure: n_coef must be 1..81 (lmax <= 8)");
    if (numfac < 1 || numfac > PS_MAX_FAC) return psb_fail(PS_ERR_ARG, "ps_gpu_configure: numfac must be 1..1024");
    if (curves->n_curves < 1) return psb_fail(PS_ERR_ARG, "ps_gpu_configure: no lightcurves");
    long tot = 0;
    for (int c = 0; c < curves->n_curves; ++c) {
        if (curves->curve_len[c] < 1) return psb_fail(PS_ERR_ARG, "ps_gpu_configure: empty lightcurve");
        tot += curves->curve_len[c];
    }
    if (tot != ndata) return psb_fail(PS_ERR_ARG, "ps_gpu_configure: curve lengths do not sum to ndata");
    if (!(freq_step > 0)) return psb_fail(PS_ERR_ARG, "ps_gpu_configure: freq_step must be > 0");
    PSB_CUDA(cudaSetDevice(h->device));

    // fitted-parameter list; the phase-function flags come from ia_par as in
    // start_CUDA.cu:852-853
    std::vector<int> iav(ia, ia + ma + 1);
    for (int i = 0; i < 3; ++i) iav[nc + 4 + i] = ia_par[i];
    std::vector<int> fidx;
    for (int p = 1; p <= ma; ++p)
        if (iav[p]) fidx.push_back(p);
    const int mfit = (int)fidx.size();
    if (mfit < 1) return psb_fail(PS_ERR_ARG, "ps_gpu_configure: no fitted parameters");
    const int ncp = psb::padded_ncoef(nc);

    cudaDeviceProp prop;
    PSB_CUDA(cudaGetDeviceProperties(&prop, h->device));
    const int mixed = h->precision == PS_PRECISION_MIXED ? 1 : 0;
    if (mixed && ncp > psb::kMaxMixedNcp)
        return psb_fail(PS_ERR_ARG, "ps_gpu_configure: mixed precision is built for n_coef <= 64 (lmax <= 7)");
    // preferred layout first: 32-row tiles with the per-curve statistics in
    // shared memory; fall back for the largest models
    int tile_rows = 32, cstat_smem = 1;
    const int rs = (ma + 2) & ~1;
    size_t smem = psb::fit_smem_bytes(numfac, mfit, ncp, curves->n_curves, rs, tile_rows, cstat_smem, mixed);
    if (smem > prop.sharedMemPerBlockOptin) {
        cstat_smem = 0;
        smem = psb::fit_smem_bytes(numfac, mfit, ncp, curves->n_curves, rs, tile_rows, cstat_smem, mixed);
    }
    if (smem > prop.sharedMemPerBlockOptin) {
        tile_rows = 16;
        smem = psb::fit_smem_bytes(numfac, mfit, ncp, curves->n_curves, rs, tile_rows, cstat_smem, mixed);
    }
    if (smem > prop.sharedMemPerBlockOptin)
        return psb_fail(PS_ERR_ARG, "ps_gpu_configure: object too large for shared memory");

    std::vector<double4> facet(numfac);
    for (int f = 0; f < numfac; ++f)
        facet[f] = make_double4(shape->normal[3 * f], shape->normal[3 * f + 1], shape->normal[3 * f + 2],
                                shape->d_area[f]);
    std::vector<double> ysh((size_t)numfac * ncp, 0.0);
    for (int f = 0; f < numfac; ++f)
        for (int k = 0; k < nc; ++k) ysh[(size_t)f * ncp + k] = shape->d_sphere[(size_t)f * nc + k];
    // mixed precision: the basis as TF32 high and low parts, chunk by chunk
    // ([chunk][hi | lo][chunk facets][ncp], zero past the last facet)
    std::vector<float> ysh32;
    if (mixed) {
        const int fc = psb::chunk_facets_of(ncp), nch = (numfac + fc - 1) / fc;
        ysh32.assign((size_t)nch * 2 * fc * ncp, 0.0f);
        for (int f = 0; f < numfac; ++f) {
            const size_t base = (size_t)(f / fc) * 2 * fc * ncp + (size_t)(f % fc) * ncp;
            for (int k = 0; k < nc; ++k) {
                const double y = shape->d_sphere[(size_t)f * nc + k];
                const float hi = tf32_round((float)y);
                ysh32[base + k] = hi;
                ysh32[base + (size_t)fc * ncp + k] = tf32_round((float)(y - (double)hi));
            }
        }
    }
    std::vector<double4> pa(ndata), pb(ndata), prec(ndata);
    std::vector<double> pw(ndata);
    std::vector<int> pcur(ndata), cstart(curves->n_curves + 1), crel(curves->n_curves);
    std::vector<double> csig(curves->n_curves);
    int q = 0;
    for (int c = 0; c < curves->n_curves; ++c) {
        cstart[c] = q;
        crel[c] = curves->curve_rel[c] ? 1 : 0;
        csig[c] = sig[q];
        for (int j = 0; j < curves->curve_len[c]; ++j, ++q) {
            pa[q] = make_double4(h->tim[q], h->ee[3 * q], h->ee[3 * q + 1], h->ee[3 * q + 2]);
            pb[q] = make_double4(h->ee0[3 * q], h->ee0[3 * q + 1], h->ee0[3 * q + 2], brightness[q]);
            pw[q] = sigr2[q] * h->weight[q];
            pcur[q] = c;
            prec[q] = make_double4(brightness[q], pw[q], (double)c, (double)crel[c]);
        }
    }
    cstart[curves->n_curves] = q;
    std::vector<double> cgf(cg_first, cg_first + nc);

    cudaStream_t s = h->stream;
    PSB_CUDA(psb::upload(h->facet, facet, s));
    PSB_CUDA(psb::upload(h->ysh, ysh, s));
    if (mixed) PSB_CUDA(psb::upload(h->ysh32, ysh32, s));
    PSB_CUDA(psb::upload(h->pt_a, pa, s));
    PSB_CUDA(psb::upload(h->pt_b, pb, s));
    PSB_CUDA(psb::upload(h->pt_w, pw, s));
    PSB_CUDA(psb::upload(h->pt_rec, prec, s));
    PSB_CUDA(psb::upload(h->pt_curve, pcur, s));
    PSB_CUDA(psb::upload(h->curve_start, cstart, s));
    PSB_CUDA(psb::upload(h->curve_rel, crel, s));
    PSB_CUDA(psb::upload(h->curve_sig, csig, s));
    PSB_CUDA(psb::upload(h->fidx, fidx, s));
    PSB_CUDA(psb::upload(h->cg_first, cgf, s));
    PSB_CUDA(h->queue.ensure(1));
    if (!h->status.ptr) {
        PSB_CUDA(h->status.ensure(1));
        PSB_CUDA(cudaMemsetAsync(h->status.ptr, 0, sizeof(int), s));
    }
    PSB_CUDA(cudaStreamSynchronize(s));

    psb::DevObject &o = h->obj;
    o.n_points = ndata;
    o.n_curves = curves->n_curves;
    o.n_fac = numfac;
    o.n_coef = nc;
    o.ncp = ncp;
    o.ma = ma;
    o.mfit = mfit;
    o.row_stride = (ma + 1 + 1) & ~1;
    o.tile_rows = tile_rows;
    o.cstat_smem = cstat_smem;
    o.facet = h->facet.ptr;
    o.ysh = h->ysh.ptr;
    o.pt_a = h->pt_a.ptr;
    o.pt_b = h->pt_b.ptr;
    o.pt_w = h->pt_w.ptr;
    o.pt_rec = h->pt_rec.ptr;
    o.pt_curve = h->pt_curve.ptr;
    o.curve_start = h->curve_start.ptr;
    o.curve_rel = h->curve_rel.ptr;
    o.curve_sig = h->curve_sig.ptr;
    o.fidx = h->fidx.ptr;
    o.cg_first = h->cg_first.ptr;
    o.mixed = mixed;
    o.ysh32 = mixed ? h->ysh32.ptr : nullptr;

    psb::DevParams &p = h->prm;
    p.phi0 = h->phi0;
    for (int i = 0; i < 3; ++i) p.par[i] = h->par[i];
    p.lcl = h->lcl;
    p.alamda_start = h->alamda_start;
    p.alamda_incr = h->alamda_incr;
    p.alamda_incrr = h->alamda_incrr;
    for (int i = 0; i < PS_N_POLES; ++i) {
        p.beta_pole[i] = h->beta_pole[i];
        p.lambda_pole[i] = h->lambda_pole[i];
    }
    // stop condition (start_CUDA.cu:855-869)
    int n_iter_max = 0;
    double iter_diff_max = -1;
    if (stop_condition > 1) {
        n_iter_max = (int)stop_condition;
        iter_diff_max = 0;
        n_iter_min = 0;
    }
    if (stop_condition < 1) {
        n_iter_max = psb::kMaxIter;
        iter_diff_max = stop_condition;
    }
    p.n_iter_max = n_iter_max;
    p.n_iter_min = n_iter_min;
    p.iter_diff_max = iter_diff_max;
    p.conw_r = conw_r;
    p.conw_r_dev = conw_r_rms;
    p.freq_start = freq_start;
    p.freq_step = freq_step;
    p.phase_cycles = h->phase.ptr;

    h->ctas_per_sm = psb::fit_ctas_per_sm(o);
    if (h->ctas_per_sm < 1) return psb_fail(PS_ERR_CUDA, "ps_gpu_configure: fit kernel cannot be resident");
    h->scratch_per_cta = psb::fit_scratch_doubles(o);
    h->configured = true;
    return PS_OK;
}

extern "C" ps_status ps_gpu_occupancy(ps_gpu *h, int32_t *ctas_per_sm, int32_t *n_sm)
{
    if (!h || !h->configured) return psb_fail(PS_ERR_NOT_PREPARED, "ps_gpu_occupancy: not configured");
    if (ctas_per_sm) *ctas_per_sm = h->ctas_per_sm;
    if (n_sm) *n_sm = h->n_sm;
    return PS_OK;
}

// Enqueues the fit kernel over n device-resident items.
static ps_status enqueue_fits(ps_gpu *h, int n, const psb::FitItem *d_items, psb::FitOut *d_out)
{
    const int n_ctas = std::max(1, std::min(n, h->ctas_per_sm * h->n_sm));
    PSB_CUDA(h->scratch.ensure(h->scratch_per_cta * (size_t)n_ctas));
    PSB_CUDA(cudaMemsetAsync(h->queue.ptr, 0, sizeof(int), h->stream));
    int e = psb::launch_fits(h->obj, h->prm, d_items, n, h->queue.ptr, d_out, h->scratch.ptr, h->scratch_per_cta,
                             n_ctas, h->status.ptr, h->stream);
    if (e) return psb_fail_cuda(e, "fit kernel launch");
    return PS_OK;
}

extern "C" ps_status ps_gpu_fit_items_device(ps_gpu *h, int32_t n, const int32_t *d_items, ps_fit_result *d_out)
{
    if (!h || !h->configured) return psb_fail(PS_ERR_NOT_PREPARED, "ps_gpu_fit_items_device: not configured");
    if (n <= 0 || !d_items || !d_out) return psb_fail(PS_ERR_ARG, "ps_gpu_fit_items_device: bad arguments");
    static_assert(sizeof(psb::FitOut) == sizeof(ps_fit_result), "result layout");
    static_assert(sizeof(psb::FitItem) == 2 * sizeof(int32_t), "item layout");
    return enqueue_fits(h, n, reinterpret_cast<const psb::FitItem *>(d_items),
                        reinterpret_cast<psb::FitOut *>(d_out));
}

static ps_status run_items(ps_gpu *h, const std::vector<psb::FitItem> &items, std::vector<psb::FitOut> &res)
{
    const int n = (int)items.size();
    res.resize(n);
    if (n == 0) return PS_OK;
    PSB_CUDA(psb::upload(h->items, items, h->stream));
    PSB_CUDA(h->out.ensure(n));
    ps_status st = enqueue_fits(h, n, h->items.ptr, h->out.ptr);
    if (st != PS_OK) return st;
    PSB_CUDA(cudaMemcpyAsync(res.data(), h->out.ptr, n * sizeof(psb::FitOut), cudaMemcpyDeviceToHost, h->stream));
    PSB_CUDA(cudaStreamSynchronize(h->stream));
    return PS_OK;
}

extern "C" ps_status ps_gpu_fit_items(ps_gpu *h, int32_t n, const int32_t *n_freq, const int32_t *pole,
                                      ps_fit_result *out)
{
    if (!h || !h->configured) return psb_fail(PS_ERR_NOT_PREPARED, "ps_gpu_fit_items: not configured");
    if (n < 0 || (n > 0 && (!n_freq || !pole || !out))) return psb_fail(PS_ERR_ARG, "ps_gpu_fit_items: bad arguments");
    PSB_CUDA(cudaSetDevice(h->device));
    std::vector<psb::FitItem> items(n);
    for (int i = 0; i < n; ++i) {
        if (n_freq[i] < 1 || pole[i] < 0 || pole[i] >= PS_N_POLES)
            return psb_fail(PS_ERR_ARG, "ps_gpu_fit_items: frequency index < 1 or pole outside 0..9");
        items[i] = psb::FitItem{n_freq[i], pole[i]};
    }
    std::vector<psb::FitOut> res;
    ps_status st = run_items(h, items, res);
    if (st != PS_OK) return st;
    std::memcpy(out, res.data(), sizeof(ps_fit_result) * (size_t)n);
    return PS_OK;
}

extern "C" ps_status ps_gpu_eval(ps_gpu *h, const double *a, double *chisq, double *alpha, double *beta,
                                 double *area_sum)
{
    if (!h || !h->configured) return psb_fail(PS_ERR_NOT_PREPARED, "ps_gpu_eval: not configured");
    if (!a || !chisq || !alpha || !beta) return psb_fail(PS_ERR_ARG, "ps_gpu_eval: null argument");
    PSB_CUDA(cudaSetDevice(h->device));
    const int ma = h->obj.ma, mfit = h->obj.mfit;
    const size_t need = (size_t)(ma + 1) + (size_t)mfit * mfit + mfit + 2;
    PSB_CUDA(h->eval_buf.ensure(need));
    PSB_CUDA(h->scratch.ensure(h->scratch_per_cta));
    double *d_a = h->eval_buf.ptr;
    double *d_alpha = d_a + (ma + 1);
    double *d_beta = d_alpha + (size_t)mfit * mfit;
    double *d_chisq = d_beta + mfit;
    double *d_area = d_chisq + 1;
    PSB_CUDA(cudaMemcpyAsync(d_a, a, sizeof(double) * (ma + 1), cudaMemcpyHostToDevice, h->stream));
    psb::EvalOut ev{d_alpha, d_beta, d_chisq, d_area, d_a};
    int e = psb::launch_eval(h->obj, h->prm, ev, h->scratch.ptr, h->stream);
    if (e) return psb_fail_cuda(e, "eval kernel launch");
    std::vector<double> back(need - (ma + 1));
    PSB_CUDA(cudaMemcpyAsync(back.data(), d_alpha, back.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    PSB_CUDA(cudaStreamSynchronize(h->stream));
    std::memcpy(alpha, back.data(), sizeof(double) * (size_t)mfit * mfit);
    std::memcpy(beta, back.data() + (size_t)mfit * mfit, sizeof(double) * mfit);
    *chisq = back[(size_t)mfit * mfit + mfit];
    if (area_sum) *area_sum = back[(size_t)mfit * mfit + mfit + 1];
    return PS_OK;
}

extern "C" ps_status ps_gpu_phase_clocks(ps_gpu *h, int32_t enable, int64_t *out)
{
    if (!h) return psb_fail(PS_ERR_NOT_PREPARED, "ps_gpu_phase_clocks: null handle");
    PSB_CUDA(cudaSetDevice(h->device));
    if (out) {
        for (int i = 0; i < psb::kPhaseSlots; ++i) out[i] = 0;
        if (h->phase.ptr) {
            PSB_CUDA(cudaMemcpyAsync(out, h->phase.ptr, sizeof(int64_t) * psb::kPhaseSlots, cudaMemcpyDeviceToHost,
                                     h->stream));
            PSB_CUDA(cudaStreamSynchronize(h->stream));
        }
    }
    if (enable) {
        PSB_CUDA(h->phase.ensure(psb::kPhaseSlots));
        PSB_CUDA(cudaMemsetAsync(h->phase.ptr, 0, sizeof(unsigned long long) * psb::kPhaseSlots, h->stream));
        h->prm.phase_cycles = h->phase.ptr;
    } else {
        h->prm.phase_cycles = nullptr;
        h->phase.release();
    }
    return PS_OK;
}

extern "C" ps_status ps_gpu_status(ps_gpu *h, int32_t *flags)
{
    if (!h || !flags) return psb_fail(PS_ERR_ARG, "ps_gpu_status: null argument");
    *flags = 0;
    if (!h->status.ptr) return PS_OK;
    PSB_CUDA(cudaSetDevice(h->device));
    PSB_CUDA(cudaMemcpyAsync(flags, h->status.ptr, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    PSB_CUDA(cudaStreamSynchronize(h->stream));
    return PS_OK;
}

// Best pole of one frequency: NaN-safe, earliest pole wins ties
// (start_CUDA.cu:1200-1229).
int psb_best_pole(const psb::FitOut *r)
{
    int best = -1;
    for (int p = 0; p < PS_N_POLES; ++p)
        if (best < 0 || (!std::isnan(r[p].dev) && !(r[p].dev >= r[best].dev))) best = p;
    return best;
}

extern "C" ps_status ps_gpu_precalc(ps_gpu *h, double freq_start, double freq_end, double freq_step,
                                    double stop_condition, int32_t n_iter_min, double *conw_r, int32_t ndata,
                                    const int32_t *ia, const int32_t *ia_par, int32_t *new_conw,
                                    const double *cg_first, const double *sig, const double *sigr2, int32_t numfac,
                                    const double *brightness, const ps_curves *curves, const ps_shape *shape)
{
    (void)freq_end;
    if (!h) return psb_fail(PS_ERR_NOT_PREPARED, "ps_gpu_precalc: null handle");
    if (!conw_r || !new_conw) return psb_fail(PS_ERR_ARG, "ps_gpu_precalc: null argument");
    const double rms_w = (h->quirks & PS_QUIRK_PRECALC_CONW) ? 0.0 : *conw_r;
    ps_status st = ps_gpu_configure(h, freq_start, freq_step, stop_condition, n_iter_min, *conw_r, rms_w, ndata, ia,
                                    ia_par, cg_first, sig, sigr2, numfac, brightness, curves, shape);
    if (st != PS_OK) return st;
    const int max_test_periods = 10;  // start_CUDA.cu:420
    std::vector<psb::FitItem> items;
    for (int n = 1; n <= max_test_periods; ++n)
        for (int pl = 0; pl < PS_N_POLES; ++pl) items.push_back(psb::FitItem{n, pl});
    std::vector<psb::FitOut> res;
    st = run_items(h, items, res);
    if (st != PS_OK) return st;
    double sum_dark = 0.0;
    for (int t = 0; t < max_test_periods; ++t) sum_dark = sum_dark + res[t * PS_N_POLES + psb_best_pole(&res[t * PS_N_POLES])].dark;
    const double ave = sum_dark / max_test_periods;
    if (ave < 1.0) *new_conw = 1;
    if (ave >= 1.0) *conw_r = *conw_r * 2;
    return PS_OK;
}

extern "C" ps_status ps_gpu_start(ps_gpu *h, int32_t n_start_from, double freq_start, double freq_end,
                                  double freq_step, double stop_condition, int32_t n_iter_min, double conw_r,
                                  int32_t ndata, const int32_t *ia, const int32_t *ia_par, const double *cg_first,
                                  double escl, const double *sig, const double *sigr2, int32_t numfac,
                                  const double *brightness, const ps_curves *curves, const ps_shape *shape,
                                  ps_line *lines, int32_t max_lines, int32_t *n_lines, ps_progress_fn progress,
                                  void *user)
{
    if (!h) return psb_fail(PS_ERR_NOT_PREPARED, "ps_gpu_start: null handle");
    if (!lines || !n_lines || max_lines < 0) return psb_fail(PS_ERR_ARG, "ps_gpu_start: bad output arguments");
    *n_lines = 0;
    ps_status st = ps_gpu_configure(h, freq_start, freq_step, stop_condition, n_iter_min, conw_r, conw_r, ndata, ia,
                                    ia_par, cg_first, sig, sigr2, numfac, brightness, curves, shape);
    if (st != PS_OK) return st;
    const int n_max = (int)((freq_start - freq_end) / freq_step) + 1;
    if (n_start_from < 1) return psb_fail(PS_ERR_ARG, "ps_gpu_start: n_start_from < 1");
    int n_freq = std::min(n_max - n_start_from + 1, (int)max_lines);
    if (n_freq <= 0) return PS_OK;

    // chunks of frequencies: one persistent launch each; with a progress
    // callback about 20 chunks, each still several waves of CTAs
    const int resident = h->ctas_per_sm * h->n_sm;
    int chunk = n_freq;
    if (progress) chunk = std::max((2 * resident + PS_N_POLES - 1) / PS_N_POLES, (n_freq + 19) / 20);
    std::vector<psb::FitOut> res;
    for (int f0 = 0; f0 < n_freq; f0 += chunk) {
        const int nf = std::min(chunk, n_freq - f0);
        std::vector<psb::FitItem> items;
        items.reserve((size_t)nf * PS_N_POLES);
        for (int q = 0; q < nf; ++q)
            for (int pl = 0; pl < PS_N_POLES; ++pl) items.push_back(psb::FitItem{n_start_from + f0 + q, pl});
        st = run_items(h, items, res);
        if (st != PS_OK) return st;
        for (int q = 0; q < nf; ++q) {
            const psb::FitOut *r = &res[(size_t)q * PS_N_POLES];
            const psb::FitOut &b = r[psb_best_pole(r)];
            ps_line &L = lines[f0 + q];
            L.period_h = 24 * b.per;
            L.rms = b.dev;
            L.chisq = b.dev * b.dev * ndata;
            L.dark = (n_start_from + f0 + q == 1) ? conw_r * escl * escl : b.dark;
            L.lambda_deg = b.lambda_deg;
            L.beta_deg = b.beta_deg;
        }
        *n_lines = f0 + nf;
        if (progress && progress(user, f0 + nf, n_freq)) return psb_fail(PS_ERR_CANCELLED, "ps_gpu_start: cancelled");
    }
    return PS_OK;
}
