// noalloc.cu -- a fit entry point for callers that cannot allocate memory.
//
// Some hosts of this library run under an allocator they do not control: a
// framework whose caching allocator owns all device memory of the process
// (a cudaMalloc behind its back can fail on a full pool or fragment it), or a
// real-time pipeline that forbids allocation once it is running (cudaMalloc
// can synchronise the device and stall its other streams).  They cannot call
// cudaMalloc, so ps_gpu_prepare / ps_gpu_configure (which allocate device
// buffers) are closed to them.  ps_fit_items_noalloc runs the same persistent
// LM fit kernel as ps_gpu_fit_items, but every device byte it touches -- the
// object tables, the work items, the results, the queue and status words and
// the kernel's per-CTA scratch -- lives in one file-scope __device__ array of
// kNoAllocArenaBytes.  The caller passes host inputs and a host output array;
// the call allocates nothing, on the device or on the host heap.
//
// Contract (also in include/ps_b200.h):
//   * the arena is kNoAllocArenaBytes per device, reserved when this file's
//     module first loads on that device and held until the process exits.
//     CUDA loads modules lazily, so the reservation happens inside the first
//     call on the device, which may fail if the device is already full by
//     then; a call with n = 0 does only that (select the device, load the
//     module, look up the arena) and lets a caller reserve the arena at start
//     time, before its own allocator grows;
//   * every call looks up the arena's device address with the device current
//     (cudaGetSymbolAddress: cheap once the module is loaded, and never stale
//     after a cudaDeviceReset); the first call with work also sets the fit
//     kernel's shared-memory limit; make the first call before any stream
//     capture;
//   * every call reuses the arena and leaves the last call's contents there;
//     calls that overlap on the GPU (two host threads, or two streams) race
//     on it -- serialise them;
//   * an object whose tables plus one CTA's scratch exceed the arena is
//     rejected with PS_ERR_ARG; otherwise the grid is as many CTAs as the
//     remaining scratch holds (fewer than the resident maximum for large
//     objects, so slower than ps_gpu_fit_items, never different).
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>

#include "engine.h"
#include "ps_b200.h"
#include "util.h"

namespace {

constexpr size_t kNoAllocArenaBytes = size_t(64) << 20;  // 64 MiB
constexpr int kMaxDevices = 64;
constexpr int kMaxCurves = 200;   // the reference's MAX_LC (constants.h:10)
constexpr int kMaxIterCap = 60;   // constants.h:12

static __device__ __align__(256) unsigned char g_arena[kNoAllocArenaBytes];

// Device address of g_arena on the current device.  In host code g_arena
// names a host-side shadow, not device memory, so the kernels get this
// address.  Looked up on every call: cheap once the module is loaded, and a
// cached address would go stale if the host reset the device.
ps_status arena_address(unsigned char **out)
{
    void *ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&ptr, g_arena);
    if (e != cudaSuccess) return psb_fail_cuda(e, "cudaGetSymbolAddress(arena)");
    *out = static_cast<unsigned char *>(ptr);
    return PS_OK;
}

// Point-record tables that need arithmetic: w = sigr2 * weight and the
// per-point record {brightness, w, curve, relative}.  pw holds sigr2 on entry
// and tmp holds the weights.
__global__ void pack_points(int np, const int *curve_start, int n_curves, const int *curve_rel,
                            const double4 *pt_b, const double *tmp_weight, double *pw, double4 *prec, int *pcur)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= np) return;
    int c = 0;
    while (c + 1 < n_curves && curve_start[c + 1] <= q) ++c;
    const double w = pw[q] * tmp_weight[q];
    pw[q] = w;
    pcur[q] = c;
    prec[q] = make_double4(pt_b[q].w, w, (double)c, (double)curve_rel[c]);
}

struct Carver {
    size_t off = 0;
    template <typename T>
    size_t take(size_t count)
    {
        const size_t o = off;
        off = (off + count * sizeof(T) + 255) & ~size_t(255);
        return o;
    }
};

}  // namespace

#define NA_CUDA(call)                                          \
    do {                                                       \
        cudaError_t e_ = (call);                               \
        if (e_ != cudaSuccess) return psb_fail_cuda(e_, #call); \
    } while (0)

extern "C" ps_status ps_fit_items_noalloc(
    int32_t device, void *stream, const double *beta_pole, const double *lambda_pole, const double *par, double cl,
    double alamda_start, double alamda_incr, double alamda_incrr, const double *ee, const double *ee0,
    const double *tim, double phi0, const double *weight, double freq_start, double freq_step,
    double stop_condition, int32_t n_iter_min, double conw_r, double conw_r_rms, int32_t ndata,
    const int32_t *ia, const int32_t *ia_par, const double *cg_first, const double *sig, const double *sigr2,
    int32_t numfac, const double *brightness, const ps_curves *curves, const ps_shape *shape, int32_t n,
    const int32_t *n_freq, const int32_t *pole, ps_fit_result *out)
{
    if (device < 0 || device >= kMaxDevices || n < 0)
        return psb_fail(PS_ERR_ARG, "ps_fit_items_noalloc: device index or n < 0");
    if (n == 0) {
        // warm-up: select the device and load this module there, which
        // reserves the arena; nothing else is read or launched
        NA_CUDA(cudaSetDevice(device));
        unsigned char *arena = nullptr;
        return arena_address(&arena);
    }
    if (!beta_pole || !lambda_pole || !par || !ee || !ee0 || !tim || !weight || !ia || !ia_par || !cg_first ||
        !sig || !sigr2 || !brightness || !curves || !shape || !curves->curve_len || !curves->curve_rel ||
        !shape->normal || !shape->d_area || !shape->d_sphere || !n_freq || !pole || !out)
        return psb_fail(PS_ERR_ARG, "ps_fit_items_noalloc: null argument");
    if (!(cl > 0) || ndata <= 0 || !(freq_step > 0))
        return psb_fail(PS_ERR_ARG, "ps_fit_items_noalloc: cl, ndata and freq_step must be > 0");
    const int nc = shape->n_coef, ma = nc + 8, nfac = numfac, ncur = curves->n_curves;
    if (nc < 1 || ma > 89 || nfac < 1 || nfac > PS_MAX_FAC || ncur < 1 || ncur > kMaxCurves)
        return psb_fail(PS_ERR_ARG, "ps_fit_items_noalloc: n_coef 1..81, numfac 1..1024, 1..200 curves");
    for (int i = 0; i < n; ++i)
        if (n_freq[i] < 1 || pole[i] < 0 || pole[i] >= PS_N_POLES)
            return psb_fail(PS_ERR_ARG, "ps_fit_items_noalloc: frequency index < 1 or pole outside 0..9");

    // small host tables on the stack: curve starts, curve sigmas, fitted parameters
    int cstart[kMaxCurves + 1];
    int crel[kMaxCurves];
    double csig[kMaxCurves];
    int q = 0;
    for (int c = 0; c < ncur; ++c) {
        if (curves->curve_len[c] < 1) return psb_fail(PS_ERR_ARG, "ps_fit_items_noalloc: empty lightcurve");
        cstart[c] = q;
        crel[c] = curves->curve_rel[c] ? 1 : 0;
        csig[c] = sig[q < ndata ? q : 0];
        q += curves->curve_len[c];
    }
    cstart[ncur] = q;
    if (q != ndata) return psb_fail(PS_ERR_ARG, "ps_fit_items_noalloc: curve lengths do not sum to ndata");
    int fidx[PS_MAX_PAR];
    int mfit = 0;
    for (int p = 1; p <= ma; ++p) {
        const int on = (p >= nc + 4 && p <= nc + 6) ? ia_par[p - nc - 4] : ia[p];
        if (on) fidx[mfit++] = p;
    }
    if (mfit < 1) return psb_fail(PS_ERR_ARG, "ps_fit_items_noalloc: no fitted parameters");
    const int ncp = psb::padded_ncoef(nc);

    NA_CUDA(cudaSetDevice(device));
    unsigned char *arena = nullptr;
    ps_status st = arena_address(&arena);
    if (st != PS_OK) return st;
    int smem_optin = 0, n_sm = 0;
    NA_CUDA(cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
    NA_CUDA(cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, device));
    const size_t smem_limit = (size_t)smem_optin;
    int tile_rows = 32, cstat_smem = 1;
    const int rs = (ma + 2) & ~1;
    size_t smem = psb::fit_smem_bytes(nfac, mfit, ncp, ncur, rs, tile_rows, cstat_smem, 0);
    if (smem > smem_limit) {
        cstat_smem = 0;
        smem = psb::fit_smem_bytes(nfac, mfit, ncp, ncur, rs, tile_rows, cstat_smem, 0);
    }
    if (smem > smem_limit) {
        tile_rows = 16;
        smem = psb::fit_smem_bytes(nfac, mfit, ncp, ncur, rs, tile_rows, cstat_smem, 0);
    }
    if (smem > smem_limit)
        return psb_fail(PS_ERR_ARG, "ps_fit_items_noalloc: object too large for shared memory");

    // arena layout
    Carver cv;
    const size_t o_facet = cv.take<double4>(nfac), o_ysh = cv.take<double>((size_t)nfac * ncp);
    const size_t o_pa = cv.take<double4>(ndata), o_pb = cv.take<double4>(ndata);
    const size_t o_pw = cv.take<double>(ndata), o_tmp = cv.take<double>(ndata);
    const size_t o_prec = cv.take<double4>(ndata), o_pcur = cv.take<int>(ndata);
    const size_t o_cstart = cv.take<int>(ncur + 1), o_crel = cv.take<int>(ncur), o_csig = cv.take<double>(ncur);
    const size_t o_fidx = cv.take<int>(mfit), o_cg = cv.take<double>(nc);
    const size_t o_items = cv.take<psb::FitItem>(n), o_out = cv.take<psb::FitOut>(n);
    const size_t o_ctl = cv.take<int>(2);
    const size_t o_scratch = cv.off;

    psb::DevObject o{};
    o.n_points = ndata;
    o.n_curves = ncur;
    o.n_fac = nfac;
    o.n_coef = nc;
    o.ncp = ncp;
    o.ma = ma;
    o.mfit = mfit;
    o.row_stride = rs;
    o.tile_rows = tile_rows;
    o.cstat_smem = cstat_smem;
    const size_t per_cta = psb::fit_scratch_doubles(o) * sizeof(double);
    if (o_scratch + per_cta > kNoAllocArenaBytes)
        return psb_fail(PS_ERR_ARG, "ps_fit_items_noalloc: object and items exceed the 64 MiB arena");
    o.facet = reinterpret_cast<const double4 *>(arena + o_facet);
    o.ysh = reinterpret_cast<const double *>(arena + o_ysh);
    o.pt_a = reinterpret_cast<const double4 *>(arena + o_pa);
    o.pt_b = reinterpret_cast<const double4 *>(arena + o_pb);
    o.pt_w = reinterpret_cast<const double *>(arena + o_pw);
    o.pt_rec = reinterpret_cast<const double4 *>(arena + o_prec);
    o.pt_curve = reinterpret_cast<const int *>(arena + o_pcur);
    o.curve_start = reinterpret_cast<const int *>(arena + o_cstart);
    o.curve_rel = reinterpret_cast<const int *>(arena + o_crel);
    o.curve_sig = reinterpret_cast<const double *>(arena + o_csig);
    o.fidx = reinterpret_cast<const int *>(arena + o_fidx);
    o.cg_first = reinterpret_cast<const double *>(arena + o_cg);

    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const cudaMemcpyKind h2d = cudaMemcpyHostToDevice;
    // facet records {normal, d_area} and the zero-padded basis
    NA_CUDA(cudaMemcpy2DAsync(arena + o_facet, sizeof(double4), shape->normal, 3 * sizeof(double),
                              3 * sizeof(double), nfac, h2d, s));
    NA_CUDA(cudaMemcpy2DAsync(arena + o_facet + 3 * sizeof(double), sizeof(double4), shape->d_area, sizeof(double),
                              sizeof(double), nfac, h2d, s));
    NA_CUDA(cudaMemsetAsync(arena + o_ysh, 0, (size_t)nfac * ncp * sizeof(double), s));
    NA_CUDA(cudaMemcpy2DAsync(arena + o_ysh, ncp * sizeof(double), shape->d_sphere, nc * sizeof(double),
                              nc * sizeof(double), nfac, h2d, s));
    // point records {t, ee} and {ee0, brightness}
    NA_CUDA(cudaMemcpy2DAsync(arena + o_pa, sizeof(double4), tim, sizeof(double), sizeof(double), ndata, h2d, s));
    NA_CUDA(cudaMemcpy2DAsync(arena + o_pa + sizeof(double), sizeof(double4), ee, 3 * sizeof(double),
                              3 * sizeof(double), ndata, h2d, s));
    NA_CUDA(cudaMemcpy2DAsync(arena + o_pb, sizeof(double4), ee0, 3 * sizeof(double), 3 * sizeof(double), ndata,
                              h2d, s));
    NA_CUDA(cudaMemcpy2DAsync(arena + o_pb + 3 * sizeof(double), sizeof(double4), brightness, sizeof(double),
                              sizeof(double), ndata, h2d, s));
    NA_CUDA(cudaMemcpyAsync(arena + o_pw, sigr2, ndata * sizeof(double), h2d, s));
    NA_CUDA(cudaMemcpyAsync(arena + o_tmp, weight, ndata * sizeof(double), h2d, s));
    NA_CUDA(cudaMemcpyAsync(arena + o_cstart, cstart, (ncur + 1) * sizeof(int), h2d, s));
    NA_CUDA(cudaMemcpyAsync(arena + o_crel, crel, ncur * sizeof(int), h2d, s));
    NA_CUDA(cudaMemcpyAsync(arena + o_csig, csig, ncur * sizeof(double), h2d, s));
    NA_CUDA(cudaMemcpyAsync(arena + o_fidx, fidx, mfit * sizeof(int), h2d, s));
    NA_CUDA(cudaMemcpyAsync(arena + o_cg, cg_first, nc * sizeof(double), h2d, s));
    // work items {n_freq, pole}
    NA_CUDA(cudaMemcpy2DAsync(arena + o_items, sizeof(psb::FitItem), n_freq, sizeof(int32_t), sizeof(int32_t), n,
                              h2d, s));
    NA_CUDA(cudaMemcpy2DAsync(arena + o_items + sizeof(int32_t), sizeof(psb::FitItem), pole, sizeof(int32_t),
                              sizeof(int32_t), n, h2d, s));
    // the queue counter and the status word must start at zero on every call
    NA_CUDA(cudaMemsetAsync(arena + o_ctl, 0, 2 * sizeof(int), s));
    pack_points<<<(ndata + 255) / 256, 256, 0, s>>>(
        ndata, reinterpret_cast<const int *>(arena + o_cstart), ncur, reinterpret_cast<const int *>(arena + o_crel),
        reinterpret_cast<const double4 *>(arena + o_pb), reinterpret_cast<const double *>(arena + o_tmp),
        reinterpret_cast<double *>(arena + o_pw), reinterpret_cast<double4 *>(arena + o_prec),
        reinterpret_cast<int *>(arena + o_pcur));
    NA_CUDA(cudaGetLastError());

    psb::DevParams p{};
    p.phi0 = phi0;
    for (int i = 0; i < 3; ++i) p.par[i] = par[i];
    p.lcl = std::log(cl);
    p.alamda_start = alamda_start;
    p.alamda_incr = alamda_incr;
    p.alamda_incrr = alamda_incrr;
    for (int i = 0; i < PS_N_POLES; ++i) {
        p.beta_pole[i] = beta_pole[i];
        p.lambda_pole[i] = lambda_pole[i];
    }
    // stop condition (start_CUDA.cu:855-869)
    p.n_iter_max = 0;
    p.iter_diff_max = -1;
    p.n_iter_min = n_iter_min;
    if (stop_condition > 1) {
        p.n_iter_max = (int)stop_condition;
        p.iter_diff_max = 0;
        p.n_iter_min = 0;
    }
    if (stop_condition < 1) {
        p.n_iter_max = kMaxIterCap;
        p.iter_diff_max = stop_condition;
    }
    p.conw_r = conw_r;
    p.conw_r_dev = conw_r_rms;
    p.freq_start = freq_start;
    p.freq_step = freq_step;
    p.phase_cycles = nullptr;

    const int per_sm = psb::fit_ctas_per_sm(o);
    if (per_sm < 1) return psb_fail(PS_ERR_CUDA, "ps_fit_items_noalloc: fit kernel cannot be resident");
    const size_t fit_scratch = (kNoAllocArenaBytes - o_scratch) / per_cta;
    int n_ctas = per_sm * n_sm;
    if ((size_t)n_ctas > fit_scratch) n_ctas = (int)fit_scratch;
    if (n_ctas > n) n_ctas = n;
    int *ctl = reinterpret_cast<int *>(arena + o_ctl);
    int e = psb::launch_fits(o, p, reinterpret_cast<const psb::FitItem *>(arena + o_items), n, ctl,
                             reinterpret_cast<psb::FitOut *>(arena + o_out),
                             reinterpret_cast<double *>(arena + o_scratch), per_cta / sizeof(double), n_ctas,
                             ctl + 1, s);
    if (e) return psb_fail_cuda(e, "ps_fit_items_noalloc: fit kernel launch");
    NA_CUDA(cudaMemcpyAsync(out, arena + o_out, (size_t)n * sizeof(ps_fit_result), cudaMemcpyDeviceToHost, s));
    NA_CUDA(cudaStreamSynchronize(s));
    return PS_OK;
}
