// engine.cu -- template dispatch and launch wrappers of the fit kernel.
#include <cuda_runtime.h>

#include "engine.h"
#include "fit_kernel.cuh"

namespace psb {

using KernelFn = void (*)(DevObject, DevParams, const FitItem *, int, int *, FitOut *, double *, size_t,
                          int *, EvalOut, int, const DevObject *, const DevParams *);

// The shape-derivative accumulators live in registers, so the kernel is
// compiled per padded coefficient count.
#define PSB_NCP_LIST(X) X(16) X(24) X(32) X(40) X(48) X(56) X(64) X(72) X(80) X(88)

int padded_ncoef(int n_coef)
{
#define PSB_PICK(N) if (n_coef <= N) return N;
    PSB_NCP_LIST(PSB_PICK)
#undef PSB_PICK
    return -1;
}

size_t fit_smem_bytes(int n_fac, int mfit, int ncp, int n_curves, int row_stride, int tile_rows, int cstat_smem,
                      int mixed)
{
    return carve_bytes(n_fac, mfit, ncp, n_curves, row_stride, tile_rows, cstat_smem, mixed, nullptr, nullptr);
}

int chunk_facets_of(int ncp) { return chunk_facets(ncp); }

size_t fit_scratch_doubles(const DevObject &o)
{
    size_t n = scratch_perm(o.n_points, o.row_stride, o.n_curves, o.ma) + (size_t)o.n_points;
    return (n + 31) & ~size_t(31);
}

// The mixed-precision sweep is built for the smaller bases (chunks of 32
// facets, ncp <= kMaxMixedNcp).
#define PSB_MIXED_LIST(X) X(16) X(24) X(32) X(40) X(48) X(56) X(64)

// One translation unit per instance (fit_inst.cu) exports its kernel.
#define PSB_DECL(N) KernelFn fit_kernel_ptr_##N();
PSB_NCP_LIST(PSB_DECL)
#undef PSB_DECL
#define PSB_DECLM(N) KernelFn fit_kernel_mixed_ptr_##N();
PSB_MIXED_LIST(PSB_DECLM)
#undef PSB_DECLM
#define PSB_DECLB(N) KernelFn fit_kernel_batch_ptr_##N();
PSB_NCP_LIST(PSB_DECLB)
#undef PSB_DECLB

static KernelFn batch_kernel_for(int ncp)
{
    switch (ncp) {
#define PSB_CASEB(N) \
    case N:          \
        return fit_kernel_batch_ptr_##N();
        PSB_NCP_LIST(PSB_CASEB)
#undef PSB_CASEB
    default:
        return nullptr;
    }
}

static KernelFn kernel_for(int ncp, int mixed)
{
    if (mixed) {
        switch (ncp) {
#define PSB_CASEM(N) \
    case N:          \
        return fit_kernel_mixed_ptr_##N();
            PSB_MIXED_LIST(PSB_CASEM)
#undef PSB_CASEM
        default:
            return nullptr;
        }
    }
    switch (ncp) {
#define PSB_CASE(N) \
    case N:         \
        return fit_kernel_ptr_##N();
        PSB_NCP_LIST(PSB_CASE)
#undef PSB_CASE
    default:
        return nullptr;
    }
}

static int prepare_kernel(const DevObject &o, KernelFn *fn, size_t *smem)
{
    *fn = kernel_for(o.ncp, o.mixed);
    if (!*fn) return (int)cudaErrorInvalidValue;
    *smem = fit_smem_bytes(o.n_fac, o.mfit, o.ncp, o.n_curves, o.row_stride, o.tile_rows, o.cstat_smem, o.mixed);
    cudaError_t e = cudaFuncSetAttribute(*fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)*smem);
    return (int)e;
}

int fit_ctas_per_sm(const DevObject &o)
{
    KernelFn fn;
    size_t smem;
    if (prepare_kernel(o, &fn, &smem) != 0) return 0;
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, kThreads, smem) != cudaSuccess) return 0;
    return n;
}

int launch_fits(const DevObject &o, const DevParams &p, const FitItem *items, int n_items, int *queue,
                FitOut *out, double *scratch, size_t scratch_per_cta, int n_ctas, int *status, void *stream)
{
    KernelFn fn;
    size_t smem;
    int e = prepare_kernel(o, &fn, &smem);
    if (e) return e;
    EvalOut ev{};
    fn<<<n_ctas, kThreads, smem, (cudaStream_t)stream>>>(o, p, items, n_items, queue, out, scratch,
                                                         scratch_per_cta, status, ev, 0, nullptr, nullptr);
    return (int)cudaGetLastError();
}

int prepare_batch_kernel(const DevObject &env)
{
    KernelFn fn = batch_kernel_for(env.ncp);
    if (!fn || env.mixed) return (int)cudaErrorInvalidValue;
    const size_t smem = fit_smem_bytes(env.n_fac, env.mfit, env.ncp, env.n_curves, env.row_stride, env.tile_rows,
                                       env.cstat_smem, 0);
    return (int)cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

int fit_batch_ctas_per_sm(const DevObject &env)
{
    if (prepare_batch_kernel(env) != 0) return 0;
    const size_t smem = fit_smem_bytes(env.n_fac, env.mfit, env.ncp, env.n_curves, env.row_stride, env.tile_rows,
                                       env.cstat_smem, 0);
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, batch_kernel_for(env.ncp), kThreads, smem) != cudaSuccess)
        return 0;
    return n;
}

int launch_fits_batch(const DevObject &env, const DevObject *d_objs, const DevParams *d_prms, const FitItem *items,
                      int n_items, int *queue, FitOut *out, double *scratch, size_t scratch_per_cta, int n_ctas,
                      int *status, void *stream)
{
    KernelFn fn = batch_kernel_for(env.ncp);
    if (!fn || env.mixed) return (int)cudaErrorInvalidValue;
    const size_t smem = fit_smem_bytes(env.n_fac, env.mfit, env.ncp, env.n_curves, env.row_stride, env.tile_rows,
                                       env.cstat_smem, 0);
    DevParams p{};
    EvalOut ev{};
    fn<<<n_ctas, kThreads, smem, (cudaStream_t)stream>>>(env, p, items, n_items, queue, out, scratch,
                                                         scratch_per_cta, status, ev, 0, d_objs, d_prms);
    return (int)cudaGetLastError();
}

int launch_eval(const DevObject &o, const DevParams &p, EvalOut ev, double *scratch, void *stream)
{
    KernelFn fn;
    size_t smem;
    int e = prepare_kernel(o, &fn, &smem);
    if (e) return e;
    fn<<<1, kThreads, smem, (cudaStream_t)stream>>>(o, p, nullptr, 1, nullptr, nullptr, scratch, 0, nullptr,
                                                    ev, 1, nullptr, nullptr);
    return (int)cudaGetLastError();
}

}  // namespace psb
