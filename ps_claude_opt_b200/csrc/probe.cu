// probe.cu -- FP64 FMA throughput probe: the compute roofline denominator of
// the fit kernel.  Independent FMA chains per thread, enough warps per SM to
// keep the FP64 pipe busy; returns achieved TFLOP/s (2 FLOP per FMA).
#include <cuda_runtime.h>

#include "devmath.cuh"
#include "fit_kernel.cuh"
#include "ps_b200.h"
#include "util.h"

namespace {

constexpr int kChains = 8;
constexpr int kIters = 4096;

__global__ void __launch_bounds__(256) fma_probe(double *out, double x)
{
    double a[kChains];
#pragma unroll
    for (int c = 0; c < kChains; ++c) a[c] = x + threadIdx.x * 1e-9 + c;
    const double m = 0.999999, s = 1e-7;
#pragma unroll 4
    for (int i = 0; i < kIters; ++i)
#pragma unroll
        for (int c = 0; c < kChains; ++c) a[c] = fma(a[c], m, s);
    double t = 0;
#pragma unroll
    for (int c = 0; c < kChains; ++c) t += a[c];
    if (t == 12345.678) out[blockIdx.x] = t;  // never true; keeps the work live
}

__global__ void rcp_probe(const double *d, double *r, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) r[i] = psb::rcp_nr(d[i]);
}

// A bulk-copy barrier that nothing will ever complete: the fit kernel's
// bounded wait on it must give up and report, leaving the context usable.
__global__ void wait_probe(unsigned limit, int *status)
{
    __shared__ unsigned long long bar;
    if (threadIdx.x == 0) psb::mbar_init(&bar, 1);
    __syncthreads();
    if (threadIdx.x == 0) status[0] = psb::mbar_wait(&bar, 0, limit) ? 0 : psb::kStatusTimeout;
}

// The fit kernel's damped solve on one n x n system (one CTA, the kernel's
// shared-memory layout for covar, da, red and ctl).
__global__ void __launch_bounds__(psb::kThreads) solve_probe(const double *a, const double *b, int n, double *x,
                                                             int *err)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const int ld = psb::fit_ld(n);
    psb::Sh s{};
    double *covar = reinterpret_cast<double *>(smem);
    double *da = covar + (size_t)n * ld + (n * ld & 1);
    double *red = da + psb::kMaxFit;
    int *ctl = reinterpret_cast<int *>(red + psb::kWarps * 4);
    s.covar = covar;
    s.da = da;
    s.red = red;
    s.ctl = ctl;
    s.ld = ld;
    for (int idx = threadIdx.x; idx < n * n; idx += blockDim.x) covar[(idx / n) * ld + idx % n] = a[idx];
    for (int j = threadIdx.x; j < n; j += blockDim.x) da[j] = b[j];
    __syncthreads();
    const int e = n <= 64 ? psb::gauss_jordan<64>(s, n) : psb::gauss_jordan<psb::kMaxFit>(s, n);
    for (int j = threadIdx.x; j < n; j += blockDim.x) x[j] = da[j];
    if (threadIdx.x == 0) err[0] = e;
}

size_t solve_probe_smem(int n)
{
    const size_t ld = psb::fit_ld(n);
    return sizeof(double) * ((size_t)n * ld + 1 + psb::kMaxFit + psb::kWarps * 4) + sizeof(int) * psb::C_NCTL;
}

}  // namespace

extern "C" ps_status ps_probe_solve(int32_t n, const double *a, const double *b, double *x, int32_t *err)
{
    if (n < 1 || n > psb::kMaxFit - 1 || !a || !b || !x || !err)
        return psb_fail(PS_ERR_ARG, "ps_probe_solve: bad arguments");
    double *d = nullptr;
    const size_t nn = (size_t)n * n;
    cudaError_t e = cudaMalloc(&d, sizeof(double) * (nn + 2 * (size_t)n) + sizeof(int) * 2);
    if (e != cudaSuccess) return psb_fail_cuda(e, "cudaMalloc");
    int *derr = reinterpret_cast<int *>(d + nn + 2 * n);
    const size_t smem = solve_probe_smem(n);
    e = cudaFuncSetAttribute(solve_probe, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess) e = cudaMemcpy(d, a, sizeof(double) * nn, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d + nn, b, sizeof(double) * n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        solve_probe<<<1, psb::kThreads, smem>>>(d, d + nn, n, d + nn + n, derr);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(x, d + nn + n, sizeof(double) * n, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(err, derr, sizeof(int), cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return psb_fail_cuda(e, "ps_probe_solve");
    return PS_OK;
}

extern "C" ps_status ps_probe_wait_timeout(int32_t polls, int32_t *status)
{
    if (polls < 1 || !status) return psb_fail(PS_ERR_ARG, "ps_probe_wait_timeout: bad arguments");
    int *d = nullptr;
    cudaError_t e = cudaMalloc(&d, sizeof(int));
    if (e != cudaSuccess) return psb_fail_cuda(e, "cudaMalloc");
    e = cudaMemset(d, 0xff, sizeof(int));
    if (e == cudaSuccess) {
        wait_probe<<<1, 32>>>((unsigned)polls, d);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(status, d, sizeof(int), cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return psb_fail_cuda(e, "ps_probe_wait_timeout");
    return PS_OK;
}

extern "C" ps_status ps_probe_reciprocal(int32_t n, const double *d, double *r)
{
    if (n <= 0 || !d || !r) return psb_fail(PS_ERR_ARG, "ps_probe_reciprocal: bad arguments");
    double *dd = nullptr;
    cudaError_t e = cudaMalloc(&dd, sizeof(double) * 2 * (size_t)n);
    if (e != cudaSuccess) return psb_fail_cuda(e, "cudaMalloc");
    e = cudaMemcpy(dd, d, sizeof(double) * n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        rcp_probe<<<(n + 255) / 256, 256>>>(dd, dd + n, n);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(r, dd + n, sizeof(double) * n, cudaMemcpyDeviceToHost);
    cudaFree(dd);
    if (e != cudaSuccess) return psb_fail_cuda(e, "ps_probe_reciprocal");
    return PS_OK;
}

extern "C" ps_status ps_measure_fp64_peak(int32_t device, double *tflops)
{
    if (!tflops) return psb_fail(PS_ERR_ARG, "ps_measure_fp64_peak: null argument");
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return psb_fail_cuda(e, "cudaSetDevice");
    cudaDeviceProp prop;
    if ((e = cudaGetDeviceProperties(&prop, device)) != cudaSuccess) return psb_fail_cuda(e, "cudaGetDeviceProperties");
    const int blocks = prop.multiProcessorCount * 8;
    double *out = nullptr;
    if ((e = cudaMalloc(&out, sizeof(double) * blocks)) != cudaSuccess) return psb_fail_cuda(e, "cudaMalloc");
    cudaEvent_t t0, t1;
    cudaEventCreate(&t0);
    cudaEventCreate(&t1);
    fma_probe<<<blocks, 256>>>(out, 1.0);  // warm-up
    float best_ms = 1e30f;
    for (int r = 0; r < 5; ++r) {
        cudaEventRecord(t0);
        fma_probe<<<blocks, 256>>>(out, 1.0 + r);
        cudaEventRecord(t1);
        cudaEventSynchronize(t1);
        float ms = 0;
        cudaEventElapsedTime(&ms, t0, t1);
        if (ms < best_ms) best_ms = ms;
    }
    e = cudaGetLastError();
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    cudaFree(out);
    if (e != cudaSuccess) return psb_fail_cuda(e, "fma_probe");
    const double flop = 2.0 * kChains * (double)kIters * 256.0 * blocks;
    *tflops = flop / (best_ms * 1e-3) / 1e12;
    return PS_OK;
}
