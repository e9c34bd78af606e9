// handle.h -- the ps_gpu handle behind the C ABI and the helpers its entry
// points share (host side only).
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "engine.h"
#include "ps_b200.h"
#include "util.h"

#define PSB_CUDA(call)                                         \
    do {                                                       \
        cudaError_t e_ = (call);                               \
        if (e_ != cudaSuccess) return psb_fail_cuda(e_, #call); \
    } while (0)

namespace psb {

constexpr int kMaxIter = 60;  // the reference's MAX_N_ITER (constants.h:12)

// A device buffer that grows on demand and never shrinks.
template <typename T>
struct DevBuf {
    T *ptr = nullptr;
    size_t cap = 0;
    cudaError_t ensure(size_t n)
    {
        if (n <= cap && ptr) return cudaSuccess;
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        cap = 0;
        cudaError_t e = cudaMalloc(&ptr, std::max<size_t>(n, 1) * sizeof(T));
        if (e == cudaSuccess) cap = std::max<size_t>(n, 1);
        return e;
    }
    void release()
    {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        cap = 0;
    }
};

template <typename T>
cudaError_t upload(DevBuf<T> &b, const std::vector<T> &v, cudaStream_t s)
{
    cudaError_t e = b.ensure(v.size());
    if (e != cudaSuccess) return e;
    return cudaMemcpyAsync(b.ptr, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s);
}

}  // namespace psb

struct ps_gpu {
    int device = 0;
    int n_sm = 0;
    cudaStream_t stream = nullptr;
    int quirks = 0;
    int precision = PS_PRECISION_FP64;  // applies from the next configure
    // prepare-time inputs
    int ndata = 0;
    std::vector<double> tim, ee, ee0, weight;
    double beta_pole[PS_N_POLES], lambda_pole[PS_N_POLES], par[3];
    double lcl = 0, alamda_start = 0, alamda_incr = 0, alamda_incrr = 0, phi0 = 0;
    // configured object
    bool configured = false;
    psb::DevObject obj{};
    psb::DevParams prm{};
    int ctas_per_sm = 0;
    psb::DevBuf<double4> facet, pt_a, pt_b, pt_rec;
    psb::DevBuf<double> ysh, pt_w, curve_sig, cg_first, scratch, eval_buf;
    psb::DevBuf<float> ysh32;
    psb::DevBuf<int> pt_curve, curve_start, curve_rel, fidx, queue, status;
    psb::DevBuf<psb::FitItem> items;
    psb::DevBuf<unsigned long long> phase;
    psb::DevBuf<psb::FitOut> out;
    size_t scratch_per_cta = 0;
};

// Best pole of one frequency's 10 results: NaN-safe, earliest pole wins ties
// (start_CUDA.cu:1200-1229).
int psb_best_pole(const psb::FitOut *r);
