// screen.cu -- learned frequency screening: phase-folded lightcurve features
// per trial frequency and the kernels of a small BF16 multilayer perceptron
// (forward, backward, Adam) that ranks trial frequencies by predicted chi^2.
//
// No counterpart in the reference, which fits every trial frequency.  The
// screen proposes a subset (top-ranked frequencies plus a random audit
// sample); the plain scan of that subset then decides, and the full scan
// stays the fallback.
//
// Features (per frequency, 88 floats): each lightcurve c is folded at the
// trial frequency f (phase = frac(t f)) into 64 phase bins of its brightness
// relative to its mean; per curve 8 statistics: the phase-dispersion ratios
// theta_B = within-bin variance / total variance for B = 64, 32, 16, 8 bins,
// and the shares H_1..H_4 of the first four harmonics in the power of the
// 32-bin mean curve; over the curves 8 aggregates of each statistic: mean
// weighted by points, plain mean, standard deviation, min, 25 %, 50 %,
// 75 % quantiles, max (features 8 * statistic + aggregate, 0..63).  Single
// nights cannot tell neighbouring grid frequencies apart (the grid step is a
// few rotations over the whole time span), so the same 8 statistics follow
// for three folds of all points together: all of them, those before the
// middle of the time span, those after it (features 64 + 8 * fold + stat).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "ps_b200.h"
#include "util.h"

namespace {

constexpr int kBins = 64;
constexpr int kStats = 8;
constexpr int kAggs = 8;
constexpr int kFeatThreads = 256;
constexpr int kFeatWarps = kFeatThreads / 32;
constexpr int kMaxScreenCurves = 256;
constexpr int kGlobalFolds = 3;
constexpr int kFeatures = kStats * kAggs + kGlobalFolds * kStats;

// Bin sums are fixed-point (2^-32 units) 64-bit integers: shared-memory
// atomics on them add in any order to the same total, so the features -- and
// the screen's choice of frequencies -- are the same on every run.
constexpr double kFix = 4294967296.0;  // 2^32

__device__ __forceinline__ void bin_add(unsigned long long *cnt, unsigned long long *sum, unsigned long long *ssq,
                                        int b, float v)
{
    atomicAdd(&cnt[b], 1ull);
    atomicAdd(&sum[b], (unsigned long long)__double2ll_rn((double)v * kFix));
    atomicAdd(&ssq[b], (unsigned long long)__double2ll_rn((double)v * (double)v * kFix));
}

// Per-curve statistics of one fold (lane 0 of a warp, bins in shared memory).
__device__ void curve_stats(const unsigned long long *cntb, const unsigned long long *sumb,
                            const unsigned long long *ssqb, float *st)
{
    auto cnt = [&](int b) { return (double)cntb[b]; };
    auto sum = [&](int b) { return (double)(long long)sumb[b] / kFix; };
    auto ssq = [&](int b) { return (double)(long long)ssqb[b] / kFix; };
    double n = 0, s1 = 0, s2 = 0;
    for (int b = 0; b < kBins; ++b) {
        n += cnt(b);
        s1 += sum(b);
        s2 += ssq(b);
    }
    const double total = s2 - (n > 0 ? s1 * s1 / n : 0.0);
    for (int lev = 0; lev < 4; ++lev) {  // B = 64 >> lev bins
        const int w = 1 << lev;
        double within = 0;
        for (int b = 0; b < kBins; b += w) {
            double c = 0, a = 0, q = 0;
            for (int i = 0; i < w; ++i) {
                c += cnt(b + i);
                a += sum(b + i);
                q += ssq(b + i);
            }
            if (c > 0) within += q - a * a / c;
        }
        st[lev] = total > 0 ? (float)(within / total) : 1.0f;
    }
    // harmonics of the 32-bin mean curve (empty bins left out)
    double re[4] = {0, 0, 0, 0}, im[4] = {0, 0, 0, 0};
    for (int b = 0; b < 32; ++b) {
        const double c = cnt(2 * b) + cnt(2 * b + 1);
        if (c <= 0) continue;
        const double m = (sum(2 * b) + sum(2 * b + 1)) / c;
        for (int k = 0; k < 4; ++k) {
            double sn, cs;
            sincospi((double)(2 * (k + 1) * b) / 32.0, &sn, &cs);
            re[k] += m * cs;
            im[k] -= m * sn;
        }
    }
    double pw[4], tot = 0;
    for (int k = 0; k < 4; ++k) {
        pw[k] = re[k] * re[k] + im[k] * im[k];
        tot += pw[k];
    }
    for (int k = 0; k < 4; ++k) st[4 + k] = tot > 0 ? (float)(pw[k] / tot) : 0.25f;
}

// One block per trial frequency; each warp folds one lightcurve at a time.
// y[i] = brightness / curve mean - 1.
__global__ void __launch_bounds__(kFeatThreads) features_kernel(const double *tim, const float *y,
                                                                 const int *cstart, int n_curves,
                                                                 const double *freqs, int n_freq, double t_mid,
                                                                 float *out)
{
    __shared__ unsigned long long bins[kFeatWarps][3][kBins];
    __shared__ float cst[kStats][kMaxScreenCurves];
    __shared__ float cw[kMaxScreenCurves];
    const int f = blockIdx.x;
    if (f >= n_freq) return;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const double fr = freqs[f];
    unsigned long long *cnt = bins[warp][0], *sum = bins[warp][1], *ssq = bins[warp][2];
    for (int c = warp; c < n_curves; c += kFeatWarps) {
        for (int b = lane; b < kBins; b += 32) cnt[b] = sum[b] = ssq[b] = 0ull;
        __syncwarp();
        const int p0 = cstart[c], p1 = cstart[c + 1];
        for (int i = p0 + lane; i < p1; i += 32) {
            const double ph = tim[i] * fr;
            const double frac = ph - floor(ph);
            const int b = min(kBins - 1, max(0, (int)(frac * kBins)));
            bin_add(cnt, sum, ssq, b, y[i]);
        }
        __syncwarp();
        if (lane == 0) {
            float st[kStats];
            curve_stats(cnt, sum, ssq, st);
            for (int k = 0; k < kStats; ++k) cst[k][c] = st[k];
            cw[c] = (float)(p1 - p0);
        }
        __syncwarp();
    }
    __syncthreads();
    // folds of all points together: every warp bins a share of the points,
    // warp 0 adds the eight partial histograms and lane 0 takes the stats
    const int n_pts = cstart[n_curves];
    for (int fold = 0; fold < kGlobalFolds; ++fold) {
        for (int b = lane; b < kBins; b += 32) cnt[b] = sum[b] = ssq[b] = 0ull;
        __syncwarp();
        for (int i = threadIdx.x; i < n_pts; i += kFeatThreads) {
            const double t = tim[i];
            if ((fold == 1 && !(t < t_mid)) || (fold == 2 && t < t_mid)) continue;
            const double ph = t * fr;
            const double frac = ph - floor(ph);
            const int b = min(kBins - 1, max(0, (int)(frac * kBins)));
            bin_add(cnt, sum, ssq, b, y[i]);
        }
        __syncthreads();
        if (warp == 0) {
            for (int b = lane; b < kBins; b += 32)
                for (int w = 1; w < kFeatWarps; ++w) {
                    bins[0][0][b] += bins[w][0][b];
                    bins[0][1][b] += bins[w][1][b];
                    bins[0][2][b] += bins[w][2][b];
                }
            __syncwarp();
            if (lane == 0) {
                float st[kStats];
                curve_stats(bins[0][0], bins[0][1], bins[0][2], st);
                float *o = out + (size_t)f * kFeatures + kStats * kAggs + fold * kStats;
                for (int k = 0; k < kStats; ++k) o[k] = st[k];
            }
        }
        __syncthreads();
    }
    // aggregates: thread k of the first kStats sorts statistic k in place
    if (threadIdx.x < kStats) {
        float *v = cst[threadIdx.x];
        double ws = 0, wsum = 0, s = 0, s2 = 0;
        for (int c = 0; c < n_curves; ++c) {
            ws += (double)cw[c] * v[c];
            wsum += cw[c];
            s += v[c];
            s2 += (double)v[c] * v[c];
        }
        for (int i = 1; i < n_curves; ++i) {  // insertion sort (n_curves <= 256)
            const float x = v[i];
            int j = i - 1;
            while (j >= 0 && v[j] > x) {
                v[j + 1] = v[j];
                --j;
            }
            v[j + 1] = x;
        }
        const double mean = s / n_curves;
        const double var = s2 / n_curves - mean * mean;
        auto q = [&](double fq) {
            const double pos = fq * (n_curves - 1);
            const int lo = (int)floor(pos);
            const int hi = min(lo + 1, n_curves - 1);
            return (float)(v[lo] + (pos - lo) * (v[hi] - v[lo]));
        };
        float *o = out + (size_t)f * kFeatures + threadIdx.x * kAggs;
        o[0] = (float)(ws / wsum);
        o[1] = (float)mean;
        o[2] = (float)sqrt(fmax(var, 0.0));
        o[3] = v[0];
        o[4] = q(0.25);
        o[5] = q(0.5);
        o[6] = q(0.75);
        o[7] = v[n_curves - 1];
    }
}

// ---------------------------------------------------------------- BF16 GEMM

__device__ __forceinline__ uint32_t pack_bf16(__nv_bfloat16 lo, __nv_bfloat16 hi)
{
    return (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}

__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1)
{
    asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
                 "{%0,%1,%2,%3};"
                 : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
                 : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// C[m][n] (+)= sum_k A(m, k) B(k, n) (+ bias[n]) (ReLU), A(m, k) = A[m sam + k sak],
// B(k, n) = B[k sbk + n sbn], BF16 operands on the tensor cores, FP32
// accumulation.  A block of 4 warps computes a 64 x 32 tile; operands are
// read element by element with bounds checks, so any strides (transposes)
// and any sizes work.
constexpr int kGemmTM = 64, kGemmTN = 32;

__global__ void __launch_bounds__(128) gemm_bf16_kernel(int M, int N, int K, const __nv_bfloat16 *A, long sam,
                                                        long sak, const __nv_bfloat16 *B, long sbk, long sbn,
                                                        float *C, int ldc, int accumulate, const float *bias,
                                                        int relu, __nv_bfloat16 *Cb, int ldcb)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g = lane >> 2, t = lane & 3;
    const int m0 = blockIdx.y * kGemmTM + warp * 16;
    const int n0 = blockIdx.x * kGemmTN;
    const __nv_bfloat16 zero = __float2bfloat16(0.0f);
    auto ld_a = [&](int m, int k) { return (m < M && k < K) ? A[(long)m * sam + (long)k * sak] : zero; };
    auto ld_b = [&](int k, int n) { return (k < K && n < N) ? B[(long)k * sbk + (long)n * sbn] : zero; };
    float acc[4][4];
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.0f;
    for (int k0 = 0; k0 < K; k0 += 16) {
        uint32_t a[4];
        a[0] = pack_bf16(ld_a(m0 + g, k0 + 2 * t), ld_a(m0 + g, k0 + 2 * t + 1));
        a[1] = pack_bf16(ld_a(m0 + g + 8, k0 + 2 * t), ld_a(m0 + g + 8, k0 + 2 * t + 1));
        a[2] = pack_bf16(ld_a(m0 + g, k0 + 2 * t + 8), ld_a(m0 + g, k0 + 2 * t + 9));
        a[3] = pack_bf16(ld_a(m0 + g + 8, k0 + 2 * t + 8), ld_a(m0 + g + 8, k0 + 2 * t + 9));
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int n = n0 + 8 * j + g;
            const uint32_t b0 = pack_bf16(ld_b(k0 + 2 * t, n), ld_b(k0 + 2 * t + 1, n));
            const uint32_t b1 = pack_bf16(ld_b(k0 + 2 * t + 8, n), ld_b(k0 + 2 * t + 9, n));
            mma_bf16(acc[j], a, b0, b1);
        }
    }
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const int m = m0 + g + (e >= 2 ? 8 : 0);
            const int n = n0 + 8 * j + 2 * t + (e & 1);
            if (m >= M || n >= N) continue;
            float v = acc[j][e];
            if (accumulate) v += C[(long)m * ldc + n];
            if (bias) v += bias[n];
            if (relu) v = fmaxf(v, 0.0f);
            if (C) C[(long)m * ldc + n] = v;
            if (Cb) Cb[(long)m * ldcb + n] = __float2bfloat16(v);
        }
}

// dZ = dH * (Z > 0), as BF16 (the next backward GEMM's operand) and FP32.
__global__ void relu_backward_kernel(long n, const float *dh, const float *z, float *dz, __nv_bfloat16 *dzb)
{
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float v = z[i] > 0.0f ? dh[i] : 0.0f;
    if (dz) dz[i] = v;
    if (dzb) dzb[i] = __float2bfloat16(v);
}

// db[n] = sum over rows of dZ[r][n] (one thread per column, rows in order).
__global__ void column_sum_kernel(int rows, int cols, const float *dz, float *db)
{
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= cols) return;
    float s = 0.0f;
    for (int r = 0; r < rows; ++r) s += dz[(long)r * cols + n];
    db[n] = s;
}

// Adam on FP32 master weights, then the BF16 working copy.
__global__ void adam_kernel(long n, float *w, const float *grad, float *m, float *v, float lr, float b1, float b2,
                            float eps, float c1, float c2, __nv_bfloat16 *wb)
{
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gr = grad[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gr;
    const float vi = b2 * v[i] + (1.0f - b2) * gr * gr;
    m[i] = mi;
    v[i] = vi;
    const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    w[i] = wi;
    if (wb) wb[i] = __float2bfloat16(wi);
}

__global__ void to_bf16_kernel(long n, const float *x, __nv_bfloat16 *y)
{
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] = __float2bfloat16(x[i]);
}

inline unsigned blocks_for(long n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

#define SC_CUDA(call)                                          \
    do {                                                       \
        cudaError_t e_ = (call);                               \
        if (e_ != cudaSuccess) return psb_fail_cuda(e_, #call); \
    } while (0)

extern "C" ps_status ps_screen_features(int32_t device, int32_t n_points, const double *tim,
                                        const double *brightness, const ps_curves *curves, int32_t n_freq,
                                        const double *freqs, float *features)
{
    if (n_points <= 0 || !tim || !brightness || !curves || !curves->curve_len || n_freq < 0 ||
        (n_freq > 0 && (!freqs || !features)))
        return psb_fail(PS_ERR_ARG, "ps_screen_features: null argument or n_points <= 0");
    const int nc = curves->n_curves;
    if (nc < 1 || nc > kMaxScreenCurves) return psb_fail(PS_ERR_ARG, "ps_screen_features: 1..256 lightcurves");
    if (n_freq == 0) return PS_OK;
    std::vector<int> cstart(nc + 1);
    std::vector<float> y(n_points);
    int q = 0;
    for (int c = 0; c < nc; ++c) {
        const int len = curves->curve_len[c];
        if (len < 1) return psb_fail(PS_ERR_ARG, "ps_screen_features: empty lightcurve");
        cstart[c] = q;
        if (q + len > n_points) return psb_fail(PS_ERR_ARG, "ps_screen_features: curve lengths exceed n_points");
        double mean = 0;
        for (int i = 0; i < len; ++i) mean += brightness[q + i];
        mean /= len;
        for (int i = 0; i < len; ++i) y[q + i] = (float)(mean != 0 ? brightness[q + i] / mean - 1.0 : 0.0);
        q += len;
    }
    cstart[nc] = q;
    if (q != n_points) return psb_fail(PS_ERR_ARG, "ps_screen_features: curve lengths do not sum to n_points");
    double t_lo = tim[0], t_hi = tim[0];
    for (int i = 1; i < n_points; ++i) {
        t_lo = fmin(t_lo, tim[i]);
        t_hi = fmax(t_hi, tim[i]);
    }
    const double t_mid = 0.5 * (t_lo + t_hi);
    SC_CUDA(cudaSetDevice(device));
    double *d_tim = nullptr, *d_freq = nullptr;
    float *d_y = nullptr, *d_out = nullptr;
    int *d_cs = nullptr;
    cudaError_t e = cudaMalloc(&d_tim, sizeof(double) * n_points);
    if (e == cudaSuccess) e = cudaMalloc(&d_freq, sizeof(double) * n_freq);
    if (e == cudaSuccess) e = cudaMalloc(&d_y, sizeof(float) * n_points);
    if (e == cudaSuccess) e = cudaMalloc(&d_out, sizeof(float) * (size_t)n_freq * kFeatures);
    if (e == cudaSuccess) e = cudaMalloc(&d_cs, sizeof(int) * (nc + 1));
    if (e == cudaSuccess) e = cudaMemcpy(d_tim, tim, sizeof(double) * n_points, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d_freq, freqs, sizeof(double) * n_freq, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d_y, y.data(), sizeof(float) * n_points, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d_cs, cstart.data(), sizeof(int) * (nc + 1), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        features_kernel<<<n_freq, kFeatThreads>>>(d_tim, d_y, d_cs, nc, d_freq, n_freq, t_mid, d_out);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess)
        e = cudaMemcpy(features, d_out, sizeof(float) * (size_t)n_freq * kFeatures, cudaMemcpyDeviceToHost);
    cudaFree(d_tim);
    cudaFree(d_freq);
    cudaFree(d_y);
    cudaFree(d_out);
    cudaFree(d_cs);
    if (e != cudaSuccess) return psb_fail_cuda(e, "ps_screen_features");
    return PS_OK;
}

extern "C" ps_status ps_gemm_bf16(int32_t M, int32_t N, int32_t K, const void *A, int64_t sam, int64_t sak,
                                  const void *B, int64_t sbk, int64_t sbn, float *C, int32_t ldc, int32_t accumulate,
                                  const float *bias, int32_t relu, void *Cb, int32_t ldcb, void *stream)
{
    if (M < 0 || N < 0 || K < 0 || !A || !B || (!C && !Cb) || (accumulate && !C))
        return psb_fail(PS_ERR_ARG, "ps_gemm_bf16: bad arguments");
    if (M == 0 || N == 0) return PS_OK;
    dim3 grid((N + kGemmTN - 1) / kGemmTN, (M + kGemmTM - 1) / kGemmTM);
    gemm_bf16_kernel<<<grid, 128, 0, (cudaStream_t)stream>>>(
        M, N, K, (const __nv_bfloat16 *)A, sam, sak, (const __nv_bfloat16 *)B, sbk, sbn, C, ldc, accumulate, bias,
        relu, (__nv_bfloat16 *)Cb, ldcb);
    SC_CUDA(cudaGetLastError());
    return PS_OK;
}

extern "C" ps_status ps_relu_backward(int64_t n, const float *dh, const float *z, float *dz, void *dzb, void *stream)
{
    if (n < 0 || !dh || !z || (!dz && !dzb)) return psb_fail(PS_ERR_ARG, "ps_relu_backward: bad arguments");
    if (n == 0) return PS_OK;
    relu_backward_kernel<<<blocks_for(n, 256), 256, 0, (cudaStream_t)stream>>>(n, dh, z, dz, (__nv_bfloat16 *)dzb);
    SC_CUDA(cudaGetLastError());
    return PS_OK;
}

extern "C" ps_status ps_column_sum(int32_t rows, int32_t cols, const float *x, float *out, void *stream)
{
    if (rows < 0 || cols < 0 || !x || !out) return psb_fail(PS_ERR_ARG, "ps_column_sum: bad arguments");
    if (cols == 0) return PS_OK;
    column_sum_kernel<<<blocks_for(cols, 128), 128, 0, (cudaStream_t)stream>>>(rows, cols, x, out);
    SC_CUDA(cudaGetLastError());
    return PS_OK;
}

extern "C" ps_status ps_adam_step(int64_t n, float *w, const float *grad, float *m, float *v, float lr, float beta1,
                                  float beta2, float eps, int32_t step, void *wb, void *stream)
{
    if (n < 0 || !w || !grad || !m || !v || step < 1) return psb_fail(PS_ERR_ARG, "ps_adam_step: bad arguments");
    if (n == 0) return PS_OK;
    const float c1 = 1.0f - powf(beta1, (float)step), c2 = 1.0f - powf(beta2, (float)step);
    adam_kernel<<<blocks_for(n, 256), 256, 0, (cudaStream_t)stream>>>(n, w, grad, m, v, lr, beta1, beta2, eps, c1,
                                                                       c2, (__nv_bfloat16 *)wb);
    SC_CUDA(cudaGetLastError());
    return PS_OK;
}

extern "C" ps_status ps_to_bf16(int64_t n, const float *x, void *y, void *stream)
{
    if (n < 0 || !x || !y) return psb_fail(PS_ERR_ARG, "ps_to_bf16: bad arguments");
    if (n == 0) return PS_OK;
    to_bf16_kernel<<<blocks_for(n, 256), 256, 0, (cudaStream_t)stream>>>(n, x, (__nv_bfloat16 *)y);
    SC_CUDA(cudaGetLastError());
    return PS_OK;
}

extern "C" ps_status ps_screen_rank(int32_t device, int32_t n_points, const double *tim, const double *brightness,
                                    const ps_curves *curves, int32_t n_freq, const double *freqs_per_hour,
                                    int32_t n_layers, const int32_t *sizes, const float *params, float *score)
{
    if (n_freq < 0 || (n_freq > 0 && (!freqs_per_hour || !score)) || n_layers < 1 || n_layers > 16 || !sizes ||
        !params)
        return psb_fail(PS_ERR_ARG, "ps_screen_rank: bad arguments");
    if (sizes[0] != kFeatures || sizes[n_layers] != 1)
        return psb_fail(PS_ERR_ARG, "ps_screen_rank: the network must map 88 features to 1 score");
    for (int l = 1; l < n_layers; ++l)
        if (sizes[l] < 1 || sizes[l] > 4096) return psb_fail(PS_ERR_ARG, "ps_screen_rank: layer width 1..4096");
    if (n_freq == 0) return PS_OK;
    // features (1/day), then standardised per feature over this object's frequencies
    std::vector<double> fday(n_freq);
    for (int f = 0; f < n_freq; ++f) fday[f] = 24.0 * freqs_per_hour[f];
    std::vector<float> feat((size_t)n_freq * kFeatures);
    ps_status st = ps_screen_features(device, n_points, tim, brightness, curves, n_freq, fday.data(), feat.data());
    if (st != PS_OK) return st;
    for (int k = 0; k < kFeatures; ++k) {
        double m = 0, m2 = 0;
        for (int f = 0; f < n_freq; ++f) m += feat[(size_t)f * kFeatures + k];
        m /= n_freq;
        for (int f = 0; f < n_freq; ++f) {
            const double d = feat[(size_t)f * kFeatures + k] - m;
            m2 += d * d;
        }
        const double sd = std::sqrt(m2 / n_freq);
        const double inv = sd > 1e-6 ? 1.0 / sd : 1.0;
        for (int f = 0; f < n_freq; ++f) {
            float &v = feat[(size_t)f * kFeatures + k];
            v = (float)((v - m) * inv);
        }
    }
    // device buffers: parameters (FP32 + BF16 copies), two activation buffers
    size_t n_par = 0, widest = kFeatures;
    for (int l = 0; l < n_layers; ++l) {
        n_par += (size_t)sizes[l + 1] * sizes[l] + sizes[l + 1];
        widest = std::max<size_t>(widest, (size_t)sizes[l + 1]);
    }
    float *d_par = nullptr, *d_out = nullptr;
    __nv_bfloat16 *d_parb = nullptr, *d_h[2] = {nullptr, nullptr};
    cudaError_t e = cudaMalloc(&d_par, sizeof(float) * n_par);
    if (e == cudaSuccess) e = cudaMalloc(&d_parb, sizeof(__nv_bfloat16) * n_par);
    if (e == cudaSuccess) e = cudaMalloc(&d_out, sizeof(float) * ((size_t)n_freq * widest + n_freq * kFeatures));
    if (e == cudaSuccess) e = cudaMalloc(&d_h[0], sizeof(__nv_bfloat16) * (size_t)n_freq * widest);
    if (e == cudaSuccess) e = cudaMalloc(&d_h[1], sizeof(__nv_bfloat16) * (size_t)n_freq * widest);
    float *d_feat = d_out + (size_t)n_freq * widest;
    if (e == cudaSuccess) e = cudaMemcpy(d_par, params, sizeof(float) * n_par, cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(d_feat, feat.data(), sizeof(float) * feat.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        to_bf16_kernel<<<blocks_for((long)n_par, 256), 256>>>((long)n_par, d_par, d_parb);
        to_bf16_kernel<<<blocks_for((long)feat.size(), 256), 256>>>((long)feat.size(), d_feat, d_h[0]);
        e = cudaGetLastError();
    }
    size_t off = 0;
    int cur = 0;
    for (int l = 0; l < n_layers && e == cudaSuccess; ++l) {
        const int k = sizes[l], n = sizes[l + 1];
        const __nv_bfloat16 *W = d_parb + off;
        const float *b = d_par + off + (size_t)n * k;
        off += (size_t)n * k + n;
        const bool last = l == n_layers - 1;
        dim3 grid((n + kGemmTN - 1) / kGemmTN, (n_freq + kGemmTM - 1) / kGemmTM);
        gemm_bf16_kernel<<<grid, 128>>>(n_freq, n, k, d_h[cur], k, 1, W, 1, k, last ? d_out : nullptr, n, 0, b,
                                        last ? 0 : 1, last ? nullptr : d_h[1 - cur], n);
        e = cudaGetLastError();
        cur = 1 - cur;
    }
    if (e == cudaSuccess) e = cudaMemcpy(score, d_out, sizeof(float) * n_freq, cudaMemcpyDeviceToHost);
    cudaFree(d_par);
    cudaFree(d_parb);
    cudaFree(d_out);
    cudaFree(d_h[0]);
    cudaFree(d_h[1]);
    if (e != cudaSuccess) return psb_fail_cuda(e, "ps_screen_rank");
    return PS_OK;
}
