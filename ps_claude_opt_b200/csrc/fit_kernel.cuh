// fit_kernel.cuh -- persistent FP64 Levenberg-Marquardt fit kernel for sm_100a.
//
// One CTA (256 threads) owns one (frequency, pole) fit at a time and runs its
// whole LM loop on the device; CTAs pop items from a device queue, so ragged
// iteration counts never idle the grid.  Per function evaluation (the
// reference's mrqcof, Start.cu:535-629 + 2262-2828):
//
//   A  curv: facet areas exp(sum a_k Y_k) into shared memory  (Start.cu:421-528)
//   B  brightness rows: a warp takes 32 points (lane = point) and sweeps every
//      facet once; visibility and the Lambert+Lommel-Seeliger terms per lane,
//      the shape derivatives sum_f w_f Y_k(f) as a GEMM on the FP64 tensor
//      cores (mma.sync m8n8k4).  The rotation derivatives use
//      dT/dq . (sum_f ar dS/dmu n_f), i.e. 6 accumulators per point instead of
//      6 dot products per facet.  Rows go to HBM scratch.
//   C  per relative curve: column sums and 1/sum(ymod)  (Start.cu:2519-2533)
//   D  J^T W J, J^T W dy, chi^2: one rank-k update of the augmented matrix
//      [J | dy] on the FP64 tensor cores, tiles of rows bulk-copied into
//      shared memory and renormalised on the fly.
//
// The LM step (damped Gauss-Jordan with full pivoting, accept/reject, lambda
// update, rms and convergence test) follows Start.cu:300-392, 2838-3021,
// 4421-4462, 5129-5248 with Numerical-Recipes ia compaction.
#pragma once
#include <climits>
#include <type_traits>
#include <cuda_runtime.h>

#include "devmath.cuh"
#include "engine.h"

namespace psb {

constexpr double kPi = 3.14159265358979323846;
constexpr double kTiny = 1e-8;
constexpr int kPoleBits = 8;                  // FitItem::pole = pole | object << kPoleBits (batch)
constexpr int kPoleMask = (1 << kPoleBits) - 1;
constexpr int kStages = 4;          // basis chunks in flight in the facet sweep
constexpr int kSortBands = 8;       // point sort: bands in cos(theta) ...
constexpr int kSortSectors = 32;    // ... x sectors in longitude of the Sun-observer bisector
constexpr int kSortCells = kSortBands * kSortSectors;
constexpr unsigned kWaitLimit = 1u << 24;  // bounded mbarrier waits

// LM scalar slots in shared memory
enum { S_ALAMDA, S_CHISQ, S_OCHISQ, S_ITERDIFF, S_DEVOLD, S_DEVNEW, S_CHCK, S_AREA, S_TRIAL, S_PIVINV, S_NSCAL };
enum { C_ITEM, C_NITER, C_STATUS, C_GJROW0, C_GO, C_TIMEOUT,
       C_YUSE,                       // [kStages] completed uses of each chunk buffer
       C_REL = C_YUSE + kStages,     // [kStages] warps done with the chunk in each buffer
       C_TUSE = C_REL + kStages,     // [2] completed uses of each J^T W J tile buffer
       C_TREL = C_TUSE + 2,          // [2] warps done with each tile buffer (k-slice mode)
       C_NCTL = C_TREL + 2 };
// per-CTA phase clocks (optional instrumentation)
enum { T_CURV, T_SORT, T_SWEEP, T_CSTAT, T_TILES, T_PSEUDO, T_SOLVE, T_REST, T_TWAIT, T_TSTAGE, T_TSYRK,
       T_NPHASE };

constexpr int kWS = 12;  // row stride (floats) of the mixed-precision weight tile: conflict-free A fragments

// Facets per basis chunk: keeps kStages chunks within ~60 KB of shared memory.
__host__ __device__ inline int chunk_facets(int ncp) { return ncp <= 64 ? 32 : 16; }
constexpr int kMaxChunkGroups = 8;  // 4-facet groups per basis chunk, at most

struct Sh {
    double4 *F;       // [n_fac] normal + current area
    float4 *cone;     // [ceil(n_fac / 4)] per 4-facet group: unit axis, sine of the half-angle + margin
    double *alpha;    // [mfit][ld]
    double *covar;    // [mfit][ld]
    double *beta;     // [kMaxFit]
    double *da;       // [kMaxFit]
    double *a;        // [kMaxPar]
    double *atry;     // [kMaxPar]
    double *T;        // [tile_rows][mfp]       (shares storage with ybuf)
    double *TW;       // [tile_rows][mfp]       (shares storage with ybuf)
    double *raw;      // [2][tile_rows][row_stride] raw rows of the tile (shares with ybuf)
    double4 *recb;    // [2][tile_rows] per-point records of the tile (shares with ybuf)
    unsigned long long *tbar;  // [2] completion barriers of the tile copies
    double *ccoef;    // [n_curves] renormalisation coefficient of each relative curve
    double *crave;    // [n_curves] 1 / sum(ymod) of each relative curve
    double *cst;      // [n_curves][ma + 3] per-curve statistics (when they fit here)
    double *wst;      // [kWarps][32][4] facet weights of one k-step, per warp (sweep MMA operand A)
    float *wst32;     // mixed precision: [kWarps][hi | lo][32][kWS] TF32 facet weights (same storage as wst)
    float4 *F32;      // mixed precision: [n_fac] normal + current area in FP32
    float2 *G32;      // mixed precision: [n_fac] area x Lambert weight, area x Lommel-Seeliger weight
    double *ybuf;     // [kStages][chunk_facets][ncp] basis chunks of the facet sweep
    unsigned long long *mbar;  // [kStages] completion barriers of the chunk copies
    long long *tclk;  // [T_NPHASE + 1] phase clocks, last slot = previous mark
    int *hist;        // [2][kSortCells] point-sort histogram and offsets
    double *rdy;      // [kTile] per-row residual y - ymod
    double *rw;       // [kTile] per-row weight sigr2 * weight
    double *rcoef;    // [kTile] per-row renormalisation coefficient (relative curves)
    double *rsub;     // [kTile] per-row ymod * rave (relative curves)
    int *rcur;        // [kTile] per-row curve index if relative, else -1
    double *red;      // [kWarps * 4]
    double *inv;      // [40] per-evaluation invariants
    double *scal;     // [S_NSCAL]
    int *fidx;        // [kMaxFit]
    int *ctl;         // [C_NCTL]
    int ld, mfp, tr;
};

__device__ __forceinline__ double4 ldg4(const double4 *p)
{
    const double2 *q = reinterpret_cast<const double2 *>(p);
    const double2 a = __ldg(q), b = __ldg(q + 1);
    return make_double4(a.x, a.y, b.x, b.y);
}

// ---------------------------------------------------------------- bulk copies

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(unsigned long long *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// One-thread producer: expect `bytes` on bar, then copy them global -> shared
// with the bulk-copy engine (cp.async.bulk, no cluster multicast).
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, unsigned long long *bar)
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

// Waits for the phase with the given parity to complete; gives up after
// `limit` polls (kWaitLimit in the fit kernel) and returns false (the caller
// records a timeout).
__device__ __forceinline__ bool mbar_wait(unsigned long long *bar, uint32_t parity, unsigned limit = kWaitLimit)
{
    for (unsigned i = 0; i < limit; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(smem_u32(bar)), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// Charges the cycles since the previous mark to `phase` (thread 0, when the
// caller asked for phase clocks).
__device__ __forceinline__ void tmark(const DevParams &p, const Sh &s, int phase)
{
    if (p.phase_cycles && threadIdx.x == 0) {
        const long long now = clock64();
        s.tclk[phase] += now - s.tclk[T_NPHASE];
        s.tclk[T_NPHASE] = now;
    }
}

// Row stride of alpha and covar: 4 mod 8 doubles, so the 8 rows x 4
// consecutive columns a warp touches in the solve's elimination spread evenly
// over the shared-memory banks.
__host__ __device__ inline int fit_ld(int mfit) { return mfit + ((4 - mfit) & 7); }
// Row stride of the J^T W J staging tiles: the augmented width mfit + 1
// rounded to whole 8-column MMA blocks, then to 4 mod 16 doubles so the
// 8x4 / 4x8 fragment loads of a half-warp hit 16 distinct 8-byte banks.
__host__ __device__ inline int fit_mpad(int mfit) { return (mfit + 1 + 7) & ~7; }
__host__ __device__ inline int fit_mfp(int mfit)
{
    const int mp = fit_mpad(mfit);
    return mp + ((4 - mp) & 15);
}

__host__ __device__ inline size_t align16(size_t x) { return (x + 15) & ~size_t(15); }

// Scratch slab of one CTA, in doubles from its start:
//   [0, n_points * row_stride)             derivative rows
//   [.., + n_curves * (ma + 3))            per-curve statistics
//   [gpart, + kWarps * 36 * 64)            rank-k partial sums (16-byte aligned)
//   [perm, + n_points)                     point order and sort keys (2 ints each)
__host__ __device__ inline size_t scratch_gpart(int n_points, int row_stride, int n_curves, int ma)
{
    return ((size_t)n_points * row_stride + (size_t)n_curves * (ma + 3) + 1) & ~size_t(1);
}
__host__ __device__ inline size_t scratch_perm(int n_points, int row_stride, int n_curves, int ma)
{
    return scratch_gpart(n_points, row_stride, n_curves, ma) + (size_t)kWarps * 36 * 64;
}

__host__ __device__ inline size_t carve_bytes(int n_fac, int mfit, int ncp, int n_curves, int rs, int tr,
                                              int cstat_smem, int mixed, Sh *s, unsigned char *base)
{
    int ld = fit_ld(mfit), mfp = fit_mfp(mfit);
    size_t off = 0;
    auto take = [&](size_t bytes) {
        size_t o = off;
        off = align16(off + bytes);
        return base ? (void *)(base + o) : nullptr;
    };
    void *F = take(sizeof(double4) * n_fac);
    void *cone = take(sizeof(float4) * ((n_fac + 3) / 4));
    void *alpha = take(sizeof(double) * mfit * ld);
    void *covar = take(sizeof(double) * mfit * ld);
    void *beta = take(sizeof(double) * kMaxFit);
    void *da = take(sizeof(double) * kMaxFit);
    void *a = take(sizeof(double) * kMaxPar);
    void *atry = take(sizeof(double) * kMaxPar);
    // the J^T W J tile buffers (phase D) and the basis chunks (phase B) are
    // never live at the same time: one region serves both
    const size_t tsz = align16(sizeof(double) * tr * mfp);
    const size_t rsz = align16(sizeof(double) * tr * rs);
    const size_t csz = align16(sizeof(double4) * tr);
    const size_t tiles = 2 * tsz + 2 * rsz + 2 * csz;
    const size_t chunks = (size_t)kStages * sizeof(double) * chunk_facets(ncp) * ncp;
    unsigned char *un = (unsigned char *)take(tiles > chunks ? tiles : chunks);
    void *rdy = take(sizeof(double) * kTile);
    void *rw = take(sizeof(double) * kTile);
    void *rcoef = take(sizeof(double) * kTile);
    void *rsub = take(sizeof(double) * kTile);
    void *rcur = take(sizeof(int) * kTile);
    void *red = take(sizeof(double) * kWarps * 4);
    void *inv = take(sizeof(double) * 40);
    void *scal = take(sizeof(double) * S_NSCAL);
    void *fidx = take(sizeof(int) * kMaxFit);
    void *ctl = take(sizeof(int) * C_NCTL);
    void *mbar = take(sizeof(unsigned long long) * kStages);
    void *tbar = take(sizeof(unsigned long long) * 2);
    void *tclk = take(sizeof(long long) * (T_NPHASE + 1));
    void *hist = take(sizeof(int) * 2 * kSortCells);
    void *ccoef = take(sizeof(double) * n_curves);
    void *crave = take(sizeof(double) * n_curves);
    // rs = row stride = ma + 1 rounded to even, so ma + 3 <= rs + 2
    void *cst = take(cstat_smem ? sizeof(double) * n_curves * (rs + 2) : 0);
    void *wst = take(mixed ? sizeof(float) * kWarps * 2 * 32 * kWS : sizeof(double) * kWarps * 32 * 4);
    void *f32 = take(mixed ? sizeof(float4) * n_fac : 0);
    void *g32 = take(mixed ? sizeof(float2) * n_fac : 0);
    if (s) {
        s->F = (double4 *)F; s->cone = (float4 *)cone; s->alpha = (double *)alpha; s->covar = (double *)covar;
        s->beta = (double *)beta; s->da = (double *)da; s->a = (double *)a; s->atry = (double *)atry;
        s->T = (double *)un;
        s->TW = (double *)(un + tsz);
        s->raw = (double *)(un + 2 * tsz);
        s->recb = (double4 *)(un + 2 * tsz + 2 * rsz);
        s->ybuf = (double *)un;
        s->rdy = (double *)rdy; s->rw = (double *)rw;
        s->rcoef = (double *)rcoef; s->rsub = (double *)rsub; s->rcur = (int *)rcur;
        s->red = (double *)red; s->inv = (double *)inv; s->scal = (double *)scal;
        s->fidx = (int *)fidx; s->ctl = (int *)ctl;
        s->mbar = (unsigned long long *)mbar; s->tbar = (unsigned long long *)tbar;
        s->tclk = (long long *)tclk; s->hist = (int *)hist;
        s->ccoef = (double *)ccoef; s->crave = (double *)crave; s->cst = (double *)cst;
        s->wst = (double *)wst;
        s->wst32 = (float *)wst;
        s->F32 = (float4 *)f32;
        s->G32 = (float2 *)g32;
        s->ld = ld; s->mfp = mfp; s->tr = tr;
    }
    return off;
}

// ---------------------------------------------------------------- reductions

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Sums up to 4 values over the CTA; every thread gets the totals.
template <int NV>
__device__ __forceinline__ void block_sum(double *v, double *red)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int i = 0; i < NV; ++i) v[i] = warp_sum(v[i]);
    if (lane == 0)
#pragma unroll
        for (int i = 0; i < NV; ++i) red[warp * 4 + i] = v[i];
    __syncthreads();
#pragma unroll
    for (int i = 0; i < NV; ++i) {
        double t = 0;
        for (int w = 0; w < kWarps; ++w) t += red[w * 4 + i];
        v[i] = t;
    }
    __syncthreads();
}

// ---------------------------------------------------------------- curv

// Facet areas at parameter vector a (1-based, shared memory).  Returns the sum.
static __device__ double shape_areas(const DevObject &o, const Sh &s, const double *a)
{
    double part = 0;
    const int nc = o.n_coef;
    for (int f = threadIdx.x; f < o.n_fac; f += kThreads) {
        const double *y = o.ysh + (size_t)f * o.ncp;
        double g = 0;
        for (int k = 0; k < nc; ++k) g += a[k + 1] * __ldg(y + k);
        double ar = __ldg(&o.facet[f].w) * exp(g);
        s.F[f].w = ar;
        part += ar;
    }
    double v[1] = {part};
    block_sum<1>(v, s.red);
    return v[0];
}

// Bounding cone of each group of 4 consecutive facets (the facet sweep's
// step): axis c = normalised sum of the normals, half-angle t = the largest
// angle between c and a normal.  A unit normal n within t of c has
// n.e <= cos(angle(c, e) - t), so c.e <= -sin t rules out n.e > 0 for every
// facet of the group; the sweep skips a group when that holds for every lane
// and for e or e0.  The sine is stored with a margin of 1e-5 that covers the
// FP32 rounding of the test (|error| < 1e-6 for unit vectors); a group wider
// than a hemisphere always passes.  Reads the object's facet table.
static __device__ void facet_cones(const DevObject &o, const Sh &s)
{
    const int ng = (o.n_fac + 3) >> 2;
    for (int g = threadIdx.x; g < ng; g += kThreads) {
        const int f0 = 4 * g, nq = min(4, o.n_fac - f0);
        double4 n[4];
        double cx = 0, cy = 0, cz = 0;
        for (int q = 0; q < nq; ++q) {
            n[q] = ldg4(&o.facet[f0 + q]);
            cx += n[q].x; cy += n[q].y; cz += n[q].z;
        }
        const double len = sqrt(cx * cx + cy * cy + cz * cz);
        float4 c = make_float4(1.f, 0.f, 0.f, 2.f);  // degenerate: always passes
        if (len > 1e-3) {
            cx /= len; cy /= len; cz /= len;
            double cmin = 1.0;
            for (int q = 0; q < nq; ++q) cmin = fmin(cmin, n[q].x * cx + n[q].y * cy + n[q].z * cz);
            if (cmin > 0.0) {
                const double sn = sqrt(fmax(0.0, 1.0 - cmin * cmin));
                c = make_float4((float)cx, (float)cy, (float)cz, (float)(sn + 1e-5));
            }
        }
        s.cone[g] = c;
    }
}

// Per-evaluation invariants from a: phase function, scattering weights and the
// pole rotation B(beta', lambda) with its two derivatives (blmatrix,
// Start.cu:399-417).
static __device__ void set_invariants(const DevObject &o, const DevParams &p, const Sh &s, const double *a)
{
    if (threadIdx.x == 0) {
        const int nc = o.n_coef, ma = o.ma;
        double *v = s.inv;
        double bet = a[nc + 1], lam = a[nc + 2];
        v[0] = a[nc + 3];
        v[1] = p.phi0;
        v[2] = a[nc + 4];
        v[3] = 1.0 / a[nc + 5];
        v[4] = a[nc + 6];
        v[5] = exp(a[ma - 1]);
        v[6] = a[ma];
        double sb, cb, sl, cl;
        sincos(bet, &sb, &cb);
        sincos(lam, &sl, &cl);
        const double B[9] = {cb * cl, cb * sl, -sb, -sl, cl, 0, sb * cl, sb * sl, cb};
        const double Bb[9] = {-sb * cl, -sb * sl, -cb, 0, 0, 0, cb * cl, cb * sl, -sb};
        const double Bl[9] = {-cb * sl, cb * cl, 0, -cl, -sl, 0, -sb * sl, sb * cl, 0};
        for (int i = 0; i < 9; ++i) {
            v[8 + i] = B[i];
            v[17 + i] = Bb[i];
            v[26 + i] = Bl[i];
        }
    }
    __syncthreads();
}

// ---------------------------------------------------------------- phase B

// Body-frame geometry of one point: T = Rz(phi) B(beta', lambda) applied to the
// observer and Sun directions, and (full = true) the derivatives of those
// vectors w.r.t. beta', lambda, omega plus the phase-function terms
// (curve1_point_geometry, Start.cu:2095-2195; ps_phase_mod2pi, Start.cu:687-692).
// B and its derivatives are read from shared memory through volatile loads so
// the compiler cannot keep them live in registers across the facet sweep.
struct PointGeo {
    double e[3], e0[3];
    double db[3], d0b[3], dl[3], d0l[3], dw[2], d0w[2];
    double scale, ff, d2, alph;
};

template <bool FULL>
__device__ __forceinline__ void point_geometry(const double *inv, double t, const double *ee,
                                               const double *es, PointGeo &g)
{
    const volatile double *v = inv;
    const double om = v[0], phi0 = v[1];
    double f = om * t + phi0;
    f = f - 2.0 * kPi * round(f * (1.0 / (2.0 * kPi)));
    double sf, cf;
    sincos(f, &sf, &cf);
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        double Ti[3];
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const double b0 = v[8 + j], b1 = v[11 + j], b2 = v[14 + j];
            Ti[j] = (i == 0) ? cf * b0 + sf * b1 : (i == 1) ? -sf * b0 + cf * b1 : b2;
        }
        g.e[i] = Ti[0] * ee[0] + Ti[1] * ee[1] + Ti[2] * ee[2];
        g.e0[i] = Ti[0] * es[0] + Ti[1] * es[1] + Ti[2] * es[2];
    }
    if (!FULL) return;
    const double A = v[2], rD = v[3], K = v[4];
    double cdot = ((ee[0] * es[0]) + ee[1] * es[1]) + ee[2] * es[2];
    g.alph = acos(fmin(1.0, fmax(-1.0, cdot)));
    g.ff = exp2(-1.44269504088896 * (g.alph * rD));
    g.scale = 1.0 + A * g.ff + K * g.alph;
    g.d2 = A * g.ff * g.alph * (rD * rD);
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        double Tb[3], Tl[3];
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const double b0 = v[17 + j], b1 = v[20 + j], b2 = v[23 + j];
            const double l0 = v[26 + j], l1 = v[29 + j], l2 = v[32 + j];
            Tb[j] = (i == 0) ? cf * b0 + sf * b1 : (i == 1) ? -sf * b0 + cf * b1 : b2;
            Tl[j] = (i == 0) ? cf * l0 + sf * l1 : (i == 1) ? -sf * l0 + cf * l1 : l2;
        }
        g.db[i] = Tb[0] * ee[0] + Tb[1] * ee[1] + Tb[2] * ee[2];
        g.d0b[i] = Tb[0] * es[0] + Tb[1] * es[1] + Tb[2] * es[2];
        g.dl[i] = Tl[0] * ee[0] + Tl[1] * ee[1] + Tl[2] * ee[2];
        g.d0l[i] = Tl[0] * es[0] + Tl[1] * es[1] + Tl[2] * es[2];
    }
#pragma unroll
    for (int i = 0; i < 2; ++i) {
        double To[3];
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const double b0 = v[8 + j], b1 = v[11 + j];
            To[j] = (i == 0) ? (-sf * t) * b0 + (cf * t) * b1 : (-cf * t) * b0 + (-sf * t) * b1;
        }
        g.dw[i] = To[0] * ee[0] + To[1] * ee[1] + To[2] * ee[2];
        g.d0w[i] = To[0] * es[0] + To[1] * es[1] + To[2] * es[2];
    }
}

// Order of the points for the facet sweep: counting sort on the body-frame
// direction of the Sun-observer bisector, so the 32 points of a warp see
// nearly the same facets and whole warps skip facets none of them sees.  Rows
// are written at the original point index and every skipped term is an exact
// zero, so the order changes nothing in the results.
static __device__ void sort_points(const DevObject &o, const Sh &s, int *perm, int *keys)
{
    const int tid = threadIdx.x, np = o.n_points;
    int *hist = s.hist, *offs = s.hist + kSortCells;
    for (int c = tid; c < kSortCells; c += kThreads) hist[c] = 0;
    __syncthreads();
    for (int q = tid; q < np; q += kThreads) {
        const double4 pa = ldg4(&o.pt_a[q]);
        const double4 pb = ldg4(&o.pt_b[q]);
        const double ee[3] = {pa.y, pa.z, pa.w}, es[3] = {pb.x, pb.y, pb.z};
        PointGeo g;
        point_geometry<false>(s.inv, pa.x, ee, es, g);
        const double bx = g.e[0] + g.e0[0], by = g.e[1] + g.e0[1], bz = g.e[2] + g.e0[2];
        const double n = sqrt(bx * bx + by * by + bz * bz);
        const double cz = n > 0 ? bz / n : 0.0;
        int band = (int)((cz + 1.0) * (0.5 * kSortBands));
        band = min(max(band, 0), kSortBands - 1);
        // pseudo-angle of (bx, by) in [0, 4): monotone in longitude, no trig
        const double ax = fabs(bx), ay = fabs(by), sum = ax + ay;
        double pa4 = sum > 0 ? ay / sum : 0.0;
        if (bx < 0) pa4 = 2.0 - pa4;
        if (by < 0) pa4 = 4.0 - pa4;
        int sec = (int)(pa4 * (0.25 * kSortSectors));
        sec = min(max(sec, 0), kSortSectors - 1);
        const int key = band * kSortSectors + ((band & 1) ? kSortSectors - 1 - sec : sec);
        keys[q] = key;
        atomicAdd(&hist[key], 1);
    }
    __syncthreads();
    if (threadIdx.x < 32) {
        const int lane = threadIdx.x, per = kSortCells / 32;
        int local[kSortCells / 32], sum = 0;
#pragma unroll
        for (int i = 0; i < per; ++i) {
            local[i] = hist[lane * per + i];
            sum += local[i];
        }
        int incl = sum;
#pragma unroll
        for (int o2 = 1; o2 < 32; o2 <<= 1) {
            const int v = __shfl_up_sync(0xffffffffu, incl, o2);
            if (lane >= o2) incl += v;
        }
        int run = incl - sum;
#pragma unroll
        for (int i = 0; i < per; ++i) {
            offs[lane * per + i] = run;
            run += local[i];
        }
    }
    __syncthreads();
    for (int q = tid; q < np; q += kThreads) perm[atomicAdd(&offs[keys[q]], 1)] = q;
    __syncthreads();
}

// Brightness and raw derivative rows of all points: mrqcof_curve1_opt
// (Start.cu:2262-2535).  Row layout: column p-1 = d ymod / d a_p for
// p = 1..ma, column ma = ymod (un-renormalised).
//
__device__ __forceinline__ void dmma_8x8x4(double &d0, double &d1, double a, double b)
{
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

// The facet sweep is a kStages-deep pipeline of basis chunks (chunk_facets
// facets x ncp doubles each) that the bulk-copy engine brings into shared
// memory.  Every warp walks the same chunk sequence; the last warp to finish
// with a buffer issues the copy of the chunk kStages ahead into it, so warps
// drift apart by up to kStages - 1 chunks instead of meeting at a CTA barrier
// per chunk.
//
// One warp = 32 points.  Per facet, lane = point computes visibility, the
// Lambert + Lommel-Seeliger terms and the rotation-derivative sums; whole
// facets no lane sees are skipped.  The shape derivatives
//     J[p][k] = sum_f w[p][f] Y[f][k],   w[p][f] = Areag_f s(mu, mu0)
// are a GEMM: each group of 4 facets is one k-step of FP64 tensor-core
// MMAs (m8n8k4), A = w (8 points x 4 facets, staged through a per-warp
// shared-memory tile), B = the basis chunk (4 facets x 8 coefficients),
// accumulators [4 point blocks][ncp / 8 coefficient blocks] in registers.
//
// When the last coefficient block holds a single coefficient (n_coef = 8k + 1:
// every lmax = mmax model with lmax even, e.g. 25, 49, 81 coefficients), that
// coefficient runs on the FP64 FMA pipe instead (lane = point, four FMAs per
// step) and the block's MMAs are skipped: they would spend 8 columns of tensor
// work on one.  The lane's accumulator is element C[0][NT - 1][0], which the
// skipped MMAs leave free.
template <int NCP, bool X1>
__device__ void brightness_rows(const DevObject &o, const Sh &s, double *rows, const int *perm)
{
    constexpr int NT = NCP / 8;
    constexpr int NTM = X1 ? NT - 1 : NT;  // coefficient blocks on the tensor cores
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int np = o.n_points, nf = o.n_fac, nc = o.n_coef;
    const double cl = s.inv[5], cls = s.inv[6];
    const int fc = chunk_facets(NCP);
    const int nchunks = (nf + fc - 1) / fc;
    const int ntiles = (np + 31) / 32;
    const int nrounds = (ntiles + kWarps - 1) / kWarps;
    const int total = nrounds * nchunks;
    double *wt = s.wst + warp * 32 * 4;
    bool timeout = false;

    auto issue = [&](int g) {
        const int c = g % nchunks, f0 = c * fc;
        const int rows_c = min(fc, nf - f0);
        const int b = g % kStages;
        bulk_load(s.ybuf + (size_t)b * fc * NCP, o.ysh + (size_t)f0 * NCP,
                  (uint32_t)(rows_c * NCP * sizeof(double)), &s.mbar[b]);
    };
    if (tid == 0)
        for (int g = 0; g < kStages && g < total; ++g) issue(g);

    int g = 0;
    for (int round = 0; round < nrounds; ++round) {
        const int tile = round * kWarps + warp;
        const bool tile_act = tile < ntiles;
        const int idx = tile * 32 + lane;
        const bool act = tile_act && idx < np;
        const int p = perm[min(idx, np - 1)];
        double ex, ey, ez, sx, sy, sz;
        {
            const double4 pa = ldg4(&o.pt_a[p]);
            const double4 pb = ldg4(&o.pt_b[p]);
            const double ee[3] = {pa.y, pa.z, pa.w}, es[3] = {pb.x, pb.y, pb.z};
            PointGeo geo;
            point_geometry<false>(s.inv, pa.x, ee, es, geo);
            ex = geo.e[0]; ey = geo.e[1]; ez = geo.e[2];
            sx = geo.e0[0]; sy = geo.e0[1]; sz = geo.e0[2];
        }

        double C[4][NT][2];
#pragma unroll
        for (int m = 0; m < 4; ++m)
#pragma unroll
            for (int n = 0; n < NT; ++n) C[m][n][0] = C[m][n][1] = 0.0;
        double br = 0, u0 = 0, u1 = 0, u2 = 0, w0 = 0, w1 = 0, w2 = 0, t4 = 0, t5 = 0;

        // Lambert + Lommel-Seeliger terms of facets k0..k0+3 of the chunk for
        // this lane's point: the rotation sums, the brightness and the facet
        // weights wk (the MMA's A operand); with X1 also the single last
        // coefficient.  Lanes that do not see a facet run the same arithmetic
        // on finite stand-ins and contribute exact zeros.
        auto facet_terms = [&](int f0, int nfc, const double *yb, int k0, double (&wk)[4]) {
            double4 fr[4];
            double mu[4], mu0[4];
            bool vis[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const bool inside = k0 + q < nfc;
                fr[q] = s.F[f0 + (inside ? k0 + q : 0)];
                mu[q] = ex * fr[q].x + ey * fr[q].y + ez * fr[q].z;
                mu0[q] = sx * fr[q].x + sy * fr[q].y + sz * fr[q].z;
                vis[q] = act && inside && (mu[q] > kTiny) && (mu0[q] > kTiny);
            }
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const double ar = vis[q] ? fr[q].w : 0.0;
                const double r = rcp_nr(vis[q] ? mu[q] + mu0[q] : 1.0);
                const double sv = mu[q] * mu0[q] * (cl + cls * r);
                const double q0 = mu0[q] * r, q1 = mu[q] * r;
                const double dsmu = cls * (q0 * q0) + cl * mu0[q];
                const double dsmu0 = cls * (q1 * q1) + cl * mu[q];
                const double amm = ar * mu[q] * mu0[q];
                const double w = ar * sv;
                const double gg = ar * dsmu;
                const double g0 = ar * dsmu0;
                br += w;
                u0 = fma(gg, fr[q].x, u0);
                u1 = fma(gg, fr[q].y, u1);
                u2 = fma(gg, fr[q].z, u2);
                w0 = fma(g0, fr[q].x, w0);
                w1 = fma(g0, fr[q].y, w1);
                w2 = fma(g0, fr[q].z, w2);
                t4 += amm;
                t5 += amm * r;
                wk[q] = w;
            }
            if constexpr (X1) {
                // the single last coefficient, lane = point
                const double *yl = yb + (size_t)k0 * NCP + 8 * (NT - 1);
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const double y = (k0 + q < nfc) ? yl[(size_t)q * NCP] : 0.0;
                    C[0][NT - 1][0] = fma(wk[q], y, C[0][NT - 1][0]);
                }
            }
        };
        // The weights of one group through the warp's shared-memory tile into
        // the m8n8k4 A fragments: a[m] = w[point 8m + lane/4][facet lane%4].
        auto stage = [&](const double (&wk)[4], double (&a)[4]) {
            __syncwarp();  // every lane has read the previous group's tile
            reinterpret_cast<double2 *>(wt)[2 * lane] = make_double2(wk[0], wk[1]);
            reinterpret_cast<double2 *>(wt)[2 * lane + 1] = make_double2(wk[2], wk[3]);
            __syncwarp();
#pragma unroll
            for (int m = 0; m < 4; ++m) a[m] = wt[(8 * m + (lane >> 2)) * 4 + (lane & 3)];
        };
        // One k-step of the shape-derivative GEMM: facets kp..kp+3 of the chunk.
        auto mma_step = [&](const double *yb, int nfc, int kp, const double (&a)[4]) {
            // B row = facet kp + (lane & 3); rows past the chunk's end hold
            // stale data and must contribute zeros
            const bool brow = kp + (lane & 3) < nfc;
            const double *yr = yb + (size_t)(kp + (lane & 3)) * NCP + (lane >> 2);
#pragma unroll
            for (int n = 0; n < NTM; ++n) {
                const double bv = brow ? yr[8 * n] : 0.0;
#pragma unroll
                for (int m = 0; m < 4; ++m) dmma_8x8x4(C[m][n][0], C[m][n][1], a[m], bv);
            }
        };

        for (int c = 0; c < nchunks; ++c, ++g) {
            const int b = g % kStages;
            const int use = s.ctl[C_YUSE + b] + g / kStages;  // phase parity of this fill
            if (!mbar_wait(&s.mbar[b], (uint32_t)(use & 1))) timeout = true;
            if (tile_act) {
                const int f0 = c * fc, nfc = min(fc, nf - f0);
                const double *yb = s.ybuf + (size_t)b * fc * NCP;
                // the chunk's 4-facet groups that some lane may see: a bounding-cone
                // test per group in FP32 (necessary for visibility, see facet_cones);
                // the groups it rules out would add exact zeros
                unsigned gmask = 0;
                if (act) {
                    const float ex32 = (float)ex, ey32 = (float)ey, ez32 = (float)ez;
                    const float sx32 = (float)sx, sy32 = (float)sy, sz32 = (float)sz;
                    const float4 *cg = s.cone + (f0 >> 2);
#pragma unroll
                    for (int q = 0; q < kMaxChunkGroups; ++q) {
                        if (4 * q < nfc) {
                            const float4 cn = cg[q];
                            const float ce = fmaf(ez32, cn.z, fmaf(ey32, cn.y, ex32 * cn.x));
                            const float c0 = fmaf(sz32, cn.z, fmaf(sy32, cn.y, sx32 * cn.x));
                            if (ce > -cn.w && c0 > -cn.w) gmask |= 1u << q;
                        }
                    }
                }
                gmask = __reduce_or_sync(0xffffffffu, gmask);
                // Software pipeline over the chunk's groups: the facet terms of
                // group k0 and the tensor-core step of the group before it (A
                // fragments already in registers) form one branch-free stretch, so
                // each warp always has FP64 FMA and MMA work ready to interleave.
                // Groups the cone test passes but no lane sees add exact zeros.
                if (gmask) {
                    double a[4], wk[4];
                    int k0 = 4 * (__ffs(gmask) - 1);
                    gmask &= gmask - 1;
                    facet_terms(f0, nfc, yb, k0, wk);
                    stage(wk, a);
                    int kp = k0;
#pragma unroll 1
                    while (gmask) {
                        k0 = 4 * (__ffs(gmask) - 1);
                        gmask &= gmask - 1;
                        facet_terms(f0, nfc, yb, k0, wk);
                        mma_step(yb, nfc, kp, a);
                        stage(wk, a);
                        kp = k0;
                    }
                    mma_step(yb, nfc, kp, a);
                }
            }
            // release the buffer; the last of the kWarps warps refills it
            __syncwarp();
            if (lane == 0) {
                __threadfence_block();
                if (atomicAdd(&s.ctl[C_REL + b], 1) == kWarps - 1) {
                    s.ctl[C_REL + b] = 0;
                    if (g + kStages < total) issue(g + kStages);
                }
            }
        }

        if (tile_act) {
            const double4 pa = ldg4(&o.pt_a[p]);
            const double4 pb = ldg4(&o.pt_b[p]);
            const double ee[3] = {pa.y, pa.z, pa.w}, es[3] = {pb.x, pb.y, pb.z};
            PointGeo geo;
            point_geometry<true>(s.inv, pa.x, ee, es, geo);
            const double t1 = (geo.db[0] * u0 + geo.db[1] * u1 + geo.db[2] * u2) +
                              (geo.d0b[0] * w0 + geo.d0b[1] * w1 + geo.d0b[2] * w2);
            const double t2 = (geo.dl[0] * u0 + geo.dl[1] * u1 + geo.dl[2] * u2) +
                              (geo.d0l[0] * w0 + geo.d0l[1] * w1 + geo.d0l[2] * w2);
            const double t3 = (geo.dw[0] * u0 + geo.dw[1] * u1) + (geo.d0w[0] * w0 + geo.d0w[1] * w1);
            const double scale = geo.scale;
            if (act) {
                double *row = rows + (size_t)p * o.row_stride;
                if constexpr (X1) row[nc - 1] = scale * C[0][NT - 1][0];
                row[nc + 0] = scale * t1;
                row[nc + 1] = scale * t2;
                row[nc + 2] = scale * t3;
                row[nc + 3] = br * geo.ff;
                row[nc + 4] = br * geo.d2;
                row[nc + 5] = br * geo.alph;
                row[nc + 6] = scale * t4 * cl;
                row[nc + 7] = scale * t5;
                row[nc + 8] = br * scale;
            }
            // shape columns from the MMA accumulators: element (m, n, e) of this
            // lane is point 8m + lane/4 of the tile, coefficient 8n + 2(lane%4) + e
#pragma unroll
            for (int m = 0; m < 4; ++m) {
                const int src = 8 * m + (lane >> 2);
                const int pm = __shfl_sync(0xffffffffu, p, src);
                const double sm = __shfl_sync(0xffffffffu, scale, src);
                const bool am = __shfl_sync(0xffffffffu, act ? 1 : 0, src) != 0;
                if (!am) continue;
                double *row = rows + (size_t)pm * o.row_stride;
#pragma unroll
                for (int n = 0; n < NT; ++n) {
                    if (n >= NTM) break;
                    const int k = 8 * n + 2 * (lane & 3);
                    if (k + 1 < nc)
                        *reinterpret_cast<double2 *>(row + k) = make_double2(sm * C[m][n][0], sm * C[m][n][1]);
                    else if (k < nc)
                        row[k] = sm * C[m][n][0];
                }
            }
        }
    }
    if (timeout) s.ctl[C_TIMEOUT] = 1;
    __syncthreads();
    // per-buffer fill counts carry the mbarrier phases into the next evaluation
    if (tid == 0) {
        for (int b = 0; b < kStages; ++b) {
            const int uses_b = (total > b) ? (total - b + kStages - 1) / kStages : 0;
            s.ctl[C_YUSE + b] += uses_b;
        }
    }
}

// ---------------------------------------------------------------- phase B, mixed precision

__device__ __forceinline__ uint32_t tf32_rna(float x)
{
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return r;
}

// FP32 reciprocal: the special-function unit's approximation refined by one
// Newton-Raphson step, r1 = r0 + r0 (1 - x r0), which brings its relative
// error from about 2^-23 to the last bit or two of FP32.
__device__ __forceinline__ float rcp_f32(float x)
{
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    const float e = fmaf(-x, r, 1.0f);
    return fmaf(r, e, r);
}

// D += A B on the tensor cores, m16n8k8, TF32 operands, FP32 accumulation.
__device__ __forceinline__ void mma_tf32(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1)
{
    asm volatile("mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
                 "{%0,%1,%2,%3};"
                 : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
                 : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// The facet sweep in mixed precision: the point geometry and the output rows
// stay FP64; the per-facet Lambert + Lommel-Seeliger terms run in FP32 (with
// a Newton-refined reciprocal) and the per-point sums of each 8-facet step
// are flushed into FP64 accumulators, so no FP32 sum runs over more than 8
// terms; the shape
// derivatives J = W Y run on the tensor cores as 3xTF32 products
// (W_lo Y_hi + W_hi Y_lo + W_hi Y_hi, each operand split into a TF32 high
// part and a TF32 remainder) with FP32 accumulation.  The chunk pipeline is
// the FP64 sweep's; a chunk holds the basis as [hi | lo][chunk_facets][ncp]
// floats, zero-padded past the last facet.  One warp = 32 points, steps of 8
// facets (the MMA's k); a step no lane sees is skipped whole, a 16-point half
// that sees none of its 8 facets skips its MMAs.
template <int NCP>
__device__ void brightness_rows_mixed(const DevObject &o, const Sh &s, double *rows, const int *perm)
{
    constexpr int NT = NCP / 8;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, t = lane & 3;
    const int np = o.n_points, nf = o.n_fac, nc = o.n_coef;
    const float cl = (float)s.inv[5], cls = (float)s.inv[6];
    const int fc = chunk_facets(NCP);
    const int nchunks = (nf + fc - 1) / fc;
    const int ntiles = (np + 31) / 32;
    const int nrounds = (ntiles + kWarps - 1) / kWarps;
    const int total = nrounds * nchunks;
    float *whi = s.wst32 + warp * 2 * 32 * kWS;
    float *wlo = whi + 32 * kWS;
    float *ybuf = reinterpret_cast<float *>(s.ybuf);
    bool timeout = false;

    auto issue = [&](int gg) {
        const int c = gg % nchunks;
        const int b = gg % kStages;
        bulk_load(ybuf + (size_t)b * 2 * fc * NCP, o.ysh32 + (size_t)c * 2 * fc * NCP,
                  (uint32_t)(2 * fc * NCP * sizeof(float)), &s.mbar[b]);
    };
    if (tid == 0)
        for (int gg = 0; gg < kStages && gg < total; ++gg) issue(gg);

    int gi = 0;
    for (int round = 0; round < nrounds; ++round) {
        const int tile = round * kWarps + warp;
        const bool tile_act = tile < ntiles;
        const int idx = tile * 32 + lane;
        const bool act = tile_act && idx < np;
        const int p = perm[min(idx, np - 1)];
        float ex, ey, ez, sx, sy, sz;
        {
            const double4 pa = ldg4(&o.pt_a[p]);
            const double4 pb = ldg4(&o.pt_b[p]);
            const double ee[3] = {pa.y, pa.z, pa.w}, es[3] = {pb.x, pb.y, pb.z};
            PointGeo geo;
            point_geometry<false>(s.inv, pa.x, ee, es, geo);
            ex = (float)geo.e[0]; ey = (float)geo.e[1]; ez = (float)geo.e[2];
            sx = (float)geo.e0[0]; sy = (float)geo.e0[1]; sz = (float)geo.e0[2];
        }

        float C[2][NT][4];
#pragma unroll
        for (int m = 0; m < 2; ++m)
#pragma unroll
            for (int n = 0; n < NT; ++n) C[m][n][0] = C[m][n][1] = C[m][n][2] = C[m][n][3] = 0.0f;
        // br, u0..u2, w0..w2, t4, t5 in FP64, fed by FP32 chunk partial sums
        double S64[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};

        for (int c = 0; c < nchunks; ++c, ++gi) {
            const int b = gi % kStages;
            const int use = s.ctl[C_YUSE + b] + gi / kStages;  // phase parity of this fill
            if (!mbar_wait(&s.mbar[b], (uint32_t)(use & 1))) timeout = true;
            if (tile_act) {
                const int f0 = c * fc, nfc = min(fc, nf - f0);
                const float *yh = ybuf + (size_t)b * 2 * fc * NCP;
                const float *yl = yh + fc * NCP;
#pragma unroll 1
                for (int k0 = 0; k0 < nfc; k0 += 8) {
                    // visibility of the step's 8 facets, one vote
                    float mu[8], mu0[8];
                    bool vis[8];
                    bool v8 = false;
#pragma unroll
                    for (int q = 0; q < 8; ++q) {
                        const bool inside = k0 + q < nfc;
                        const float4 fr = s.F32[f0 + (inside ? k0 + q : 0)];
                        mu[q] = ex * fr.x + ey * fr.y + ez * fr.z;
                        mu0[q] = sx * fr.x + sy * fr.y + sz * fr.z;
                        vis[q] = act && inside && (mu[q] > (float)kTiny) && (mu0[q] > (float)kTiny);
                        v8 = v8 || vis[q];
                    }
                    const unsigned vm = __ballot_sync(0xffffffffu, v8);
                    if (!vm) continue;  // warp-uniform
                    float S[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
                    uint32_t hi[8], lo[8];
#pragma unroll
                    for (int q = 0; q < 8; ++q) {
                        // lanes that do not see the facet take mu = mu0 = 0, which zeroes
                        // every term they add; with a = area, L = a cl, S = a cls and
                        // r = 1 / (mu + mu0):
                        //   w  = a mu mu0 (cl + cls r)            (brightness term)
                        //   gg = mu0 (S mu0 r^2 + L) = a dS/dmu,  g0 = mu (S mu r^2 + L)
                        const int fq = f0 + (k0 + q < nfc ? k0 + q : 0);
                        const float4 fr = s.F32[fq];
                        const float2 ls = s.G32[fq];
                        const float mv = vis[q] ? mu[q] : 0.0f, m0v = vis[q] ? mu0[q] : 0.0f;
                        const float r = rcp_f32(vis[q] ? mu[q] + mu0[q] : 1.0f);
                        const float z = fr.w * (mv * m0v);
                        const float zr = z * r;
                        const float w = fmaf(cls, zr, cl * z);
                        const float y = ls.y * r;
                        const float gg = m0v * fmaf(y * m0v, r, ls.x);
                        const float g0 = mv * fmaf(y * mv, r, ls.x);
                        S[0] += w;
                        S[1] = fmaf(gg, fr.x, S[1]);
                        S[2] = fmaf(gg, fr.y, S[2]);
                        S[3] = fmaf(gg, fr.z, S[3]);
                        S[4] = fmaf(g0, fr.x, S[4]);
                        S[5] = fmaf(g0, fr.y, S[5]);
                        S[6] = fmaf(g0, fr.z, S[6]);
                        S[7] += z;
                        S[8] += zr;
                        hi[q] = tf32_rna(w);
                        lo[q] = tf32_rna(w - __uint_as_float(hi[q]));
                    }
#pragma unroll
                    for (int i = 0; i < 9; ++i) S64[i] += (double)S[i];
                    // this lane's row of the step's weight tile, high and low parts
                    uint4 *ph = reinterpret_cast<uint4 *>(whi + lane * kWS);
                    uint4 *pl = reinterpret_cast<uint4 *>(wlo + lane * kWS);
                    ph[0] = make_uint4(hi[0], hi[1], hi[2], hi[3]);
                    ph[1] = make_uint4(hi[4], hi[5], hi[6], hi[7]);
                    pl[0] = make_uint4(lo[0], lo[1], lo[2], lo[3]);
                    pl[1] = make_uint4(lo[4], lo[5], lo[6], lo[7]);
                    __syncwarp();
                    // A fragments: rows = points 16m + g (+8), columns = facets t (+4)
                    uint32_t ah[2][4], al[2][4];
#pragma unroll
                    for (int m = 0; m < 2; ++m) {
                        const int r0 = (16 * m + g) * kWS + t, r1 = r0 + 8 * kWS;
                        ah[m][0] = __float_as_uint(whi[r0]);
                        ah[m][1] = __float_as_uint(whi[r1]);
                        ah[m][2] = __float_as_uint(whi[r0 + 4]);
                        ah[m][3] = __float_as_uint(whi[r1 + 4]);
                        al[m][0] = __float_as_uint(wlo[r0]);
                        al[m][1] = __float_as_uint(wlo[r1]);
                        al[m][2] = __float_as_uint(wlo[r0 + 4]);
                        al[m][3] = __float_as_uint(wlo[r1 + 4]);
                    }
                    const bool mt0 = (vm & 0xffffu) != 0, mt1 = (vm >> 16) != 0;
                    // B fragments: rows = facets k0 + t (+4), columns = coefficients 8n + g
                    const float *bh = yh + (k0 + t) * NCP + g;
                    const float *bl = yl + (k0 + t) * NCP + g;
#pragma unroll
                    for (int n = 0; n < NT; ++n) {
                        const uint32_t b0h = __float_as_uint(bh[8 * n]), b1h = __float_as_uint(bh[4 * NCP + 8 * n]);
                        const uint32_t b0l = __float_as_uint(bl[8 * n]), b1l = __float_as_uint(bl[4 * NCP + 8 * n]);
                        if (mt0) {
                            mma_tf32(C[0][n], al[0], b0h, b1h);
                            mma_tf32(C[0][n], ah[0], b0l, b1l);
                            mma_tf32(C[0][n], ah[0], b0h, b1h);
                        }
                        if (mt1) {
                            mma_tf32(C[1][n], al[1], b0h, b1h);
                            mma_tf32(C[1][n], ah[1], b0l, b1l);
                            mma_tf32(C[1][n], ah[1], b0h, b1h);
                        }
                    }
                    __syncwarp();
                }
            }
            // release the buffer; the last of the kWarps warps refills it
            __syncwarp();
            if (lane == 0) {
                __threadfence_block();
                if (atomicAdd(&s.ctl[C_REL + b], 1) == kWarps - 1) {
                    s.ctl[C_REL + b] = 0;
                    if (gi + kStages < total) issue(gi + kStages);
                }
            }
        }

        if (tile_act) {
            const double4 pa = ldg4(&o.pt_a[p]);
            const double4 pb = ldg4(&o.pt_b[p]);
            const double ee[3] = {pa.y, pa.z, pa.w}, es[3] = {pb.x, pb.y, pb.z};
            PointGeo geo;
            point_geometry<true>(s.inv, pa.x, ee, es, geo);
            const double br = S64[0], u0 = S64[1], u1 = S64[2], u2 = S64[3];
            const double w0 = S64[4], w1 = S64[5], w2 = S64[6], t4 = S64[7], t5 = S64[8];
            const double t1 = (geo.db[0] * u0 + geo.db[1] * u1 + geo.db[2] * u2) +
                              (geo.d0b[0] * w0 + geo.d0b[1] * w1 + geo.d0b[2] * w2);
            const double t2 = (geo.dl[0] * u0 + geo.dl[1] * u1 + geo.dl[2] * u2) +
                              (geo.d0l[0] * w0 + geo.d0l[1] * w1 + geo.d0l[2] * w2);
            const double t3 = (geo.dw[0] * u0 + geo.dw[1] * u1) + (geo.d0w[0] * w0 + geo.d0w[1] * w1);
            const double scale = geo.scale;
            if (act) {
                double *row = rows + (size_t)p * o.row_stride;
                row[nc + 0] = scale * t1;
                row[nc + 1] = scale * t2;
                row[nc + 2] = scale * t3;
                row[nc + 3] = br * geo.ff;
                row[nc + 4] = br * geo.d2;
                row[nc + 5] = br * geo.alph;
                row[nc + 6] = scale * t4 * s.inv[5];
                row[nc + 7] = scale * t5;
                row[nc + 8] = br * scale;
            }
            // shape columns from the accumulators: element (m, n, e) of this lane
            // is point 16m + g (+8 for e >= 2), coefficient 8n + 2t + (e & 1)
#pragma unroll
            for (int m = 0; m < 2; ++m)
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int src = 16 * m + g + 8 * h;
                    const int pm = __shfl_sync(0xffffffffu, p, src);
                    const double sm = __shfl_sync(0xffffffffu, scale, src);
                    const bool am = __shfl_sync(0xffffffffu, act ? 1 : 0, src) != 0;
                    if (!am) continue;
                    double *row = rows + (size_t)pm * o.row_stride;
#pragma unroll
                    for (int n = 0; n < NT; ++n) {
                        const int k = 8 * n + 2 * t;
                        const double v0 = sm * (double)C[m][n][2 * h], v1 = sm * (double)C[m][n][2 * h + 1];
                        if (k + 1 < nc)
                            *reinterpret_cast<double2 *>(row + k) = make_double2(v0, v1);
                        else if (k < nc)
                            row[k] = v0;
                    }
                }
        }
    }
    if (timeout) s.ctl[C_TIMEOUT] = 1;
    __syncthreads();
    // per-buffer fill counts carry the mbarrier phases into the next evaluation
    if (tid == 0) {
        for (int b = 0; b < kStages; ++b) {
            const int uses_b = (total > b) ? (total - b + kStages - 1) / kStages : 0;
            s.ctl[C_YUSE + b] += uses_b;
        }
    }
}

// ---------------------------------------------------------------- phases C, D

// J^T W J, J^T W dy and chi^2 as one symmetric rank-k update of the augmented
// matrix [J | dy] on the FP64 tensor cores (mma.sync m8n8k4 .f64):
//   C = A B,  A[j][r] = TW[r][j] = J[r][j] w_r,  B[r][k] = T[r][k] = J[r][k],
// with column mfit of T holding dy_r and of TW holding dy_r w_r, so
//   C[j][k] = alpha_jk,  C[mfit][k] = beta_k,  C[mfit][mfit] = chi^2.
// Only lower-triangle 8x8 blocks are computed; warps own blocks round-robin
// and keep their accumulators in registers for the whole evaluation.
constexpr int kSliceBlk = 36;  // k-slice mode: all 8 x 9 / 2 lower blocks of a <= 64-wide matrix
constexpr int kMaxBlk = 10;    // block mode: ceil(78 / 8) blocks per warp for <= 96-wide matrices

// Two ways to spread the augmented rank-k update over the 8 warps:
//  * k-slice mode (<= 8 x 8 blocks): warp w takes rows 4w..4w+3 of every tile
//    and updates every lower block with them, so each A / B fragment is
//    loaded once per k-step and reused by up to 8 MMAs; the 8 partial sums
//    are added in warp order at the end.
//  * block mode (larger models): warps own blocks round-robin over all rows.
struct SyrkAcc {
    double c[kSliceBlk][2];
    int nb;       // blocks per dimension
    int slice;    // 1: k-slice mode
    int bj[kMaxBlk], bk[kMaxBlk], nblk;   // block mode
};

__device__ __forceinline__ void syrk_init(int mfit, int tile_rows, SyrkAcc &acc)
{
    const int warp = threadIdx.x >> 5;
    acc.nb = fit_mpad(mfit) / 8;
    acc.slice = (acc.nb <= 8 && tile_rows == 4 * kWarps) ? 1 : 0;
    const int nblocks = acc.nb * (acc.nb + 1) / 2;
    acc.nblk = 0;
#pragma unroll
    for (int i = 0; i < kMaxBlk; ++i) {
        const int b = warp + i * kWarps;
        int bj = 0;
        while ((bj + 1) * (bj + 2) / 2 <= b) ++bj;
        acc.bj[i] = bj;
        acc.bk[i] = b - bj * (bj + 1) / 2;
        if (b < nblocks) acc.nblk = i + 1;
    }
#pragma unroll
    for (int i = 0; i < kSliceBlk; ++i) acc.c[i][0] = acc.c[i][1] = 0.0;
}

// Accumulates one staged tile (rows 0..nrows-1 of T/TW, zero beyond).
__device__ __forceinline__ void syrk_update(const Sh &s, int nrows, SyrkAcc &acc)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int S = s.mfp;
    const int kq = lane & 3, cq = lane >> 2;
    if (acc.slice) {
        const int r0 = 4 * warp;
        if (r0 >= nrows) return;
        const double *tw = s.TW + (r0 + kq) * S + cq;
        const double *tt = s.T + (r0 + kq) * S + cq;
        double a[8], b[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            a[q] = (q < acc.nb) ? tw[8 * q] : 0.0;
            b[q] = (q < acc.nb) ? tt[8 * q] : 0.0;
        }
#pragma unroll
        for (int bj = 0; bj < 8; ++bj)
#pragma unroll
            for (int bk = 0; bk <= bj; ++bk)
                if (bj < acc.nb) {
                    const int i = bj * (bj + 1) / 2 + bk;
                    dmma_8x8x4(acc.c[i][0], acc.c[i][1], a[bj], b[bk]);
                }
        return;
    }
    for (int r0 = 0; r0 < nrows; r0 += 4) {
        const double *tw = s.TW + (r0 + kq) * S + cq;
        const double *tt = s.T + (r0 + kq) * S + cq;
#pragma unroll
        for (int i = 0; i < kMaxBlk; ++i)
            if (i < acc.nblk) dmma_8x8x4(acc.c[i][0], acc.c[i][1], tw[8 * acc.bj[i]], tt[8 * acc.bk[i]]);
    }
}

// Adds one warp's accumulators into alpha (lower triangle mirrored, stride
// ld), beta and chi^2.
__device__ __forceinline__ void syrk_add_block(const Sh &s, int mfit, int bj, int bk, double v0, double v1,
                                               double *dst, double *dvec, bool first)
{
    const int lane = threadIdx.x & 31, ld = s.ld;
#pragma unroll
    for (int e = 0; e < 2; ++e) {
        const int row = 8 * bj + (lane >> 2);
        const int col = 8 * bk + 2 * (lane & 3) + e;
        const double v = e ? v1 : v0;
        if (row < mfit && col <= row) {
            const double t = first ? v : dst[row * ld + col] + v;
            dst[row * ld + col] = t;
            if (col != row) dst[col * ld + row] = t;
        } else if (row == mfit && col < mfit) {
            dvec[col] = first ? v : dvec[col] + v;
        } else if (row == mfit && col == mfit) {
            s.scal[S_TRIAL] = first ? v : s.scal[S_TRIAL] + v;
        }
    }
}

// Writes the accumulated alpha, beta and chi^2 (all threads call this).  In
// k-slice mode the 8 warps' partial sums go through a scratch slab (L2) and
// are added in warp order, element by element, by all threads.
__device__ __forceinline__ void syrk_store(const Sh &s, int mfit, const SyrkAcc &acc, double *dst, double *dvec,
                                           double *gpart)
{
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (acc.slice) {
        const int nblocks = acc.nb * (acc.nb + 1) / 2;
        double2 *mine = reinterpret_cast<double2 *>(gpart) + (size_t)warp * kSliceBlk * 32;
#pragma unroll
        for (int i = 0; i < kSliceBlk; ++i)
            if (i < nblocks) mine[i * 32 + lane] = make_double2(acc.c[i][0], acc.c[i][1]);
        __syncthreads();
        const int ld = s.ld;
        for (int idx = tid; idx < nblocks * 64; idx += kThreads) {
            const int i = idx >> 6, l = (idx >> 1) & 31, e = idx & 1;
            double v = 0.0;
            for (int w = 0; w < kWarps; ++w) v += gpart[((size_t)w * kSliceBlk * 32 + i * 32 + l) * 2 + e];
            int bj = 0;
            while ((bj + 1) * (bj + 2) / 2 <= i) ++bj;
            const int bk = i - bj * (bj + 1) / 2;
            const int row = 8 * bj + (l >> 2), col = 8 * bk + 2 * (l & 3) + e;
            if (row < mfit && col <= row) {
                dst[row * ld + col] = v;
                dst[col * ld + row] = v;
            } else if (row == mfit && col < mfit) {
                dvec[col] = v;
            } else if (row == mfit && col == mfit) {
                s.scal[S_TRIAL] = v;
            }
        }
        __syncthreads();
        return;
    }
#pragma unroll
    for (int i = 0; i < kMaxBlk; ++i)
        if (i < acc.nblk) syrk_add_block(s, mfit, acc.bj[i], acc.bk[i], acc.c[i][0], acc.c[i][1], dst, dvec, true);
    __syncthreads();
}

// One full evaluation (mrqcof) at parameter vector a in shared memory.
// Writes alpha (symmetric, stride ld) to dst, beta to dvec; returns chi^2 to
// every thread.
template <int NCP, bool MIXED>
__device__ double evaluate(const DevObject &o, const DevParams &p, const Sh &s, const double *a,
                           double *dst, double *dvec, double *rows, double *cstat, int *perm, double conw_r)
{
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int ma = o.ma, mfit = o.mfit, mfp = s.mfp, RS = o.row_stride, CS = ma + 3;

    if (o.cstat_smem) cstat = s.cst;  // stride ma + 3 fits inside rs + 2
    tmark(p, s, T_REST);
    double area_sum = shape_areas(o, s, a);
    if (tid == 0) s.scal[S_AREA] = area_sum;
    set_invariants(o, p, s, a);
    if constexpr (MIXED) {  // FP32 facet tables of the mixed-precision sweep
        const double cl = s.inv[5], cls = s.inv[6];
        for (int f = tid; f < o.n_fac; f += kThreads) {
            const double4 fr = s.F[f];
            s.F32[f] = make_float4((float)fr.x, (float)fr.y, (float)fr.z, (float)fr.w);
            s.G32[f] = make_float2((float)(fr.w * cl), (float)(fr.w * cls));
        }
        __syncthreads();
    }
    tmark(p, s, T_CURV);

    sort_points(o, s, perm, perm + o.n_points);
    tmark(p, s, T_SORT);
    if constexpr (MIXED)
        brightness_rows_mixed<NCP>(o, s, rows, perm);
    else
        if (o.n_coef == NCP - 7)
            brightness_rows<NCP, true>(o, s, rows, perm);
        else
            brightness_rows<NCP, false>(o, s, rows, perm);
    // the tile phase reads the rows back through the bulk-copy (async) proxy
    asm volatile("fence.proxy.async.global;" ::: "memory");
    __syncthreads();
    tmark(p, s, T_SWEEP);

    // per relative curve: column sums, 1/sum(ymod) and the renormalisation coefficient
    for (int c = warp; c < o.n_curves; c += kWarps) {
        if (!o.curve_rel[c]) continue;
        const int p0 = o.curve_start[c], p1 = o.curve_start[c + 1];
        // columns lane, lane + 32, lane + 64 (ma + 1 <= 90); the rows come from
        // HBM, so each step issues the loads of 16 points before adding them
        constexpr int kStep = 16;
        double sum[3] = {0, 0, 0};
        for (int q0 = p0; q0 < p1; q0 += kStep) {
            double v[kStep][3];
#pragma unroll
            for (int u = 0; u < kStep; ++u) {
                const bool ok = q0 + u < p1;
                const double *r = rows + (size_t)(ok ? q0 + u : p0) * RS;
#pragma unroll
                for (int j = 0; j < 3; ++j) v[u][j] = (ok && lane + 32 * j <= ma) ? r[lane + 32 * j] : 0.0;
            }
#pragma unroll
            for (int u = 0; u < kStep; ++u)
#pragma unroll
                for (int j = 0; j < 3; ++j) sum[j] += v[u][j];
        }
#pragma unroll
        for (int j = 0; j < 3; ++j)
            if (lane + 32 * j <= ma) cstat[(size_t)c * CS + lane + 32 * j] = sum[j];
        __syncwarp();
        if (lane == 0) {
            const double rave = 1.0 / cstat[(size_t)c * CS + ma];
            const double coef = o.curve_sig[c] * (p1 - p0) * rave;
            cstat[(size_t)c * CS + ma + 1] = rave;
            cstat[(size_t)c * CS + ma + 2] = coef;
            s.crave[c] = rave;
            s.ccoef[c] = coef;
        }
    }
    __syncthreads();
    tmark(p, s, T_CSTAT);

    SyrkAcc acc;
    syrk_init(mfit, s.tr, acc);

    // J^T W J tiles: the raw rows of tile t (tile_rows consecutive points)
    // and their per-point records arrive by bulk copy, double-buffered, while
    // the tensor cores work on tile t - 1.  Each warp stages tile_rows / 8
    // rows: renormalisation (relative curves, Start.cu:2660-2693) and
    // compaction to the fitted parameters.
    const int np = o.n_points, TR = s.tr, rpw = TR / kWarps;
    const int ntile = (np + TR - 1) / TR;
    auto tissue = [&](int t) {
        const int r0 = t * TR, nr = min(TR, np - r0), b = t & 1;
        bulk_load(s.raw + (size_t)b * TR * RS, rows + (size_t)r0 * RS, (uint32_t)(nr * RS * sizeof(double)),
                  &s.tbar[b]);
        bulk_load(s.recb + b * TR, o.pt_rec + r0, (uint32_t)(nr * sizeof(double4)), &s.tbar[b]);
    };
    if (tid == 0) {
        tissue(0);
        if (ntile > 1) tissue(1);
    }
    bool timeout = false;
    if (acc.slice) {
        // k-slice mode: warp w owns rows 4w..4w+3 of every tile and builds its
        // MMA fragments straight from the raw rows in shared memory (lane row
        // 4w + lane%4, fit column 8q + lane/4), so the tile loop needs no CTA
        // barrier; the last warp done with a buffer refills it.  Software
        // pipelined: the fragments of tile t+1 are built (and its buffer
        // released) in the same branch-free stretch of code that issues the
        // MMAs of tile t, so the gathers overlap the tensor-core work.
        const int rr = 4 * warp + (lane & 3);
        const int jl = lane >> 2;
        int colq[8];  // raw-row column of this lane's fit column 8 q + jl (clamped)
#pragma unroll
        for (int q = 0; q < 8; ++q) colq[q] = s.fidx[min(8 * q + jl, mfit - 1)] - 1;
        auto wait_tile = [&](int t) {
            const int b = t & 1;
            if (!mbar_wait(&s.tbar[b], (uint32_t)((s.ctl[C_TUSE + b] + (t >> 1)) & 1))) timeout = true;
        };
        // rows past the tile's end (and whole warps past it) read stale but
        // in-buffer data and contribute exact zeros
        auto build = [&](int t, double (&fa)[8], double (&fb)[8]) {
            const int b = t & 1, nrows = min(TR, np - t * TR);
            const double *rb = s.raw + (size_t)b * TR * RS;
            const bool valid = rr < nrows;
            const double4 rec = s.recb[b * TR + rr];
            const double ymod0 = rb[rr * RS + ma];
            const bool rel = valid && rec.w != 0.0;
            const int cur = rel ? (int)rec.z : 0;
            const double coef = rel ? s.ccoef[cur] : 0.0;
            const double sub = rel ? ymod0 * s.crave[cur] : 0.0;
            const double ymod = rel ? coef * ymod0 : ymod0;
            const double dy = valid ? rec.x - ymod : 0.0;
            const double w = valid ? rec.y : 0.0;
            const double *dav = cstat + (size_t)cur * CS;
            const double *rrow = rb + rr * RS;
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const int j = 8 * q + jl;
                const int col = colq[q];
                const double raw = rrow[col];
                const double dv = rel ? dav[col] : 0.0;
                double v = rel ? coef * (raw - sub * dv) : raw;
                v = j < mfit ? v : (j == mfit ? dy : 0.0);
                v = valid ? v : 0.0;
                fb[q] = v;
                fa[q] = v * w;
            }
        };
        auto release = [&](int t) {
            const int b = t & 1;
            __syncwarp();
            if (lane == 0) {
                __threadfence_block();
                if (atomicAdd(&s.ctl[C_TREL + b], 1) == kWarps - 1) {
                    s.ctl[C_TREL + b] = 0;
                    if (t + 2 < ntile) tissue(t + 2);
                }
            }
        };
        auto run = [&](auto full8) {
            constexpr bool kFull = decltype(full8)::value;
            auto mmas = [&](const double (&fa)[8], const double (&fb)[8]) {
#pragma unroll
                for (int bj = 0; bj < 8; ++bj)
#pragma unroll
                    for (int bk = 0; bk <= bj; ++bk)
                        if (kFull || bj < acc.nb) {
                            const int i = bj * (bj + 1) / 2 + bk;
                            dmma_8x8x4(acc.c[i][0], acc.c[i][1], fa[bj], fb[bk]);
                        }
            };
            double fa[8], fb[8], ga[8], gb[8];
            wait_tile(0);
            build(0, fa, fb);
            release(0);
            for (int t = 0; t + 1 < ntile; ++t) {
                wait_tile(t + 1);
                build(t + 1, ga, gb);
                mmas(fa, fb);
                release(t + 1);
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    fa[q] = ga[q];
                    fb[q] = gb[q];
                }
            }
            mmas(fa, fb);
        };
        tmark(p, s, T_TILES);
        if (acc.nb == 8)
            run(std::true_type{});
        else
            run(std::false_type{});
        tmark(p, s, T_TSYRK);
        __syncthreads();
    } else {
    for (int t = 0; t < ntile; ++t) {
        const int b = t & 1, r0 = t * TR, nrows = min(TR, np - r0);
        tmark(p, s, T_TILES);
        if (!mbar_wait(&s.tbar[b], (uint32_t)((s.ctl[C_TUSE + b] + (t >> 1)) & 1))) timeout = true;
        tmark(p, s, T_TWAIT);
        const double *rb = s.raw + (size_t)b * TR * RS;
        const double4 *rc = s.recb + b * TR;
        // per-row scalars: lane k < rpw computes row warp * rpw + k
        double dyL = 0.0, wL = 0.0, coefL = 0.0, subL = 0.0;
        int curL = -1;
        if (lane < rpw && warp * rpw + lane < nrows) {
            const int rr = warp * rpw + lane;
            const double4 rec = rc[rr];
            double ymod = rb[rr * RS + ma];
            if (rec.w != 0.0) {
                curL = (int)rec.z;
                coefL = s.ccoef[curL];
                subL = ymod * s.crave[curL];
                ymod = coefL * ymod;
            }
            dyL = rec.x - ymod;
            wL = rec.y;
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            if (k >= rpw) break;
            const int rr = warp * rpw + k;
            const bool valid = rr < nrows;
            const double dy = __shfl_sync(0xffffffffu, dyL, k);
            const double w = __shfl_sync(0xffffffffu, wL, k);
            const double coef = __shfl_sync(0xffffffffu, coefL, k);
            const double sub = __shfl_sync(0xffffffffu, subL, k);
            const int cur = __shfl_sync(0xffffffffu, curL, k);
            const double *dav = cstat + (size_t)max(cur, 0) * CS;
            const double *rrow = rb + rr * RS;
            double *trow = s.T + rr * mfp, *twrow = s.TW + rr * mfp;
            const bool rel = cur >= 0;
            double v[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {  // branch-free gathers, as in the k-slice form
                const int j = lane + 32 * u;
                const int col = s.fidx[min(j, mfit - 1)] - 1;
                const double raw = rrow[col];
                const double dv = rel ? dav[col] : 0.0;
                v[u] = rel ? coef * (raw - sub * dv) : raw;
                v[u] = j < mfit ? v[u] : (j == mfit ? dy : 0.0);
                v[u] = valid ? v[u] : 0.0;
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int j = lane + 32 * u;
                if (j < mfp) {
                    trow[j] = v[u];
                    twrow[j] = v[u] * w;
                }
            }
        }
        __syncthreads();
        tmark(p, s, T_TSTAGE);
        if (tid == 0 && t + 2 < ntile) tissue(t + 2);
        syrk_update(s, nrows, acc);
        __syncthreads();
        tmark(p, s, T_TSYRK);
    }
    }
    if (timeout) s.ctl[C_TIMEOUT] = 1;
    if (tid == 0) {
        s.ctl[C_TUSE + 0] += (ntile + 1) / 2;
        s.ctl[C_TUSE + 1] += ntile / 2;
    }
    tmark(p, s, T_TILES);

    // convexity regularisation pseudo-points (mrqcof_curve1_last_opt, Start.cu:2539-2612)
    {
        const int nc = o.n_coef, nf = o.n_fac;
        double ym[3] = {0, 0, 0};
        for (int fi = tid; fi < nf; fi += kThreads) {
            const double4 fr = s.F[fi];
            ym[0] += fr.w * fr.x;
            ym[1] += fr.w * fr.y;
            ym[2] += fr.w * fr.z;
        }
        block_sum<3>(ym, s.red);
        // raw derivative d ym_i / d a_k for shape coefficient k = tid: groups
        // of nc threads take consecutive facet ranges, their partial sums
        // (staged in the idle tile buffer) are added in group order
        double dk[3] = {0, 0, 0};
        {
            const int ngrp = max(1, min(kThreads / nc, (s.tr * mfp) / (3 * nc)));
            const int per = (nf + ngrp - 1) / ngrp;
            const int grp = tid / nc, k = tid - grp * nc;
            if (grp < ngrp) {
                double pk[3] = {0, 0, 0};
                const int fe = min(nf, (grp + 1) * per);
                for (int fi = grp * per; fi < fe; ++fi) {
                    const double4 fr = s.F[fi];
                    const double y = __ldg(o.ysh + (size_t)fi * o.ncp + k);
                    pk[0] += (fr.w * fr.x) * y;
                    pk[1] += (fr.w * fr.y) * y;
                    pk[2] += (fr.w * fr.z) * y;
                }
#pragma unroll
                for (int i = 0; i < 3; ++i) s.T[(grp * 3 + i) * nc + k] = pk[i];
            }
            __syncthreads();
            if (tid < nc)
                for (int g2 = 0; g2 < ngrp; ++g2)
#pragma unroll
                    for (int i = 0; i < 3; ++i) dk[i] += s.T[(g2 * 3 + i) * nc + tid];
            __syncthreads();
        }
        const double wps = conw_r * conw_r;
        for (int idx = tid; idx < kTile * mfp; idx += kThreads) {
            s.T[idx] = 0.0;
            s.TW[idx] = 0.0;
        }
        __syncthreads();
        if (tid < nc) {
            int slot = -1;  // fit slot of parameter tid + 1, if fitted
            for (int j = 0; j < mfit; ++j)
                if (s.fidx[j] == tid + 1) slot = j;
            if (slot >= 0)
                for (int i = 0; i < 3; ++i) {
                    s.T[i * mfp + slot] = dk[i];
                    s.TW[i * mfp + slot] = dk[i] * wps;
                }
        }
        if (tid < 3) {
            const double dy = 0.0 - ym[tid];
            s.T[tid * mfp + mfit] = dy;
            s.TW[tid * mfp + mfit] = dy * wps;
        }
        __syncthreads();
        syrk_update(s, 3, acc);
    }
    syrk_store(s, mfit, acc, dst, dvec, rows + scratch_gpart(o.n_points, RS, o.n_curves, ma));
    tmark(p, s, T_PSEUDO);
    if (p.phase_cycles && tid == 0) atomicAdd(&p.phase_cycles[T_NPHASE], 1ull);
    return s.scal[S_TRIAL];
}

// ---------------------------------------------------------------- LM step

// Full-pivot Gauss-Jordan on covar (n x n, stride ld) and b = da
// (mrqmin_1_end_opt, Start.cu:2880-3006), one CTA barrier per pivot.
//
// The pivot is the maximum |a| over unpivoted rows and columns; among equal
// values the last one in row-major order wins, as in the serial scan: every
// candidate carries (|a|, logical row * n + column) and the CTA takes the
// lexicographic maximum (NaN is never a candidate).  The candidate search for
// pivot i+1 runs inside the elimination of pivot i, on the values just
// written.
//
// Thread (rsub, csub) owns row slots rsub + 64 r and columns csub + 4 j.  A
// row swap only swaps the logical labels of two slots (kept in registers), so
// rows never move.  The pivot row is not scaled when it is chosen: every
// reader forms the scaled value pivot_row[l] * pivinv itself (the same
// rounding as a stored product), and the row's owners apply the scale when
// they next touch it, in the following elimination.  ipiv lives in register
// bit masks, alike in all threads.  The rounding of every stored value equals
// the serial algorithm's; the inverse is not needed, so already-pivoted
// columns are left stale.  Returns the reference's error code: 0, 1 (pivot
// bookkeeping) or 2 (zero pivot).  All threads must call it.
struct __align__(16) GjCand {
    double v;  // |a| of the warp's best candidate, -1 if it has none
    int key;   // logical row * n + column
    int slot;  // row slot, bit 31 = bookkeeping fault seen
};

__device__ __forceinline__ bool gj_mask_bit(unsigned w0, unsigned w1, unsigned w2, int c)
{
    const unsigned w = c < 32 ? w0 : (c < 64 ? w1 : w2);
    return (w >> (c & 31)) & 1u;
}

// Lane holding the warp's maximum of (value, key), value given as its high
// word (signed: values >= 0 order like their bits, -1 below all) and low
// word; among equal values the largest key.  Nearly always the high words
// alone decide.
__device__ __forceinline__ int gj_argmax(int hi, unsigned lo, int key)
{
    const int mh = __reduce_max_sync(0xffffffffu, hi);
    const unsigned tie = __ballot_sync(0xffffffffu, hi == mh);
    if (__popc(tie) == 1) return __ffs(tie) - 1;
    const unsigned ml = __reduce_max_sync(0xffffffffu, hi == mh ? lo : 0u);
    const bool top = hi == mh && lo == ml;
    const unsigned mk = __reduce_max_sync(0xffffffffu, top ? (unsigned)key : 0u);
    return __ffs(__ballot_sync(0xffffffffu, top && (unsigned)key == mk)) - 1;
}

// kMaxN: the largest n the caller passes (row slots and columns per thread
// are sized for it).
template <int kMaxN>
static __device__ int gauss_jordan(const Sh &s, int n)
{
    constexpr int kSlots = kThreads / 4;
    constexpr int kRowsPer = (kMaxN + kSlots - 1) / kSlots;
    constexpr int kColsPer = (kMaxN + 3) / 4;
    static_assert(kMaxN <= kMaxFit && kMaxFit <= 96 && kRowsPer <= 2, "pivot masks are 32-bit words");
    static_assert(kMaxFit * kMaxFit < (1 << 13) && kMaxFit < (1 << 7), "key division by multiply and shift");
    static_assert(sizeof(GjCand) * 2 * kWarps <= sizeof(double) * kWarps * 4, "candidate buffers in red");
    static_assert(kWarps <= 32 && (kWarps & (kWarps - 1)) == 0, "one lane per warp candidate");
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int ld = s.ld, rsub = tid >> 2, csub = tid & 3;
    const unsigned ndiv = ((1u << 20) + n - 1) / n;  // key / n == (key * ndiv) >> 20 for key < n * n
    double *A = s.covar, *b = s.da;
    GjCand *cand_buf = reinterpret_cast<GjCand *>(s.red);

    int lab[kRowsPer];
#pragma unroll
    for (int r = 0; r < kRowsPer; ++r) lab[r] = rsub + kSlots * r;
    unsigned g1a = 0, g1b = 0, g1c = 0;  // columns with ipiv >= 1
    unsigned g2a = 0, g2b = 0, g2c = 0;  // columns with ipiv >= 2
    unsigned c1 = 0, c2 = 0;             // the same for this thread's columns, bit j = column csub + 4 j
    int pend = -1;                       // slot of the previous pivot row (scale pending)
    double pend_inv = 1.0;

    double bv = -1.0;  // the thread's best candidate
    int bkey = 0, bslot = 0;
    bool bad = false;
    // a row's best (the last of equal values, columns being visited in order)
    // joins the thread's candidate
    auto cand = [&](double big, int j, int L, int slot) {
        const int key = L * n + csub + 4 * j;
        if (big > bv || (big == bv && big >= 0.0 && key > bkey)) {
            bv = big;
            bkey = key;
            bslot = slot;
        }
    };
    auto row_open = [&](int L) {  // ipiv[L] != 1
        return !(gj_mask_bit(g1a, g1b, g1c, L) && !gj_mask_bit(g2a, g2b, g2c, L));
    };

#pragma unroll
    for (int r = 0; r < kRowsPer; ++r) {
        const int ll = rsub + kSlots * r;
        if (ll < n) {
            const double *row = A + ll * ld;
            double big = -1.0;
            int bj = 0;
#pragma unroll
            for (int j = 0; j < kColsPer; ++j) {
                const int l = csub + 4 * j;
                if (l < n) {
                    const double t = fabs(row[l]);
                    if (t >= big) {
                        big = t;
                        bj = j;
                    }
                }
            }
            cand(big, bj, ll, ll);
        }
    }

    int err = 0;
    for (int i = 0; i < n; ++i) {
        {
            const int hi = __double2hiint(bv);
            const int src = gj_argmax(hi, (unsigned)__double2loint(bv), bkey);
            const double wv = __shfl_sync(0xffffffffu, bv, src);
            const int wkey = __shfl_sync(0xffffffffu, bkey, src);
            const int wslot = __shfl_sync(0xffffffffu, bslot, src);
            const bool wbad = __any_sync(0xffffffffu, bad);
            if (lane == 0) {
                GjCand c;
                c.v = wv;
                c.key = wkey;
                c.slot = wslot | (wbad ? (int)0x80000000u : 0);
                cand_buf[(i & 1) * kWarps + warp] = c;
            }
        }
        __syncthreads();
        int irow, icol, P;
        bool none;
        {
            // every warp combines the warps' candidates alike, lane w < kWarps
            // holding warp w's
            const GjCand c = cand_buf[(i & 1) * kWarps + (lane & (kWarps - 1))];
            if (__any_sync(0xffffffffu, c.slot < 0)) {
                err = 1;
                break;
            }
            const int hi = lane < kWarps ? __double2hiint(c.v) : INT_MIN;
            const int src = gj_argmax(hi, (unsigned)__double2loint(c.v), c.key);
            const double vm = __shfl_sync(0xffffffffu, c.v, src);
            const int km = __shfl_sync(0xffffffffu, c.key, src);
            P = __shfl_sync(0xffffffffu, c.slot, src);
            none = vm < 0.0;
            irow = (int)(((unsigned)km * ndiv) >> 20);
            icol = km - irow * n;
        }
        if (none) {
            // nothing but NaN left: the serial scan's (0, 0).  Row 0 may be
            // the pending row, so scale that first, then find row 0's slot.
            irow = icol = 0;
#pragma unroll
            for (int r = 0; r < kRowsPer; ++r) {
                const int ll = rsub + kSlots * r;
                if (ll >= n) continue;
                if (ll == pend) {
                    double *row = A + ll * ld;
#pragma unroll
                    for (int j = 0; j < kColsPer; ++j) {
                        const int l = csub + 4 * j;
                        if (l < n && !((c1 >> j) & 1u)) row[l] = __dmul_rn(row[l], pend_inv);
                    }
                    if (csub == 0) b[ll] = __dmul_rn(b[ll], pend_inv);
                }
                if (lab[r] == 0 && csub == 0) s.ctl[C_GJROW0] = ll;
            }
            __syncthreads();
            P = s.ctl[C_GJROW0];
            pend = -1;
        }
        // the swap of rows irow and icol
#pragma unroll
        for (int r = 0; r < kRowsPer; ++r) lab[r] = lab[r] == irow ? icol : (lab[r] == icol ? irow : lab[r]);
        // P is an open row, never the pending one (that one is closed, or a
        // bookkeeping fault ended the solve above, or the NaN branch scaled it)
        const double piv = A[P * ld + icol];
        if (piv == 0.0) {
            err = 2;
            break;
        }
        const double pivinv = 1.0 / piv;
        const double bs = __dmul_rn(b[P], pivinv);
        // ipiv[icol] += 1
        {
            const unsigned m = 1u << (icol & 31);
            if (icol < 32) {
                if (g1a & m) g2a |= m;
                g1a |= m;
            } else if (icol < 64) {
                if (g1b & m) g2b |= m;
                g1b |= m;
            } else {
                if (g1c & m) g2c |= m;
                g1c |= m;
            }
            if ((icol & 3) == csub) {
                const unsigned mj = 1u << (icol >> 2);
                if (c1 & mj) c2 |= mj;
                c1 |= mj;
            }
        }
        // eliminate (only unpivoted columns feed later pivots and b) and look
        // for the next pivot among unpivoted rows and columns
        bv = -1.0;
        bkey = 0;
        bslot = 0;
        bad = false;
        const double *__restrict__ prow = A + P * ld;
#pragma unroll 1
        for (int r = 0; r < kRowsPer; ++r) {
            const int ll = rsub + kSlots * r;
            if (ll >= n) continue;
            const int L = r == 0 ? lab[0] : lab[kRowsPer - 1];
            const bool open = row_open(L);
            double *__restrict__ row = A + ll * ld;
            if (open && c2) bad = true;  // a column with ipiv > 1 in an open row
            double big = -1.0;
            int bj = 0;
            if (ll == P) {
                if (open) {  // only after a bookkeeping fault: keep the serial checks
#pragma unroll
                    for (int j = 0; j < kColsPer; ++j) {
                        const int l = csub + 4 * j;
                        if (l < n && !((c1 >> j) & 1u)) {
                            const double t = fabs(__dmul_rn(row[l], pivinv));
                            if (t >= big) {
                                big = t;
                                bj = j;
                            }
                        }
                    }
                    cand(big, bj, L, ll);
                }
                continue;
            }
            // x * 1.0 == x exactly: rows other than the pending one pass unscaled
            const double rs = ll == pend ? pend_inv : 1.0;
            const double cb = __dmul_rn(row[icol], rs);
#pragma unroll
            for (int j = 0; j < kColsPer; ++j) {
                const int l = csub + 4 * j;
                if (l < n && !((c1 >> j) & 1u)) {
                    const double v = __fma_rn(-__dmul_rn(prow[l], pivinv), cb, __dmul_rn(row[l], rs));
                    row[l] = v;
                    const double t = fabs(v);
                    if (t >= big) {
                        big = t;
                        bj = j;
                    }
                }
            }
            if (open) cand(big, bj, L, ll);
            if (csub == 0) b[ll] = __fma_rn(-bs, cb, __dmul_rn(b[ll], rs));
        }
        pend = P;
        pend_inv = pivinv;
    }
    // b back to logical order, the pending scale applied
    double bo[kRowsPer];
#pragma unroll
    for (int r = 0; r < kRowsPer; ++r) {
        const int ll = rsub + kSlots * r;
        bo[r] = 0.0;
        if (ll < n && csub == 0) bo[r] = ll == pend ? __dmul_rn(b[ll], pend_inv) : b[ll];
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < kRowsPer; ++r) {
        const int ll = rsub + kSlots * r;
        if (ll < n && csub == 0) b[lab[r]] = bo[r];
    }
    __syncthreads();
    return err;
}

// ---------------------------------------------------------------- kernel

// One (frequency, pole) fit, the whole LM loop, by the CTA; its result to
// out[item].  o and p are the fit's object and constants.
template <int NCP, bool MIXED>
__device__ __forceinline__ void fit_one(const DevObject &o, const DevParams &p, const Sh &s, const FitItem it,
                                        int item, FitOut *out, double *rows, int *status)
{
    const int tid = threadIdx.x;
    const int nc = o.n_coef, ma = o.ma, mfit = o.mfit, ld = s.ld;
    const int pole = it.pole & kPoleMask;
    double *cstat = rows + (size_t)o.n_points * o.row_stride;
    int *perm = reinterpret_cast<int *>(rows + scratch_perm(o.n_points, o.row_stride, o.n_curves, ma));

    // initial parameters (CudaCalculatePreparePole, Start.cu:4346-4418)
    if (tid == 0) {
        double *a = s.a;
        a[0] = 0;
        for (int k = 1; k <= nc; ++k) a[k] = __ldg(&o.cg_first[k - 1]);
        const double period = 1.0 / (p.freq_start - (it.n_freq - 1) * p.freq_step);
        a[nc + 1] = (kPi / 180) * 90 - (kPi / 180) * p.beta_pole[pole];
        a[nc + 2] = (kPi / 180) * p.lambda_pole[pole];
        a[nc + 3] = (24.0 * 2.0 * kPi) / period;
        a[nc + 4] = p.par[0];
        a[nc + 5] = p.par[1];
        a[nc + 6] = p.par[2];
        a[ma - 1] = p.lcl;
        a[ma] = 1;
        s.scal[S_ALAMDA] = -1;
        s.scal[S_ITERDIFF] = 1e40;
        s.scal[S_DEVOLD] = 1e30;
        s.scal[S_DEVNEW] = 0;
        s.scal[S_CHCK] = 0;
        s.ctl[C_NITER] = 0;
        s.ctl[C_STATUS] = 0;
    }
    __syncthreads();

    for (;;) {
        // convergence test (CudaCalculateIter1Begin, Start.cu:4421-4462)
        if (tid == 0) {
            const int niter = s.ctl[C_NITER];
            s.ctl[C_GO] = ((niter < p.n_iter_max) && (s.scal[S_ITERDIFF] > p.iter_diff_max)) ||
                          (niter < p.n_iter_min);
        }
        __syncthreads();
        if (!s.ctl[C_GO]) break;
        const bool first = s.scal[S_ALAMDA] < 0;
        __syncthreads();
        if (first) {
            if (tid == 0) s.scal[S_ALAMDA] = p.alamda_start;
            double oc = evaluate<NCP, MIXED>(o, p, s, s.a, s.alpha, s.beta, rows, cstat, perm, p.conw_r);
            if (tid == 0) s.scal[S_OCHISQ] = oc;
            for (int q = tid; q <= ma; q += kThreads) s.atry[q] = s.a[q];
            __syncthreads();
        }
        // damped normal matrix and solve (mrqmin_1_end_opt)
        const double ccc = 1 + s.scal[S_ALAMDA];
        for (int idx = tid; idx < mfit * mfit; idx += kThreads) {
            const int j = idx / mfit, k = idx - j * mfit;
            const double v = s.alpha[j * ld + k];
            s.covar[j * ld + k] = (j == k) ? v * ccc : v;
        }
        if (tid < mfit) s.da[tid] = s.beta[tid];
        __syncthreads();
        tmark(p, s, T_REST);
        // mfit <= ma = n_coef + 8 <= NCP + 8 (and < kMaxFit)
        const int err = gauss_jordan<(NCP + 8 < kMaxFit ? NCP + 8 : kMaxFit)>(s, mfit);
        tmark(p, s, T_SOLVE);
        if (err == 0 || err == 2) {
            if (tid < mfit) s.atry[s.fidx[tid]] = s.a[s.fidx[tid]] + s.da[tid];
            if (err == 2 && tid == 0) s.ctl[C_STATUS] |= kStatusSingular;
        }
        __syncthreads();
        const double chisq = evaluate<NCP, MIXED>(o, p, s, s.atry, s.covar, s.da, rows, cstat, perm, p.conw_r);
        // accept / reject (mrqmin_2_end, Start.cu:300-392)
        const bool accept = chisq < s.scal[S_OCHISQ];
        __syncthreads();
        if (accept) {
            for (int idx = tid; idx < mfit * ld; idx += kThreads) s.alpha[idx] = s.covar[idx];
            if (tid < mfit) s.beta[tid] = s.da[tid];
            for (int q = tid; q <= ma; q += kThreads) s.a[q] = s.atry[q];
        }
        if (tid == 0) {
            if (isnan(chisq)) s.ctl[C_STATUS] |= kStatusNanChisq;
            if (accept) {
                s.scal[S_ALAMDA] *= p.alamda_incrr;
                s.scal[S_CHISQ] = chisq;
            } else {
                s.scal[S_ALAMDA] = p.alamda_incr * s.scal[S_ALAMDA];
                s.scal[S_CHISQ] = s.scal[S_OCHISQ];
            }
            s.ctl[C_NITER] += 1;
        }
        __syncthreads();
        // rms and convergence bookkeeping (CudaCalculateIter2, Start.cu:5129-5248)
        const int niter = s.ctl[C_NITER];
        const double ch = s.scal[S_CHISQ];
        if (niter == 1 || ch < s.scal[S_OCHISQ]) {
            __syncthreads();
            const double area_sum = shape_areas(o, s, s.a);
            double r[3] = {0, 0, 0};
            for (int fi = tid; fi < o.n_fac; fi += kThreads) {
                const double4 fr = s.F[fi];
                r[0] += fr.w * fr.x;
                r[1] += fr.w * fr.y;
                r[2] += fr.w * fr.z;
            }
            block_sum<3>(r, s.red);
            if (tid == 0) {
                s.scal[S_OCHISQ] = ch;
                s.scal[S_AREA] = area_sum;
                const double aa = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
                const double rchisq = ch - aa * (p.conw_r_dev * p.conw_r_dev);
                const double dev_new = sqrt(rchisq / (o.n_points + 3 - 3));
                s.scal[S_DEVNEW] = dev_new;
                s.scal[S_CHCK] = sqrt(aa);
                const double diff = s.scal[S_DEVOLD] - dev_new;
                if (diff > 1e-10) {
                    s.scal[S_ITERDIFF] = diff;
                    s.scal[S_DEVOLD] = dev_new;
                }
            }
        }
        __syncthreads();
    }

    // per-fit result (CudaCalculateFinishPole, Start.cu:5056-5125)
    if (tid == 0) {
        double dd = s.scal[S_CHCK] * 100.0 * (1.0 / s.scal[S_AREA]);
        if (isnan(dd)) dd = 1.0;
        const double la = (180 / kPi) * s.a[nc + 2];
        FitOut r;
        r.dev = s.scal[S_DEVNEW];
        r.dark = dd;
        r.per = 2 * kPi / s.a[nc + 3];
        r.lambda_deg = la + (la < 0 ? 360 : 0);
        r.beta_deg = 90 - (180 / kPi) * s.a[nc + 1];
        r.chisq = s.scal[S_CHISQ];
        r.niter = s.ctl[C_NITER];
        r.status = s.ctl[C_STATUS] | (s.ctl[C_TIMEOUT] ? kStatusTimeout : 0);
        out[item] = r;
        if (r.status) atomicOr(status, r.status);
        if (p.phase_cycles) {
            tmark(p, s, T_REST);
            for (int q = 0; q < T_NPHASE; ++q) {
                atomicAdd(&p.phase_cycles[q], (unsigned long long)s.tclk[q]);
                s.tclk[q] = 0;
            }
        }
    }
}

template <int NCP, bool MIXED, bool BATCH>
__global__ void __launch_bounds__(kThreads, 1)
fit_kernel(DevObject o, DevParams p, const FitItem *items, int n_items, int *queue, FitOut *out,
           double *scratch, size_t scratch_per_cta, int *status, EvalOut ev, int mode, const DevObject *objs,
           const DevParams *prms)
{
    // batch launches: o holds the largest sizes of the batch (the shared-memory
    // layout); every item names its object (FitItem::pole >> kPoleBits),
    // whose tables and constants come from objs / prms when the CTA moves to it
    __shared__ DevObject s_obj;
    __shared__ DevParams s_prm;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Sh s;
    carve_bytes(o.n_fac, o.mfit, o.ncp, o.n_curves, o.row_stride, o.tile_rows, o.cstat_smem, MIXED ? 1 : 0, &s,
                smem_raw);
    const int tid = threadIdx.x;
    double *rows = scratch + (size_t)blockIdx.x * scratch_per_cta;

    if constexpr (!BATCH) {
        for (int f = tid; f < o.n_fac; f += kThreads) s.F[f] = ldg4(&o.facet[f]);
        facet_cones(o, s);
        if (tid < o.mfit) s.fidx[tid] = __ldg(&o.fidx[tid]);
    }
    if (tid == 0) {
        for (int b = 0; b < kStages; ++b) {
            mbar_init(&s.mbar[b], 1);
            s.ctl[C_YUSE + b] = 0;
            s.ctl[C_REL + b] = 0;
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&s.tbar[b], 2);  // two copies (rows + records) per fill
            s.ctl[C_TUSE + b] = 0;
            s.ctl[C_TREL + b] = 0;
        }
        for (int q = 0; q < T_NPHASE; ++q) s.tclk[q] = 0;
        s.tclk[T_NPHASE] = clock64();
        s.ctl[C_TIMEOUT] = 0;
    }
    __syncthreads();

    if constexpr (!BATCH) {
        if (mode == 1) {  // one stand-alone evaluation (parity hook)
            const int ma = o.ma, mfit = o.mfit, ld = s.ld;
            double *cstat = rows + (size_t)o.n_points * o.row_stride;
            int *perm = reinterpret_cast<int *>(rows + scratch_perm(o.n_points, o.row_stride, o.n_curves, ma));
            for (int q = tid; q <= ma; q += kThreads) s.a[q] = ev.a[q];
            __syncthreads();
            double chisq = evaluate<NCP, MIXED>(o, p, s, s.a, s.alpha, s.beta, rows, cstat, perm, p.conw_r);
            for (int idx = tid; idx < mfit * mfit; idx += kThreads) {
                const int j = idx / mfit, k = idx - j * mfit;
                ev.alpha[idx] = s.alpha[j * ld + k];
            }
            if (tid < mfit) ev.beta[tid] = s.beta[tid];
            if (tid == 0) {
                ev.chisq[0] = chisq;
                ev.area[0] = s.scal[S_AREA];
            }
            return;
        }
    }

    int cur = -1;  // batch: the object whose tables are loaded
    for (;;) {
        if (tid == 0) s.ctl[C_ITEM] = atomicAdd(queue, 1);
        __syncthreads();
        const int item = s.ctl[C_ITEM];
        if (item >= n_items) break;
        const FitItem it = items[item];
        if constexpr (BATCH) {
            const int k = it.pole >> kPoleBits;
            if (k != cur) {
                if (tid == 0) {
                    s_obj = objs[k];
                    s_prm = prms[k];
                }
                __syncthreads();
                for (int f = tid; f < s_obj.n_fac; f += kThreads) s.F[f] = ldg4(&s_obj.facet[f]);
                facet_cones(s_obj, s);
                if (tid < s_obj.mfit) s.fidx[tid] = __ldg(&s_obj.fidx[tid]);
                __syncthreads();
                cur = k;
            }
            fit_one<NCP, MIXED>(s_obj, s_prm, s, it, item, out, rows, status);
        } else {
            fit_one<NCP, MIXED>(o, p, s, it, item, out, rows, status);
        }
        __syncthreads();
        if (s.ctl[C_TIMEOUT]) break;  // a bulk copy never completed: stop taking items
    }
    // after a timeout, give any copy still in flight a bounded chance to land
    // before the CTA's shared memory is released
    if (tid == 0 && s.ctl[C_TIMEOUT]) {
        for (int b = 0; b < kStages; ++b) mbar_wait(&s.mbar[b], (uint32_t)(s.ctl[C_YUSE + b] & 1));
        for (int b = 0; b < 2; ++b) mbar_wait(&s.tbar[b], (uint32_t)(s.ctl[C_TUSE + b] & 1));
    }
}

}  // namespace psb
