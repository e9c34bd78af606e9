// fit_kernel.cuh -- persistent FP64 Levenberg-Marquardt fit kernel for sm_100a.
//
// One CTA (256 threads) owns one (frequency, pole) fit at a time and runs its
// whole LM loop on the device; CTAs pop items from a device queue, so ragged
// iteration counts never idle the grid.  Per function evaluation (the
// reference's mrqcof, Start.cu:535-629 + 2262-2828):
//
//   A  curv: facet areas exp(sum a_k Y_k) into shared memory  (Start.cu:421-528)
//   B  brightness rows: a warp takes 32 points (lane = point) and sweeps every
//      facet once; visibility, Lambert+Lommel-Seeliger terms, and the shape
//      derivative sum_f w_f Y_k(f) accumulate in registers.  The rotation
//      derivatives use dT/dq . (sum_f ar dS/dmu n_f), i.e. 6 accumulators per
//      point instead of 6 dot products per facet.  Rows go to HBM scratch.
//   C  per relative curve: column sums and 1/sum(ymod)  (Start.cu:2519-2533)
//   D  J^T W J, J^T W dy, chi^2: 32-row tiles staged renormalised in shared
//      memory, alpha held in registers as 2x2 blocks owned by threads.
//
// The LM step (damped Gauss-Jordan with full pivoting, accept/reject, lambda
// update, rms and convergence test) follows Start.cu:300-392, 2838-3021,
// 4421-4462, 5129-5248 with Numerical-Recipes ia compaction.
#pragma once
#include <cuda_runtime.h>

#include "engine.h"

namespace psb {

constexpr double kPi = 3.14159265358979323846;
constexpr double kTiny = 1e-8;
constexpr int kBPT = 5;  // 2x2 alpha blocks per thread: ceil(45*46/2 / 256)
constexpr int kFacetChunk = 32;     // facets per shared-memory basis chunk
constexpr int kSortBands = 8;       // point sort: bands in cos(theta) ...
constexpr int kSortSectors = 32;    // ... x sectors in longitude of the Sun-observer bisector
constexpr int kSortCells = kSortBands * kSortSectors;
constexpr unsigned kWaitLimit = 1u << 24;  // bounded mbarrier waits

// LM scalar slots in shared memory
enum { S_ALAMDA, S_CHISQ, S_OCHISQ, S_ITERDIFF, S_DEVOLD, S_DEVNEW, S_CHCK, S_AREA, S_TRIAL, S_PIVINV, S_NSCAL };
enum { C_ITEM, C_NITER, C_STATUS, C_ERR, C_IROW, C_ICOL, C_GO, C_ACCEPT, C_YUSE0, C_YUSE1, C_TIMEOUT, C_NCTL };

struct Sh {
    double4 *F;       // [n_fac] normal + current area
    double *alpha;    // [mfit][ld]
    double *covar;    // [mfit][ld]
    double *beta;     // [kMaxFit]
    double *da;       // [kMaxFit]
    double *a;        // [kMaxPar]
    double *atry;     // [kMaxPar]
    double *T;        // [kTile][mfp]       (shares storage with ybuf)
    double *TW;       // [kTile][mfp]       (shares storage with ybuf)
    double *ybuf;     // [2][kFacetChunk][ncp] basis chunks of the facet sweep
    unsigned long long *mbar;  // [2] completion barriers of the chunk copies
    int *hist;        // [2][kSortCells] point-sort histogram and offsets
    double *rdy;      // [kTile]
    double *rw;       // [kTile]
    double *red;      // [kWarps * 4]
    double *inv;      // [40] per-evaluation invariants
    double *scal;     // [S_NSCAL]
    double *colbuf;   // [kMaxFit]
    int *fidx;        // [kMaxFit]
    int *ipiv;        // [kMaxFit]
    int *ctl;         // [C_NCTL]
    int ld, mfp;
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
// kWaitLimit polls and returns false (the caller records a timeout).
__device__ __forceinline__ bool mbar_wait(unsigned long long *bar, uint32_t parity)
{
    for (unsigned i = 0; i < kWaitLimit; ++i) {
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

__host__ __device__ inline int fit_ld(int mfit) { return mfit | 1; }
__host__ __device__ inline int fit_mfp(int mfit) { return (mfit + 1) & ~1; }

__host__ __device__ inline size_t align16(size_t x) { return (x + 15) & ~size_t(15); }

__host__ __device__ inline size_t carve_bytes(int n_fac, int mfit, int ncp, Sh *s, unsigned char *base)
{
    int ld = fit_ld(mfit), mfp = fit_mfp(mfit);
    size_t off = 0;
    auto take = [&](size_t bytes) {
        size_t o = off;
        off = align16(off + bytes);
        return base ? (void *)(base + o) : nullptr;
    };
    void *F = take(sizeof(double4) * n_fac);
    void *alpha = take(sizeof(double) * mfit * ld);
    void *covar = take(sizeof(double) * mfit * ld);
    void *beta = take(sizeof(double) * kMaxFit);
    void *da = take(sizeof(double) * kMaxFit);
    void *a = take(sizeof(double) * kMaxPar);
    void *atry = take(sizeof(double) * kMaxPar);
    // the JtWJ tiles (phase D) and the basis chunks (phase B) are never live
    // at the same time: one region serves both
    const size_t tiles = 2 * align16(sizeof(double) * kTile * mfp);
    const size_t chunks = 2 * sizeof(double) * kFacetChunk * ncp;
    unsigned char *un = (unsigned char *)take(tiles > chunks ? tiles : chunks);
    void *T = un;
    void *TW = un ? un + align16(sizeof(double) * kTile * mfp) : nullptr;
    void *ybuf = un;
    void *mbar = take(sizeof(unsigned long long) * 2);
    void *hist = take(sizeof(int) * 2 * kSortCells);
    void *rdy = take(sizeof(double) * kTile);
    void *rw = take(sizeof(double) * kTile);
    void *red = take(sizeof(double) * kWarps * 4);
    void *inv = take(sizeof(double) * 40);
    void *scal = take(sizeof(double) * S_NSCAL);
    void *colbuf = take(sizeof(double) * kMaxFit);
    void *fidx = take(sizeof(int) * kMaxFit);
    void *ipiv = take(sizeof(int) * kMaxFit);
    void *ctl = take(sizeof(int) * C_NCTL);
    if (s) {
        s->F = (double4 *)F; s->alpha = (double *)alpha; s->covar = (double *)covar;
        s->beta = (double *)beta; s->da = (double *)da; s->a = (double *)a; s->atry = (double *)atry;
        s->T = (double *)T; s->TW = (double *)TW; s->rdy = (double *)rdy; s->rw = (double *)rw;
        s->ybuf = (double *)ybuf; s->mbar = (unsigned long long *)mbar; s->hist = (int *)hist;
        s->red = (double *)red; s->inv = (double *)inv; s->scal = (double *)scal;
        s->colbuf = (double *)colbuf; s->fidx = (int *)fidx; s->ipiv = (int *)ipiv; s->ctl = (int *)ctl;
        s->ld = ld; s->mfp = mfp;
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
// All warps sweep the facets in lockstep, kFacetChunk facets at a time; the
// chunk's basis rows (ncp doubles each) arrive in shared memory by bulk copy,
// double-buffered, so the shape-derivative loop reads broadcast shared-memory
// operands.  One warp = 32 points (lane = point), shape-derivative sums in
// registers.
template <int NCP>
__device__ void brightness_rows(const DevObject &o, const Sh &s, double *rows, const int *perm)
{
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int np = o.n_points, nf = o.n_fac, nc = o.n_coef, RS = o.row_stride;
    const double cl = s.inv[5], cls = s.inv[6];
    const int nchunks = (nf + kFacetChunk - 1) / kFacetChunk;
    const int ntiles = (np + 31) / 32;
    const int nrounds = (ntiles + kWarps - 1) / kWarps;
    const int total = nrounds * nchunks;
    int use[2] = {s.ctl[C_YUSE0], s.ctl[C_YUSE1]};  // completed waits per buffer (parity source)
    bool timeout = false;

    auto issue = [&](int g) {
        const int c = g % nchunks, f0 = c * kFacetChunk;
        const int rows_c = min(kFacetChunk, nf - f0);
        const int b = g & 1;
        bulk_load(s.ybuf + (size_t)b * kFacetChunk * NCP, o.ysh + (size_t)f0 * NCP,
                  (uint32_t)(rows_c * NCP * sizeof(double)), &s.mbar[b]);
    };
    if (tid == 0)
        for (int g = 0; g < 2 && g < total; ++g) issue(g);

    int g = 0;
    for (int round = 0; round < nrounds; ++round) {
        const int tile = round * kWarps + warp;
        const bool tile_act = tile < ntiles;
        const int idx = tile * 32 + lane;
        const bool act = tile_act && idx < np;
        const int p = perm[min(idx, np - 1)];
        double t = 0, ee[3] = {0, 0, 0}, es[3] = {0, 0, 0};
        {
            const double4 pa = ldg4(&o.pt_a[p]);
            const double4 pb = ldg4(&o.pt_b[p]);
            t = pa.x;
            ee[0] = pa.y; ee[1] = pa.z; ee[2] = pa.w;
            es[0] = pb.x; es[1] = pb.y; es[2] = pb.z;
        }
        PointGeo geo;
        point_geometry<false>(s.inv, t, ee, es, geo);
        const double ex = geo.e[0], ey = geo.e[1], ez = geo.e[2];
        const double sx = geo.e0[0], sy = geo.e0[1], sz = geo.e0[2];

        double J[NCP];
#pragma unroll
        for (int k = 0; k < NCP; ++k) J[k] = 0.0;
        double br = 0, u0 = 0, u1 = 0, u2 = 0, w0 = 0, w1 = 0, w2 = 0, t4 = 0, t5 = 0;

        for (int c = 0; c < nchunks; ++c, ++g) {
            const int b = g & 1;
            if (!mbar_wait(&s.mbar[b], (uint32_t)(use[b] & 1))) timeout = true;
            if (tile_act) {
                const int f0 = c * kFacetChunk, f1 = min(nf, f0 + kFacetChunk);
                const double *yb = s.ybuf + (size_t)b * kFacetChunk * NCP;
#pragma unroll 1
                for (int fi = f0; fi < f1; ++fi) {
                    const double4 fr = s.F[fi];
                    const double mu = ex * fr.x + ey * fr.y + ez * fr.z;
                    const double mu0 = sx * fr.x + sy * fr.y + sz * fr.z;
                    const bool vis = act && (mu > kTiny) && (mu0 > kTiny);
                    if (__any_sync(0xffffffffu, vis)) {
                        // lanes that do not see the facet run the same arithmetic on
                        // finite stand-ins and contribute exact zeros
                        const double ar = vis ? fr.w : 0.0;
                        const double r = __drcp_rn(vis ? mu + mu0 : 1.0);
                        const double sv = mu * mu0 * (cl + cls * r);
                        const double q0 = mu0 * r, q1 = mu * r;
                        const double dsmu = cls * (q0 * q0) + cl * mu0;
                        const double dsmu0 = cls * (q1 * q1) + cl * mu;
                        const double amm = ar * mu * mu0;
                        const double w = ar * sv;
                        const double gg = ar * dsmu;
                        const double g0 = ar * dsmu0;
                        br += w;
                        u0 = fma(gg, fr.x, u0);
                        u1 = fma(gg, fr.y, u1);
                        u2 = fma(gg, fr.z, u2);
                        w0 = fma(g0, fr.x, w0);
                        w1 = fma(g0, fr.y, w1);
                        w2 = fma(g0, fr.z, w2);
                        t4 += amm;
                        t5 += amm * r;
                        const double2 *yr = reinterpret_cast<const double2 *>(yb + (size_t)(fi - f0) * NCP);
#pragma unroll
                        for (int k = 0; k < NCP / 2; ++k) {
                            const double2 y = yr[k];
                            J[2 * k] = fma(w, y.x, J[2 * k]);
                            J[2 * k + 1] = fma(w, y.y, J[2 * k + 1]);
                        }
                    }
                }
            }
            __syncthreads();  // every warp is done with buffer b
            use[b] += 1;
            if (tid == 0 && g + 2 < total) issue(g + 2);
        }

        if (tile_act) {
            point_geometry<true>(s.inv, t, ee, es, geo);
            const double t1 = (geo.db[0] * u0 + geo.db[1] * u1 + geo.db[2] * u2) +
                              (geo.d0b[0] * w0 + geo.d0b[1] * w1 + geo.d0b[2] * w2);
            const double t2 = (geo.dl[0] * u0 + geo.dl[1] * u1 + geo.dl[2] * u2) +
                              (geo.d0l[0] * w0 + geo.d0l[1] * w1 + geo.d0l[2] * w2);
            const double t3 = (geo.dw[0] * u0 + geo.dw[1] * u1) + (geo.d0w[0] * w0 + geo.d0w[1] * w1);
            if (act) {
                const double scale = geo.scale;
                double *row = rows + (size_t)p * RS;
#pragma unroll
                for (int k = 0; k < NCP; ++k)
                    if (k < nc) row[k] = scale * J[k];
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
        }
    }
    if (timeout) s.ctl[C_TIMEOUT] = 1;
    if (tid == 0) {
        s.ctl[C_YUSE0] = use[0];
        s.ctl[C_YUSE1] = use[1];
    }
}

// ---------------------------------------------------------------- phases C, D

struct AlphaAcc {
    double v[kBPT][4];
    int bj[kBPT], bk[kBPT];
    int nb;
};

__device__ __forceinline__ void alpha_blocks(int mfit, AlphaAcc &acc)
{
    const int nb = (mfit + 1) / 2;
    const int nblocks = nb * (nb + 1) / 2;
    acc.nb = 0;
#pragma unroll
    for (int i = 0; i < kBPT; ++i) {
        int b = threadIdx.x + i * kThreads;
        int bj = 0, bk = 0;
        if (b < nblocks) {
            bj = (int)((sqrt(8.0 * b + 1.0) - 1.0) * 0.5);
            while ((bj + 1) * (bj + 2) / 2 <= b) ++bj;
            while (bj * (bj + 1) / 2 > b) --bj;
            bk = b - bj * (bj + 1) / 2;
            acc.nb = i + 1;
        }
        acc.bj[i] = bj;
        acc.bk[i] = bk;
#pragma unroll
        for (int q = 0; q < 4; ++q) acc.v[i][q] = 0.0;
    }
}

// Accumulates one staged tile of nrows rows into alpha, beta and chi^2.
__device__ __forceinline__ void tile_update(const Sh &s, int mfit, int nrows, AlphaAcc &acc,
                                            double &beta_j, double &chisq)
{
    const int mfp = s.mfp;
#pragma unroll
    for (int i = 0; i < kBPT; ++i) {
        if (i < acc.nb) {
            const int j0 = 2 * acc.bj[i], k0 = 2 * acc.bk[i];
            double a00 = acc.v[i][0], a01 = acc.v[i][1], a10 = acc.v[i][2], a11 = acc.v[i][3];
            for (int rr = 0; rr < nrows; ++rr) {
                const double2 tw = *reinterpret_cast<const double2 *>(s.TW + rr * mfp + j0);
                const double2 tt = *reinterpret_cast<const double2 *>(s.T + rr * mfp + k0);
                a00 = fma(tw.x, tt.x, a00);
                a01 = fma(tw.x, tt.y, a01);
                a10 = fma(tw.y, tt.x, a10);
                a11 = fma(tw.y, tt.y, a11);
            }
            acc.v[i][0] = a00; acc.v[i][1] = a01; acc.v[i][2] = a10; acc.v[i][3] = a11;
        }
    }
    if (threadIdx.x < mfit)
        for (int rr = 0; rr < nrows; ++rr) beta_j = fma(s.rdy[rr], s.TW[rr * mfp + threadIdx.x], beta_j);
    if (threadIdx.x == 0)
        for (int rr = 0; rr < nrows; ++rr) chisq = fma(s.rdy[rr] * s.rdy[rr], s.rw[rr], chisq);
}

// One full evaluation (mrqcof) at parameter vector a in shared memory.
// Writes alpha (symmetric, stride ld) to dst, beta to dvec; returns chi^2 to
// every thread.
template <int NCP>
__device__ double evaluate(const DevObject &o, const DevParams &p, const Sh &s, const double *a,
                           double *dst, double *dvec, double *rows, double *cstat, int *perm, double conw_r)
{
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int ma = o.ma, mfit = o.mfit, mfp = s.mfp, RS = o.row_stride, CS = ma + 3;

    double area_sum = shape_areas(o, s, a);
    if (tid == 0) s.scal[S_AREA] = area_sum;
    set_invariants(o, p, s, a);

    sort_points(o, s, perm, perm + o.n_points);
    brightness_rows<NCP>(o, s, rows, perm);
    __syncthreads();

    // per relative curve: column sums, 1/sum(ymod) and the renormalisation coefficient
    for (int c = warp; c < o.n_curves; c += kWarps) {
        if (!o.curve_rel[c]) continue;
        const int p0 = o.curve_start[c], p1 = o.curve_start[c + 1];
        for (int col = lane; col <= ma; col += 32) {
            double sum = 0;
            for (int q = p0; q < p1; ++q) sum += rows[(size_t)q * RS + col];
            cstat[(size_t)c * CS + col] = sum;
        }
        __syncwarp();
        if (lane == 0) {
            double rave = 1.0 / cstat[(size_t)c * CS + ma];
            cstat[(size_t)c * CS + ma + 1] = rave;
            cstat[(size_t)c * CS + ma + 2] = o.curve_sig[c] * (p1 - p0) * rave;
        }
    }
    __syncthreads();

    AlphaAcc acc;
    alpha_blocks(mfit, acc);
    double beta_j = 0.0, chisq = 0.0;

    const int np = o.n_points;
    for (int r0 = 0; r0 < np; r0 += kTile) {
        const int nrows = min(kTile, np - r0);
        for (int idx = tid; idx < kTile * mfp; idx += kThreads) {
            const int rr = idx / mfp, j = idx - rr * mfp;
            const int q = r0 + rr;
            double v = 0.0, vw = 0.0;
            if (rr < nrows && j < mfit) {
                const int col = s.fidx[j] - 1;
                const double raw = rows[(size_t)q * RS + col];
                const int c = __ldg(&o.pt_curve[q]);
                if (__ldg(&o.curve_rel[c])) {
                    const double *cs = cstat + (size_t)c * CS;
                    const double coef1 = rows[(size_t)q * RS + ma] * cs[ma + 1];
                    v = cs[ma + 2] * (raw - coef1 * cs[col]);
                } else {
                    v = raw;
                }
                vw = v * __ldg(&o.pt_w[q]);
            }
            s.T[idx] = v;
            s.TW[idx] = vw;
        }
        if (tid < kTile) {
            double dy = 0.0, w = 0.0;
            if (tid < nrows) {
                const int q = r0 + tid;
                const int c = __ldg(&o.pt_curve[q]);
                double ymod = rows[(size_t)q * RS + ma];
                if (__ldg(&o.curve_rel[c])) ymod = cstat[(size_t)c * CS + ma + 2] * ymod;
                dy = __ldg(&o.pt_b[q].w) - ymod;
                w = __ldg(&o.pt_w[q]);
            }
            s.rdy[tid] = dy;
            s.rw[tid] = w;
        }
        __syncthreads();
        tile_update(s, mfit, nrows, acc, beta_j, chisq);
        __syncthreads();
    }

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
        // raw derivative d ym_i / d a_k for shape coefficient k = tid
        double dk[3] = {0, 0, 0};
        if (tid < nc) {
            for (int fi = 0; fi < nf; ++fi) {
                const double4 fr = s.F[fi];
                const double y = __ldg(o.ysh + (size_t)fi * o.ncp + tid);
                dk[0] += (fr.w * fr.x) * y;
                dk[1] += (fr.w * fr.y) * y;
                dk[2] += (fr.w * fr.z) * y;
            }
            s.colbuf[tid] = 0.0;
        }
        // stage: param k (1-based k+1) maps to fit slot j via fidx; non-shape columns are 0
        const double wps = conw_r * conw_r;
        for (int idx = tid; idx < kTile * mfp; idx += kThreads) {
            s.T[idx] = 0.0;
            s.TW[idx] = 0.0;
        }
        __syncthreads();
        if (tid < nc) {
            // fit slot of parameter tid+1, if fitted
            int slot = -1;
            for (int j = 0; j < mfit; ++j)
                if (s.fidx[j] == tid + 1) slot = j;
            if (slot >= 0)
                for (int i = 0; i < 3; ++i) {
                    s.T[i * mfp + slot] = dk[i];
                    s.TW[i * mfp + slot] = dk[i] * wps;
                }
        }
        if (tid < 3) {
            s.rdy[tid] = 0.0 - ym[tid];
            s.rw[tid] = wps;
        }
        __syncthreads();
        tile_update(s, mfit, 3, acc, beta_j, chisq);
    }

    // write alpha (lower triangle mirrored), beta, chi^2
#pragma unroll
    for (int i = 0; i < kBPT; ++i) {
        if (i < acc.nb) {
            const int j0 = 2 * acc.bj[i], k0 = 2 * acc.bk[i];
            const int ld = s.ld;
            const double a00 = acc.v[i][0], a01 = acc.v[i][1], a10 = acc.v[i][2], a11 = acc.v[i][3];
            if (j0 == k0) {
                dst[j0 * ld + j0] = a00;
                if (j0 + 1 < mfit) {
                    dst[(j0 + 1) * ld + j0] = a10;
                    dst[j0 * ld + j0 + 1] = a10;
                    dst[(j0 + 1) * ld + j0 + 1] = a11;
                }
            } else {
                dst[j0 * ld + k0] = a00;
                dst[k0 * ld + j0] = a00;
                if (k0 + 1 < mfit) {
                    dst[j0 * ld + k0 + 1] = a01;
                    dst[(k0 + 1) * ld + j0] = a01;
                }
                if (j0 + 1 < mfit) {
                    dst[(j0 + 1) * ld + k0] = a10;
                    dst[k0 * ld + j0 + 1] = a10;
                    if (k0 + 1 < mfit) {
                        dst[(j0 + 1) * ld + k0 + 1] = a11;
                        dst[(k0 + 1) * ld + j0 + 1] = a11;
                    }
                }
            }
        }
    }
    if (tid < mfit) dvec[tid] = beta_j;
    if (tid == 0) s.scal[S_TRIAL] = chisq;
    __syncthreads();
    return s.scal[S_TRIAL];
}

// ---------------------------------------------------------------- LM step

// Full-pivot Gauss-Jordan on covar (n x n, stride ld) and b = da
// (mrqmin_1_end_opt, Start.cu:2880-3006).  Pivot: last maximum |a| in
// row-major order over unpivoted rows and columns.  Returns the error code.
static __device__ int gauss_jordan(const Sh &s, int n)
{
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int ld = s.ld;
    double *A = s.covar, *b = s.da;
    if (tid < n) s.ipiv[tid] = 0;
    if (tid == 0) s.ctl[C_ERR] = 0;
    __syncthreads();
    for (int i = 0; i < n; ++i) {
        // pivot search: thread j scans row j
        double big = -1.0;
        int jr = 0, kc = 0;
        if (tid < n && s.ipiv[tid] != 1) {
            const double *row = A + tid * ld;
            for (int k = 0; k < n; ++k) {
                const int ik = s.ipiv[k];
                if (ik == 0) {
                    const double t = fabs(row[k]);
                    if (t >= big) {
                        big = t;
                        jr = tid;
                        kc = k;
                    }
                } else if (ik > 1) {
                    s.ctl[C_ERR] = 1;
                }
            }
        }
        // CTA argmax on (big, row); ties go to the larger row
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            const double ob = __shfl_down_sync(0xffffffffu, big, off);
            const int oj = __shfl_down_sync(0xffffffffu, jr, off);
            const int ok = __shfl_down_sync(0xffffffffu, kc, off);
            if (ob > big || (ob == big && oj > jr)) {
                big = ob;
                jr = oj;
                kc = ok;
            }
        }
        if (lane == 0) {
            s.red[warp * 4 + 0] = big;
            s.red[warp * 4 + 1] = (double)jr;
            s.red[warp * 4 + 2] = (double)kc;
        }
        __syncthreads();
        if (s.ctl[C_ERR]) break;
        if (tid == 0) {
            double bb = s.red[0];
            int bjr = (int)s.red[1], bkc = (int)s.red[2];
            for (int w = 1; w < kWarps; ++w) {
                const double ob = s.red[w * 4];
                const int oj = (int)s.red[w * 4 + 1];
                if (ob > bb || (ob == bb && oj > bjr)) {
                    bb = ob;
                    bjr = oj;
                    bkc = (int)s.red[w * 4 + 2];
                }
            }
            if (bb < 0.0) {  // nothing but NaN left: same fallback as the serial scan
                bjr = 0;
                bkc = 0;
            }
            s.ipiv[bkc] += 1;
            s.ctl[C_IROW] = bjr;
            s.ctl[C_ICOL] = bkc;
        }
        __syncthreads();
        const int irow = s.ctl[C_IROW], icol = s.ctl[C_ICOL];
        if (irow != icol) {
            for (int l = tid; l < n; l += kThreads) {
                const double t = A[irow * ld + l];
                A[irow * ld + l] = A[icol * ld + l];
                A[icol * ld + l] = t;
            }
            if (tid == 0) {
                const double t = b[irow];
                b[irow] = b[icol];
                b[icol] = t;
            }
        }
        __syncthreads();
        const double piv = A[icol * ld + icol];
        if (piv == 0.0) {
            if (tid == 0) s.ctl[C_ERR] = 2;
            __syncthreads();
            break;
        }
        const double pivinv = 1.0 / piv;
        __syncthreads();
        for (int l = tid; l < n; l += kThreads) A[icol * ld + l] = (l == icol) ? pivinv : A[icol * ld + l] * pivinv;
        if (tid == 0) b[icol] *= pivinv;
        for (int ll = tid; ll < n; ll += kThreads) s.colbuf[ll] = A[ll * ld + icol];
        __syncthreads();
        // eliminate: only unpivoted columns feed later pivots and b
        for (int idx = tid; idx < n * n; idx += kThreads) {
            const int ll = idx / n, l = idx - ll * n;
            if (ll == icol || s.ipiv[l] != 0) continue;
            A[ll * ld + l] -= A[icol * ld + l] * s.colbuf[ll];
        }
        for (int ll = tid; ll < n; ll += kThreads)
            if (ll != icol) b[ll] -= b[icol] * s.colbuf[ll];
        __syncthreads();
    }
    __syncthreads();
    return s.ctl[C_ERR];
}

// ---------------------------------------------------------------- kernel

template <int NCP>
__global__ void __launch_bounds__(kThreads, 1)
fit_kernel(DevObject o, DevParams p, const FitItem *items, int n_items, int *queue, FitOut *out,
           double *scratch, size_t scratch_per_cta, int *status, EvalOut ev, int mode)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Sh s;
    carve_bytes(o.n_fac, o.mfit, o.ncp, &s, smem_raw);
    const int tid = threadIdx.x;
    const int nc = o.n_coef, ma = o.ma, mfit = o.mfit, ld = s.ld;
    double *rows = scratch + (size_t)blockIdx.x * scratch_per_cta;
    double *cstat = rows + (size_t)o.n_points * o.row_stride;
    int *perm = reinterpret_cast<int *>(cstat + (size_t)o.n_curves * (ma + 3));  // [2][n_points]

    for (int f = tid; f < o.n_fac; f += kThreads) s.F[f] = ldg4(&o.facet[f]);
    if (tid < mfit) s.fidx[tid] = __ldg(&o.fidx[tid]);
    if (tid == 0) {
        mbar_init(&s.mbar[0], 1);
        mbar_init(&s.mbar[1], 1);
        s.ctl[C_YUSE0] = 0;
        s.ctl[C_YUSE1] = 0;
        s.ctl[C_TIMEOUT] = 0;
    }
    __syncthreads();

    if (mode == 1) {  // one stand-alone evaluation (parity hook)
        for (int q = tid; q <= ma; q += kThreads) s.a[q] = ev.a[q];
        __syncthreads();
        double chisq = evaluate<NCP>(o, p, s, s.a, s.alpha, s.beta, rows, cstat, perm, p.conw_r);
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

    for (;;) {
        if (tid == 0) s.ctl[C_ITEM] = atomicAdd(queue, 1);
        __syncthreads();
        const int item = s.ctl[C_ITEM];
        if (item >= n_items) break;

        // initial parameters (CudaCalculatePreparePole, Start.cu:4346-4418)
        if (tid == 0) {
            const FitItem it = items[item];
            double *a = s.a;
            a[0] = 0;
            for (int k = 1; k <= nc; ++k) a[k] = __ldg(&o.cg_first[k - 1]);
            const double period = 1.0 / (p.freq_start - (it.n_freq - 1) * p.freq_step);
            a[nc + 1] = (kPi / 180) * 90 - (kPi / 180) * p.beta_pole[it.pole];
            a[nc + 2] = (kPi / 180) * p.lambda_pole[it.pole];
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
                double oc = evaluate<NCP>(o, p, s, s.a, s.alpha, s.beta, rows, cstat, perm, p.conw_r);
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
            const int err = gauss_jordan(s, mfit);
            if (err == 0 || err == 2) {
                if (tid < mfit) s.atry[s.fidx[tid]] = s.a[s.fidx[tid]] + s.da[tid];
                if (err == 2 && tid == 0) s.ctl[C_STATUS] |= kStatusSingular;
            }
            __syncthreads();
            const double chisq = evaluate<NCP>(o, p, s, s.atry, s.covar, s.da, rows, cstat, perm, p.conw_r);
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
        }
        __syncthreads();
        if (s.ctl[C_TIMEOUT]) break;  // a bulk copy never completed: stop taking items
    }
    // after a timeout, give any copy still in flight a bounded chance to land
    // before the CTA's shared memory is released
    if (tid == 0 && s.ctl[C_TIMEOUT]) {
        mbar_wait(&s.mbar[0], (uint32_t)(s.ctl[C_YUSE0] & 1));
        mbar_wait(&s.mbar[1], (uint32_t)(s.ctl[C_YUSE1] & 1));
    }
}

}  // namespace psb
