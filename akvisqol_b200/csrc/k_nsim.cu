// NSIM patch similarity (reference src/nsim.zig) for the DP table and the
// per-match band statistics.
//
// Table: NSIM of every reference patch at every degraded offset in its
// search window (reference src/accel.zig:126-146, measureSimilarityAt
// src/nsim.zig:364-424). One thread owns one (patch, offset) and walks the
// patch's cells in row-major order, so its serial sum is the CPU's order.
// The threads of a CTA share one reference patch: its values and its
// precomputed terms (3x3 mean, mean², variance) sit in shared memory and
// are read as broadcasts; the degraded plane's terms come from global
// memory, and neighbouring threads read neighbouring offsets (coalesced).
// Interior patch columns reuse the plane's terms, whose 3x3 neighbourhood
// is the patch's; the two edge columns are recomputed with the patch's
// replicate padding, as the CPU does.
#include <algorithm>

#include "device.cuh"
#include "kernels.h"

namespace vqb {

namespace {

// sign(v) sqrt(|v|): the fast forms store variances as signed roots, so a
// cell's sqrt(srs * sds) becomes a product of two stored roots (and
// srs * sds < 0 exactly when the roots' product is negative).
__device__ inline double signed_root(double v) { return v < 0.0 ? -sqrt(-v) : sqrt(v); }

// Degraded plane of one pair: the prepared spectrogram zero-padded to
// `width` frames, its 3x3 mean, mean² and variance (reference
// src/nsim.zig:236-263). out arrays are nb x width.
__global__ void __launch_bounds__(256) plane_kernel(const PlaneJob *__restrict__ jobs, int nb) {
    const PlaneJob job = jobs[blockIdx.y];
    const int w = job.width, nf = job.nf;
    const int total = nb * w;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += gridDim.x * blockDim.x) {
        const int r = e / w, c = e - r * w;
        const int rm = r == 0 ? 0 : r - 1, rp = r + 1 >= nb ? nb - 1 : r + 1;
        const int cm = c == 0 ? 0 : c - 1, cp = c + 1 >= w ? w - 1 : c + 1;
        auto P = [&](int rr, int cc) -> double { return cc < nf ? job.spec[(int64_t)rr * nf + cc] : 0.0; };
        const double p00 = P(rm, cm), p01 = P(rm, c), p02 = P(rm, cp);
        const double p10 = P(r, cm), p11 = P(r, c), p12 = P(r, cp);
        const double p20 = P(rp, cm), p21 = P(rp, c), p22 = P(rp, cp);
        const double mu = taps9(p00, p01, p02, p10, p11, p12, p20, p21, p22);
        const double csq = taps9(p00 * p00, p01 * p01, p02 * p02, p10 * p10, p11 * p11, p12 * p12, p20 * p20,
                                 p21 * p21, p22 * p22);
        const double dms = mu * mu;
        job.pad[e] = p11;
        job.mu[e] = mu;
        job.dms[e] = dms;
        job.sds[e] = job.roots ? signed_root(csq - dms) : csq - dms;
    }
}

// Reference-patch terms (reference precomputeRef, src/nsim.zig:318-329):
// out[4][nb][P] = {patch values, 3x3 mean, mean², conv(x²) - mean²}.
__global__ void __launch_bounds__(256) ref_terms_kernel(const RefTermsJob *__restrict__ jobs, int nb, int P) {
    const RefTermsJob job = jobs[blockIdx.y];
    const int total = nb * P;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += gridDim.x * blockDim.x) {
        const int r = e / P, c = e - r * P;
        const int rm = r == 0 ? 0 : r - 1, rp = r + 1 >= nb ? nb - 1 : r + 1;
        const int cm = c == 0 ? 0 : c - 1, cp = c + 1 >= P ? P - 1 : c + 1;
        auto R = [&](int rr, int cc) -> double { return job.spec[(int64_t)rr * job.nf + job.col + cc]; };
        const double p00 = R(rm, cm), p01 = R(rm, c), p02 = R(rm, cp);
        const double p10 = R(r, cm), p11 = R(r, c), p12 = R(r, cp);
        const double p20 = R(rp, cm), p21 = R(rp, c), p22 = R(rp, cp);
        const double mu = taps9(p00, p01, p02, p10, p11, p12, p20, p21, p22);
        const double csq = taps9(p00 * p00, p01 * p01, p02 * p02, p10 * p10, p11 * p11, p12 * p12, p20 * p20,
                                 p21 * p21, p22 * p22);
        const double rms = mu * mu;
        job.out[e] = p11;
        job.out[total + e] = mu;
        job.out[2 * total + e] = rms;
        job.out[3 * total + e] = job.roots ? signed_root(csq - rms) : csq - rms;
    }
}

constexpr int kTableThreads = 128;  // default offsets per CTA

// The fast forms' cell arithmetic: the 3x3 window as an FMA chain and the
// cell's two quotients as one, (2 mr md + c1)(srd + c3) /
// ((rms + dms + c1)(sqrt(srs sds) + c3)), about half the f64 instructions of
// the exact cell; values agree with it to a few ulp.
__device__ inline double taps9_fma(double a00, double a01, double a02, double a10, double a11, double a12,
                                   double a20, double a21, double a22) {
    double t = kW0 * a00;
    t = __fma_rn(kW1, a01, t);
    t = __fma_rn(kW0, a02, t);
    t = __fma_rn(kW1, a10, t);
    t = __fma_rn(kW2, a11, t);
    t = __fma_rn(kW1, a12, t);
    t = __fma_rn(kW0, a20, t);
    t = __fma_rn(kW1, a21, t);
    return __fma_rn(kW0, a22, t);
}

// sr, sd: signed roots of the reference and degraded variances.
__device__ inline double sim_cell_fast(double mr, double rms, double sr, double md, double dms, double sd,
                                       double crd) {
    const double mrd = mr * md;
    const double srd = crd - mrd;
    const double q = sr * sd;
    const double sden = q < 0.0 ? kC3 : fabs(q) + kC3;
    return (__fma_rn(2.0, mrd, kC1) * (srd + kC3)) / ((rms + dms + kC1) * sden);
}

template <bool kFast>
__device__ inline double taps(double a00, double a01, double a02, double a10, double a11, double a12, double a20,
                              double a21, double a22) {
    return kFast ? taps9_fma(a00, a01, a02, a10, a11, a12, a20, a21, a22)
                 : taps9(a00, a01, a02, a10, a11, a12, a20, a21, a22);
}

// One thread per (patch, offset); CTA = one patch x 128 offsets.
template <bool kFast, int kThreads>
__global__ void __launch_bounds__(kThreads) table_kernel(const TableTask *__restrict__ tasks, int nb, int P) {
    extern __shared__ double sm[];
    const TableTask t = tasks[blockIdx.x];
    const int total = nb * P;
    for (int e = threadIdx.x; e < 4 * total; e += blockDim.x) sm[e] = t.ref_terms[e];
    __syncthreads();
    const int64_t off = t.off0 + threadIdx.x;
    if (off > t.hi) return;
    const double *rv = sm, *mr = sm + total, *rms = sm + 2 * total, *srs = sm + 3 * total;
    const int w = t.width;
    const double *pad = t.pad, *mu = t.mu, *dmsp = t.dms, *sdsp = t.sds;
    double sum = 0.0;
    for (int r = 0; r < nb; ++r) {
        const int rm = r == 0 ? 0 : r - 1, rp = r + 1 >= nb ? nb - 1 : r + 1;
        const double *pm = pad + (int64_t)rm * w + off, *p0 = pad + (int64_t)r * w + off,
                     *pp = pad + (int64_t)rp * w + off;
        const double *qm = rv + rm * P, *q0 = rv + r * P, *qp = rv + rp * P;
        // ref x deg products of the 3 rows, columns (c-1, c, c+1) clamped
        // to the patch; slid along c.
        double am = qm[0] * pm[0], a0 = q0[0] * p0[0], ap = qp[0] * pp[0];  // column cm
        double bm = am, b0 = a0, bp = ap;                                   // column c
        for (int c = 0; c < P; ++c) {
            const int cp = c + 1 >= P ? P - 1 : c + 1;
            const double cm_ = qm[cp] * pm[cp], c0 = q0[cp] * p0[cp], cpp = qp[cp] * pp[cp];
            // Taps.row over the patch's ref x deg products.
            const double crd = taps<kFast>(am, bm, cm_, a0, b0, c0, ap, bp, cpp);
            double md, dms, sds;
            if (c == 0 || c == P - 1) {
                const int cmi = c == 0 ? 0 : c - 1;
                const double d00 = pm[cmi], d01 = pm[c], d02 = pm[cp];
                const double d10 = p0[cmi], d11 = p0[c], d12 = p0[cp];
                const double d20 = pp[cmi], d21 = pp[c], d22 = pp[cp];
                md = taps<kFast>(d00, d01, d02, d10, d11, d12, d20, d21, d22);
                const double cdsq = taps<kFast>(d00 * d00, d01 * d01, d02 * d02, d10 * d10, d11 * d11, d12 * d12,
                                                d20 * d20, d21 * d21, d22 * d22);
                dms = md * md;
                sds = kFast ? signed_root(cdsq - dms) : cdsq - dms;
            } else {
                const int64_t pi = (int64_t)r * w + off + c;
                md = mu[pi];
                dms = dmsp[pi];
                sds = sdsp[pi];
            }
            const int ri = r * P + c;
            sum += kFast ? sim_cell_fast(mr[ri], rms[ri], srs[ri], md, dms, sds, crd)
                         : sim_cell(mr[ri], rms[ri], srs[ri], md, dms, sds, crd);
            // slide: column c becomes cm, column cp becomes c
            am = bm, a0 = b0, ap = bp;
            bm = cm_, b0 = c0, bp = cpp;
        }
    }
    t.out[off] = sum / (double)(nb * P);
}

// The table with the patch width P known at compile time (30 in audio
// mode, 20 in speech mode) and W offsets per CTA. The exact form (kFast
// false) computes the cells of table_kernel<false, W> with the same
// operations in the same order; the fast forms (kFast true) compute
// table_kernel<true, W>'s cells, which need not follow the CPU's order,
// arranged for throughput:
//
// * the degraded plane's rows and the reference terms' rows are streamed
//   through shared memory, one band row at a time and double-buffered with
//   asynchronous copies: row r needs the padded spectrogram's rows r-1, r,
//   r+1 and the 3x3 mean, mean^2 and variance planes' row r over the CTA's
//   columns [off0, off0 + W + P - 1), and the same rows of the reference
//   patch's terms (about 18 KB of shared memory per CTA at W = 128, so
//   that register use, not shared memory, bounds the CTAs per SM);
// * the 3x3 window of the ref x deg products uses per-column sums (the
//   window is symmetric: corners, edges, centre), about 7 operations per
//   cell at dependency depth ~4 instead of a 9-deep FMA chain;
// * the cell's one quotient divides by a positive denominator with a
//   reciprocal estimate refined by Newton-Raphson iterations (Markstein's
//   refinement: r' = r + r(1 - d r), then q' = q + r'(n - d q)), which
//   agrees with the IEEE quotient to about an ulp.
__device__ inline double fast_quotient(double n, double d) {
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(d));
    r = __fma_rn(r, __fma_rn(-d, r, 1.0), r);
    r = __fma_rn(r, __fma_rn(-d, r, 1.0), r);
    const double q = n * r;
    return __fma_rn(r, __fma_rn(-d, q, n), q);
}

__device__ inline double sim_cell_quick(double mr, double rms, double sr, double md, double dms, double sd,
                                        double crd) {
    const double mrd = mr * md;
    const double srd = crd - mrd;
    const double q = sr * sd;
    const double sden = q < 0.0 ? kC3 : fabs(q) + kC3;
    return fast_quotient(__fma_rn(2.0, mrd, kC1) * (srd + kC3), (rms + dms + kC1) * sden);
}

constexpr int kStageRows = 6;  // pad rows r-1, r, r+1; mu, dms, sds rows r

__device__ inline void cp_async8(double *dst, const double *src, int bytes) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(src), "r"(bytes) : "memory");
}

template <bool kFast, int P, int W>
__global__ void __launch_bounds__(W) table_staged_kernel(const TableTask *__restrict__ tasks, int nb) {
    extern __shared__ __align__(16) double smf[];
    constexpr int kSpan = W + P - 1;                        // degraded columns a CTA reads
    constexpr int kStage = kStageRows * kSpan + kStageRows * P;  // one band row's stage
    const TableTask t = tasks[blockIdx.x];
    const int total = nb * P;
    const int w = t.width;
    // Row r's stage: the degraded plane's rows (pad r-1, r, r+1; mu, dms, sds
    // r) over the CTA's columns, then the reference terms' rows (values r-1,
    // r, r+1; mean, mean^2, variance r) over the patch's P columns.
    auto fetch = [&](int r, int buf) {
        const int rm = r == 0 ? 0 : r - 1, rp = r + 1 >= nb ? nb - 1 : r + 1;
        double *dst = smf + buf * kStage;
        for (int e = threadIdx.x; e < kStageRows * kSpan; e += W) {
            const int k = e / kSpan, col = t.off0 + (e - k * kSpan);
            const int row = k == 0 ? rm : k == 2 ? rp : r;
            const double *plane = k < 3 ? t.pad : k == 3 ? t.mu : k == 4 ? t.dms : t.sds;
            const double *src = plane + (int64_t)row * w;
            const bool in = col < w;
            cp_async8(dst + e, in ? src + col : src, in ? 8 : 0);
        }
        double *tdst = dst + kStageRows * kSpan;
        for (int e = threadIdx.x; e < kStageRows * P; e += W) {
            const int k = e / P, c = e - k * P;
            const int row = k == 0 ? rm : k == 2 ? rp : r;
            const int term = k < 3 ? 0 : k - 2;  // values, mean, mean^2, variance
            cp_async8(tdst + e, t.ref_terms + term * total + row * P + c, 8);
        }
        asm volatile("cp.async.commit_group;\n" ::: "memory");
    };
    fetch(0, 0);
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    __syncthreads();
    const int64_t off = t.off0 + threadIdx.x;
    double sum = 0.0;
    for (int r = 0; r < nb; ++r) {
        if (r + 1 < nb) fetch(r + 1, (r + 1) & 1);
        const double *stg = smf + (r & 1) * kStage;
        const double *st = stg + threadIdx.x;
        const double *pm = st, *p0 = st + kSpan, *pp = st + 2 * kSpan;
        const double *mu = st + 3 * kSpan, *dm = st + 4 * kSpan, *sd = st + 5 * kSpan;
        const double *tr = stg + kStageRows * kSpan;
        const double *qm = tr, *q0 = tr + P, *qp = tr + 2 * P, *mr = tr + 3 * P, *rms = tr + 4 * P, *srs = tr + 5 * P;
        if (kFast) {
            // column sums of the ref x deg products: E = rows r-1 + r+1, M = row r
            double Ec = qm[0] * pm[0] + qp[0] * pp[0], Mc = q0[0] * p0[0];
            double Em = Ec, Mm = Mc;
#pragma unroll
            for (int c = 0; c < P; ++c) {
                const int cp = c + 1 < P ? c + 1 : P - 1;
                double Ep = Ec, Mp = Mc;
                if (c + 1 < P) {
                    Ep = qm[cp] * pm[cp] + qp[cp] * pp[cp];
                    Mp = q0[cp] * p0[cp];
                }
                const double crd = __fma_rn(kW2, Mc, __fma_rn(kW1, (Mm + Mp) + Ec, kW0 * (Em + Ep)));
                double md, dms, sds;
                if (c == 0 || c == P - 1) {
                    const int cm = c == 0 ? 0 : c - 1;
                    const double d00 = pm[cm], d01 = pm[c], d02 = pm[cp];
                    const double d10 = p0[cm], d11 = p0[c], d12 = p0[cp];
                    const double d20 = pp[cm], d21 = pp[c], d22 = pp[cp];
                    md = taps9_fma(d00, d01, d02, d10, d11, d12, d20, d21, d22);
                    const double cdsq = taps9_fma(d00 * d00, d01 * d01, d02 * d02, d10 * d10, d11 * d11,
                                                  d12 * d12, d20 * d20, d21 * d21, d22 * d22);
                    dms = md * md;
                    sds = signed_root(cdsq - dms);
                } else {
                    md = mu[c];
                    dms = dm[c];
                    sds = sd[c];
                }
                sum += sim_cell_quick(mr[c], rms[c], srs[c], md, dms, sds, crd);
                Em = Ec, Mm = Mc;
                Ec = Ep, Mc = Mp;
            }
        } else {
            // exact: the operations and order of table_kernel<false> (the
            // CPU's cell, src/nsim.zig:293-308, and its row-major sum), with
            // the operands read from the stage
            double am = qm[0] * pm[0], a0 = q0[0] * p0[0], ap = qp[0] * pp[0];  // column cm
            double bm = am, b0 = a0, bp = ap;                                   // column c
#pragma unroll
            for (int c = 0; c < P; ++c) {
                const int cp = c + 1 >= P ? P - 1 : c + 1;
                const double cm_ = qm[cp] * pm[cp], c0 = q0[cp] * p0[cp], cpp = qp[cp] * pp[cp];
                const double crd = taps9(am, bm, cm_, a0, b0, c0, ap, bp, cpp);
                double md, dms, sds;
                if (c == 0 || c == P - 1) {
                    const int cmi = c == 0 ? 0 : c - 1;
                    const double d00 = pm[cmi], d01 = pm[c], d02 = pm[cp];
                    const double d10 = p0[cmi], d11 = p0[c], d12 = p0[cp];
                    const double d20 = pp[cmi], d21 = pp[c], d22 = pp[cp];
                    md = taps9(d00, d01, d02, d10, d11, d12, d20, d21, d22);
                    const double cdsq = taps9(d00 * d00, d01 * d01, d02 * d02, d10 * d10, d11 * d11, d12 * d12,
                                              d20 * d20, d21 * d21, d22 * d22);
                    dms = md * md;
                    sds = cdsq - dms;
                } else {
                    md = mu[c];
                    dms = dm[c];
                    sds = sd[c];
                }
                sum += sim_cell(mr[c], rms[c], srs[c], md, dms, sds, crd);
                am = bm, a0 = b0, ap = bp;
                bm = cm_, b0 = c0, bp = cpp;
            }
        }
        asm volatile("cp.async.wait_all;\n" ::: "memory");
        __syncthreads();
    }
    if (off <= t.hi) t.out[off] = sum / (double)(nb * P);
}

// Per-band statistics of one patch pair, one thread per band row
// (reference measurePatchSimilarity, src/nsim.zig:427-510). Cell values are
// formed from the 3x3 neighbourhood on the fly and recomputed for the
// stddev pass (same operations, same bits).
constexpr int kStatsCache = 64;  // a lane's cells kept between the mean and variance passes

__global__ void __launch_bounds__(32) stats_kernel(const StatsJob *__restrict__ jobs, int nb) {
    const StatsJob job = jobs[blockIdx.x];
    const int r = threadIdx.x;
    __shared__ double means_sm[32];
    __shared__ double cells_sm[kStatsCache][32];  // [column][lane]: each lane reads back its own
    int deg_col = job.deg_col;
    bool valid = true, reached = true;
    if (job.dp_offset) {
        const int64_t o = *job.dp_offset;
        reached = o >= 0;
        valid = *job.dp_valid != 0;
        deg_col = (int)(o < 0 ? 0 : o);
    }
    const int nc = job.ncols;
    if (!reached) {
        // Patches the backtrack never reached keep zeroed statistics.
        if (r < nb) job.means[r] = job.stddevs[r] = job.energy[r] = 0.0;
        if (r == 0) *job.similarity = 0.0;
        return;
    }
    auto R = [&](int rr, int cc) -> double { return job.ref[(int64_t)rr * job.ref_stride + job.ref_col + cc]; };
    auto D = [&](int rr, int cc) -> double {
        return deg_col + cc < job.deg_cols ? job.deg[(int64_t)rr * job.deg_stride + deg_col + cc] : 0.0;
    };
    double mean = 0.0;
    if (r < nb) {
        const int rm = r == 0 ? 0 : r - 1, rp = r + 1 >= nb ? nb - 1 : r + 1;
        const double inv_ncols = 1.0 / (double)nc;
        auto cell = [&](int c) -> double {
            const int cm = c == 0 ? 0 : c - 1, cp = c + 1 >= nc ? nc - 1 : c + 1;
            const double r00 = R(rm, cm), r01 = R(rm, c), r02 = R(rm, cp), r10 = R(r, cm), r11 = R(r, c),
                         r12 = R(r, cp), r20 = R(rp, cm), r21 = R(rp, c), r22 = R(rp, cp);
            const double d00 = D(rm, cm), d01 = D(rm, c), d02 = D(rm, cp), d10 = D(r, cm), d11 = D(r, c),
                         d12 = D(r, cp), d20 = D(rp, cm), d21 = D(rp, c), d22 = D(rp, cp);
            const double mr = taps9(r00, r01, r02, r10, r11, r12, r20, r21, r22);
            const double md = taps9(d00, d01, d02, d10, d11, d12, d20, d21, d22);
            const double crs = taps9(r00 * r00, r01 * r01, r02 * r02, r10 * r10, r11 * r11, r12 * r12, r20 * r20,
                                     r21 * r21, r22 * r22);
            const double cds = taps9(d00 * d00, d01 * d01, d02 * d02, d10 * d10, d11 * d11, d12 * d12, d20 * d20,
                                     d21 * d21, d22 * d22);
            const double crd = taps9(r00 * d00, r01 * d01, r02 * d02, r10 * d10, r11 * d11, r12 * d12, r20 * d20,
                                     r21 * d21, r22 * d22);
            const double rms = mr * mr, dms = md * md;
            return sim_cell(mr, rms, crs - rms, md, dms, cds - dms, crd);
        };
        double deg_sum = 0.0;
        for (int c = 0; c < nc; ++c) deg_sum += D(r, c);
        job.energy[r] = deg_sum * inv_ncols;
        // the variance pass reuses the mean pass's cells (the same values)
        // where they fit, instead of computing each cell twice
        const bool cached = nc <= kStatsCache;
        double sim_sum = 0.0;
        for (int c = 0; c < nc; ++c) {
            const double v = cell(c);
            if (cached) cells_sm[c][r] = v;
            sim_sum += v;
        }
        mean = sim_sum * inv_ncols;
        double sd = 0.0;
        if (nc > 1) {
            double ss = 0.0;
            for (int c = 0; c < nc; ++c) {
                const double diff = (cached ? cells_sm[c][r] : cell(c)) - mean;
                ss += diff * diff;
            }
            sd = sqrt(ss / ((double)nc - 1.0));
        }
        job.stddevs[r] = sd;
        job.means[r] = valid ? mean : 0.0;
        means_sm[r] = mean;
    }
    __syncthreads();
    if (r == 0) {
        double acc = 0.0;
        for (int b = 0; b < nb; ++b) acc += means_sm[b];
        *job.similarity = valid ? acc / (double)nb : 0.0;
    }
}

// fast_quotient over arrays (its direct test against IEEE division).
__global__ void quotient_kernel(const double *__restrict__ num, const double *__restrict__ den,
                                double *__restrict__ out, size_t count) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (size_t)gridDim.x * blockDim.x)
        out[i] = fast_quotient(num[i], den[i]);
}

}  // namespace

void launch_plane(const PlaneJob *d_jobs, int njobs, int nb, int max_width, cudaStream_t s) {
    if (njobs <= 0) return;
    const int total = nb * max_width;
    int blocks = (total + 255) / 256;
    if (blocks > 1024) blocks = 1024;
    plane_kernel<<<dim3((unsigned)blocks, (unsigned)njobs), 256, 0, s>>>(d_jobs, nb);
    launch_counter() += 1;
}

void launch_ref_terms(const RefTermsJob *d_jobs, int njobs, int nb, int P, cudaStream_t s) {
    if (njobs <= 0) return;
    const int total = nb * P;
    const int blocks = (total + 255) / 256;
    ref_terms_kernel<<<dim3((unsigned)blocks, (unsigned)njobs), 256, 0, s>>>(d_jobs, nb, P);
    launch_counter() += 1;
}

int table_offsets_per_cta() { return kTableThreads; }

std::vector<int> table_width_candidates(int P) {
    // widths the staged kernels have for the audio and speech patch widths;
    // 64 would fall back to the unstaged kernel
    if (P == 30 || P == 20) return {128, 256};
    return {128, 64, 256};
}

void nsim_init_attributes() {
    cudaFuncSetAttribute(table_kernel<false, 64>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    cudaFuncSetAttribute(table_kernel<true, 64>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    cudaFuncSetAttribute(table_kernel<false, 128>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    cudaFuncSetAttribute(table_kernel<true, 128>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    cudaFuncSetAttribute(table_kernel<false, 256>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    cudaFuncSetAttribute(table_kernel<true, 256>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
#define VQB_STAGED_ATTR(F, PP, W) \
    cudaFuncSetAttribute(table_staged_kernel<F, PP, W>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    VQB_STAGED_ATTR(true, 30, 128)
    VQB_STAGED_ATTR(true, 30, 256)
    VQB_STAGED_ATTR(true, 20, 128)
    VQB_STAGED_ATTR(true, 20, 256)
    VQB_STAGED_ATTR(false, 30, 128)
    VQB_STAGED_ATTR(false, 30, 256)
    VQB_STAGED_ATTR(false, 20, 128)
    VQB_STAGED_ATTR(false, 20, 256)
#undef VQB_STAGED_ATTR
}

void launch_table(const TableTask *d_tasks, int ntasks, int nb, int P, bool fast, int width, cudaStream_t s) {
    if (ntasks <= 0) return;
    const size_t smem = (size_t)4 * nb * P * sizeof(double);
    if ((P == 30 || P == 20) && (width == 128 || width == 256)) {
        const size_t staged = (size_t)2 * kStageRows * ((width + P - 1) + P) * sizeof(double);
#define VQB_TABLE_STAGED(F, PP, W) table_staged_kernel<F, PP, W><<<ntasks, W, staged, s>>>(d_tasks, nb);
#define VQB_TABLE_STAGED_P(F)            \
    if (P == 30) {                       \
        if (width == 256) {              \
            VQB_TABLE_STAGED(F, 30, 256) \
        } else {                         \
            VQB_TABLE_STAGED(F, 30, 128) \
        }                                \
    } else {                             \
        if (width == 256) {              \
            VQB_TABLE_STAGED(F, 20, 256) \
        } else {                         \
            VQB_TABLE_STAGED(F, 20, 128) \
        }                                \
    }
        if (fast) {
            VQB_TABLE_STAGED_P(true)
        } else {
            VQB_TABLE_STAGED_P(false)
        }
#undef VQB_TABLE_STAGED_P
#undef VQB_TABLE_STAGED
        launch_counter() += 1;
        return;
    }
#define VQB_TABLE(W)                                                             \
    if (fast)                                                                    \
        table_kernel<true, W><<<ntasks, W, smem, s>>>(d_tasks, nb, P);           \
    else                                                                         \
        table_kernel<false, W><<<ntasks, W, smem, s>>>(d_tasks, nb, P);
    if (width == 64) {
        VQB_TABLE(64)
    } else if (width == 256) {
        VQB_TABLE(256)
    } else {
        VQB_TABLE(128)
    }
#undef VQB_TABLE
    launch_counter() += 1;
}

void launch_fast_quotient(const double *num, const double *den, double *out, size_t count, cudaStream_t s) {
    if (count == 0) return;
    const size_t blocks = std::min<size_t>((count + 255) / 256, 4096);
    quotient_kernel<<<(unsigned)blocks, 256, 0, s>>>(num, den, out, count);
    launch_counter() += 1;
}

void launch_stats(const StatsJob *d_jobs, int njobs, int nb, cudaStream_t s) {
    if (njobs <= 0) return;
    stats_kernel<<<njobs, 32, 0, s>>>(d_jobs, nb);
    launch_counter() += 1;
}

}  // namespace vqb
