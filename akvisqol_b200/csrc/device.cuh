// Device-side types shared by the kernels and the host pipeline.
//
// All exact-form arithmetic is f64 with no FMA contraction (the library is
// built with --fmad=false), so every product and sum rounds exactly as the
// reference's Zig CPU code does; kernels that must match a serial CPU loop
// keep its summation order.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace vqb {

// A signal as a window onto device memory:
// sample(k) = base[k - head] when 0 <= k - head < avail, else 0, for k < len.
// Covers zero-padded slices (reference src/realign.zig:24-51) and trimmed,
// lag-shifted views (src/realign.zig:212-250) without copies.
struct VSig {
    const double *base;
    int64_t head;
    int64_t avail;
    int64_t len;
};

__host__ __device__ inline double vsig_at(const VSig &s, int64_t k) {
    const int64_t j = k - s.head;
    return (uint64_t)j < (uint64_t)s.avail ? s.base[j] : 0.0;
}

// Per-band gammatone coefficients as filterBandRmsFresh uses them
// (reference src/gammatone.zig:268-278), precomputed on the host.
struct BandCoeffs {
    double s1n0, s1n1, s2n1, s3n1, s4n1, ca0, d1, d2;
};

// One spectrogram to compute: frames f < nf of `sig` at hop spacing,
// written to out[b * nf + f].
struct SpecJob {
    VSig sig;
    int64_t nf;
    double *out;
};

// Lag candidates the f32 correlation nominates (reference
// src/xcorr.zig:270-340): at most this many are rescored in f64.
constexpr int kLagCandCap = 64;

// One CTA's nomination record in the f32 lag search: its largest |Re| over
// valid lags, and every lag within the slack of that maximum (count may
// exceed kLagCandCap; then only the first kLagCandCap are stored).
struct LagCands {
    float top;
    int32_t count;
    float v[kLagCandCap];
    int32_t key[kLagCandCap];
};

// One lag search: FFT cross-correlation of the upper envelopes of a and b
// (reference src/accel.zig:100-107), or of a and b themselves (raw).
struct LagJob {
    VSig a, b;
    int64_t n;           // FFT size, fftSizeFor(max(a.len, b.len))
    int64_t biggest;     // max(a.len, b.len)
    // serial statistics of a and b, 4 doubles each: [sum, nyquist, energy, -]
    double *stats_a, *stats_b;
    double2 *z;          // n complex values
    int64_t *lag_out;
    // f32-nominated search: f32 transform, f64 rescoring of the near-maxima
    float2 *z32;         // n complex values
    double2 *energy;     // per forward CTA: sums of squares of a's and b's envelopes
    LagCands *cands;     // per inverse CTA
    int32_t *status;     // 0: lag decided; 1: over kLagCandCap candidates or a near-tie, the f64 search decides
    int32_t *ncand;      // candidates above the job's floor
    int32_t *cand_key;   // kLagCandCap of them
    double *rescore;     // kLagCandCap x chunks partial dot products
    float *corr_out;     // test only (else null): Re of the f32 correlation, n values
    double slack_fixed;  // test only (else 0): the nomination slack, instead of the f32 error bound
};

// One spectrogram's reverse (k_grad.cu): d loss / d RMS cells g_rms[b * nf +
// f] of the frames of `sig` to d loss / d samples, added to grad[k - head]
// for the stored samples (grad indexed as sig.base).
struct GradSpecJob {
    VSig sig;
    int64_t nf;
    const double *g_rms;
    double *grad;
};

// Serial reductions over a signal, in the CPU's order, into
// out[0] = sum x, out[1] = sum (-1)^k (x - mean), out[2] = sum x*x.
struct SumJob {
    VSig sig;
    double *out;
};

// One spectrogram pair to prepare for comparison (reference
// src/spectrogram.zig:69-80): in-place on ref[nb*nfr], deg[nb*nfd].
struct PrepJob {
    const double *ref_in, *deg_in;
    double *ref, *deg;
    int32_t nfr, nfd;
};

// Per-band NSIM statistics of a patch pair (reference src/nsim.zig:427-510).
// ref column c = ref[b*ref_stride + ref_col + c]; deg column c =
// deg[b*deg_stride + deg_col + c] when deg_col + c < deg_cols, else 0.
// With dp_offset set, deg_col comes from it and dp_valid zeroes invalid
// matches (reference src/dp.zig:333-341).
struct StatsJob {
    const double *ref;
    int32_t ref_stride, ref_col;
    const double *deg;
    int32_t deg_stride, deg_col, deg_cols;
    int32_t ncols;
    const int64_t *dp_offset;
    const uint8_t *dp_valid;
    double *means, *stddevs, *energy;  // nb each
    double *similarity;
};

// Batched copy of grid-aligned spectrogram frames (reference
// src/realign.zig:262-281).
struct CopyJob {
    const double *src;
    int32_t src_stride, src_col;
    double *dst;
    int32_t ncols;
};

constexpr double kC1 = (0.01 * 1.0) * (0.01 * 1.0);
constexpr double kC3 = (0.03 * 1.0) * (0.03 * 1.0) / 2.0;

// NSIM 3x3 Gaussian window (reference src/nsim.zig:111-115), symmetric.
constexpr double kW0 = 0.0113033910173052;  // corners
constexpr double kW1 = 0.0838251475442633;  // edges
constexpr double kW2 = 0.619485845753726;   // centre

// Taps.at's fixed summation order (reference src/nsim.zig:145-155):
// rows (rm, r0, rp) x columns (cm, c, cp), flipped taps of the symmetric
// window, summed left to right.
__host__ __device__ inline double taps9(double a00, double a01, double a02, double a10, double a11, double a12,
                                        double a20, double a21, double a22) {
    return kW0 * a00 + kW1 * a01 + kW0 * a02 + kW1 * a10 + kW2 * a11 + kW1 * a12 + kW0 * a20 + kW1 * a21 +
           kW0 * a22;
}

#ifdef __CUDACC__
// simCell (reference src/nsim.zig:293-308).
__device__ inline double sim_cell(double mr, double rms, double srs, double md, double dms, double sds, double crd) {
    const double mrd = mr * md;
    const double srd = crd - mrd;
    const double intensity = (2.0 * mrd + kC1) / (rms + dms + kC1);
    const double prod = srs * sds;
    const double denom = prod < 0.0 ? kC3 : sqrt(prod) + kC3;
    const double structure = (srd + kC3) / denom;
    return intensity * structure;
}
#endif

}  // namespace vqb
