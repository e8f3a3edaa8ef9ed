// Gammatone filterbank spectrograms of the two fast forms. Both compute the
// same cascade of four biquads per (frame, band) as the exact kernel
// (reference src/gammatone.zig:268-306) without its operation order.
//
// f64 FMA form (gammatone_f64fma_kernel): each biquad in direct form I with
// its numerator normalised to 1 + beta z^-1 (the four numerator gains and
// the band gain become one f64 factor on the RMS), so a stage is three FMAs:
// y = v + beta v[-1] - d2 y[-2] - d1 y[-1]. 13 FMAs and one multiply per
// sample instead of the exact form's 31 separately rounded operations; the
// results stay within ~1e-13 of the exact form in MOS. Thread and warp
// layout as the exact kernel (a warp reads one sample per step, broadcast).
//
// f32 form (gammatone_fast_kernel) splits the cascade across the two
// arithmetic pipes of an SM:
//
// * stage 1 runs in f64 with FMA on the FP64 pipe. It sees the raw windowed
//   signal, whose out-of-band content is far larger than the band's output;
//   f32 state there would carry rounding of that content into the result.
// * stages 2-4 run in f32 on the FP32 pipe, two frames per thread as packed
//   f32x2 FMAs. Their numerators are normalised to 1 + beta z^-1 with the
//   gains (a0^3) applied to the final RMS in f64, and their pole
//   coefficients are carried as hi + lo f32 pairs: rounding the poles to a
//   single f32 shifts the upper bands' responses enough to move MOS by
//   ~6e-7. Bands whose centre frequencies are low (poles near z = 1) use the
//   direct form I recurrence, the rest the transposed direct form II; each
//   kept the smaller error in a sweep over both.
// * the squared outputs are summed in f32 over runs of 16 samples and the
//   runs are added in f64.
//
// A warp holds 8 bands x 4 frame pairs: lanes of a frame pair load the same
// sample (4 distinct addresses per load), the Hann value is warp-uniform,
// and every band of a warp takes the same form (the host groups bands by 8).
// A CTA holds ceil(nb/8) band groups x 2 frame blocks of 8 frames.
#include "device.cuh"
#include "kernels.h"

namespace vqb {

namespace {

struct Tile {
    int32_t job;
    int32_t frame0;
};

constexpr int kFramesPerBlock = 8;   // frames per warp (4 lanes rows x 2)
constexpr int kBlocksPerCta = 2;
constexpr int kRun = 16;             // f32 partial-sum run length

__device__ inline float2 f2(float v) { return make_float2(v, v); }

struct F32Stage {
    float2 a, b, c;  // DF2T: c0, c1 (c unused); DF-I: y1, y2, previous input
};

template <bool kDirectI>
__device__ inline float2 stage32(float2 v, F32Stage &s, float2 beta, float2 np1h, float2 np1l, float2 np2h,
                                 float2 np2l) {
    if (kDirectI) {
        // y = v + beta v[-1] - d1 y[-1] - d2 y[-2], small terms first
        float2 t = __ffma2_rn(beta, s.c, v);
        t = __ffma2_rn(np1l, s.a, t);
        t = __ffma2_rn(np2l, s.b, t);
        t = __ffma2_rn(np2h, s.b, t);
        const float2 y = __ffma2_rn(np1h, s.a, t);
        s.c = v;
        s.b = s.a;
        s.a = y;
        return y;
    }
    // y = v + c0; c0 = beta v + c1 - d1 y; c1 = -d2 y
    const float2 y = __fadd2_rn(v, s.a);
    float2 t = __ffma2_rn(beta, v, s.b);
    t = __ffma2_rn(np1h, y, t);
    s.a = __ffma2_rn(np1l, y, t);
    s.b = __ffma2_rn(np2h, y, __fmul2_rn(np2l, y));
    return y;
}

// Samples of a frame: straight loads when the whole window lies inside the
// signal's stored samples (nearly every frame), else VSig's bounds-checked
// view (zero padding at slice edges).
struct Direct {
    const double *p;
    __device__ double operator()(int64_t k) const { return p[k]; }
};
struct Checked {
    VSig s;
    __device__ double operator()(int64_t k) const { return vsig_at(s, k); }
};

__device__ inline bool window_inside(const VSig &sig, int64_t k0, int64_t span) {
    return k0 - sig.head >= 0 && k0 + span - sig.head <= sig.avail;
}

template <bool kDirectI, class Load>
__device__ void band_frames(const Load &sample, int64_t ka, int64_t kb, const FastBandCoeffs &k,
                            const double *__restrict__ hann, int window, double &acc_a, double &acc_b) {
    double c0a = 0.0, c1a = 0.0, c0b = 0.0, c1b = 0.0;
    F32Stage st[3];
#pragma unroll
    for (int s = 0; s < 3; ++s) st[s] = F32Stage{f2(0.f), f2(0.f), f2(0.f)};
    const float2 b0 = f2(k.beta[0]), b1 = f2(k.beta[1]), b2 = f2(k.beta[2]);
    const float2 np1h = f2(-k.p1h), np1l = f2(-k.p1l), np2h = f2(-k.p2h), np2l = f2(-k.p2l);
    const double n0 = k.n0, n1 = k.n1, nd1 = -k.d1, nd2 = -k.d2;
    acc_a = 0.0;
    acc_b = 0.0;
    auto step = [&](int i, float2 &part) {
        const double h = __ldg(hann + i);
        const double xa = sample(ka + i) * h;
        const double xb = sample(kb + i) * h;
        const double fa = __fma_rn(n0, xa, c0a);
        const double fb = __fma_rn(n0, xb, c0b);
        c0a = __fma_rn(nd1, fa, __fma_rn(n1, xa, c1a));
        c0b = __fma_rn(nd1, fb, __fma_rn(n1, xb, c1b));
        c1a = nd2 * fa;
        c1b = nd2 * fb;
        float2 v = make_float2(__double2float_rn(fa), __double2float_rn(fb));
        v = stage32<kDirectI>(v, st[0], b0, np1h, np1l, np2h, np2l);
        v = stage32<kDirectI>(v, st[1], b1, np1h, np1l, np2h, np2l);
        v = stage32<kDirectI>(v, st[2], b2, np1h, np1l, np2h, np2l);
        part = __ffma2_rn(v, v, part);
    };
    const int runs = window / kRun;
    for (int r = 0; r < runs; ++r) {
        float2 part = f2(0.f);
#pragma unroll
        for (int j = 0; j < kRun; ++j) step(r * kRun + j, part);
        acc_a += (double)part.x;
        acc_b += (double)part.y;
    }
    float2 part = f2(0.f);
    for (int i = runs * kRun; i < window; ++i) step(i, part);
    acc_a += (double)part.x;
    acc_b += (double)part.y;
}

__global__ void __launch_bounds__(256) gammatone_fast_kernel(const SpecJob *__restrict__ jobs,
                                                             const Tile *__restrict__ tiles,
                                                             const FastBandCoeffs *__restrict__ coeffs, int nb,
                                                             const double *__restrict__ hann, int window, int hop) {
    const Tile tile = tiles[blockIdx.x];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int groups = (nb + 7) >> 3;
    const int g = warp % groups, fblock = warp / groups;
    const int band = g * 8 + (lane & 7);
    const SpecJob job = jobs[tile.job];
    const int64_t f = (int64_t)tile.frame0 + fblock * kFramesPerBlock + 2 * (lane >> 3);
    if (band >= nb || f >= job.nf) return;
    const FastBandCoeffs k = coeffs[band];
    const int64_t ka = f * hop, kb = ka + hop;
    double acc_a, acc_b;
    const VSig &sig = job.sig;
    if (window_inside(sig, ka, hop + window)) {
        const Direct ld{sig.base - sig.head};
        if (k.direct_i)
            band_frames<true>(ld, ka, kb, k, hann, window, acc_a, acc_b);
        else
            band_frames<false>(ld, ka, kb, k, hann, window, acc_a, acc_b);
    } else {
        const Checked ld{sig};
        if (k.direct_i)
            band_frames<true>(ld, ka, kb, k, hann, window, acc_a, acc_b);
        else
            band_frames<false>(ld, ka, kb, k, hann, window, acc_a, acc_b);
    }
    const double inv_n = 1.0 / (double)window;
    double *out = job.out + (int64_t)band * job.nf;
    out[f] = sqrt(acc_a * inv_n) * k.post;
    if (f + 1 < job.nf) out[f + 1] = sqrt(acc_b * inv_n) * k.post;
}

// Two frames per thread (the second hop samples later): two independent
// recurrences give each warp twice the FP64 work between dependent steps.
struct Cascade64 {
    double xp = 0.0, y1a = 0.0, y2a = 0.0, y1b = 0.0, y2b = 0.0, y1c = 0.0, y2c = 0.0, y1d = 0.0, y2d = 0.0;
    double acc = 0.0;
    __device__ inline void step(double x, double b0, double b1, double b2, double b3, double nd1, double nd2) {
        // stage k input v, previous input = stage k-1's previous output
        const double ya = __fma_rn(nd1, y1a, __fma_rn(nd2, y2a, __fma_rn(b0, xp, x)));
        const double yb = __fma_rn(nd1, y1b, __fma_rn(nd2, y2b, __fma_rn(b1, y1a, ya)));
        const double yc = __fma_rn(nd1, y1c, __fma_rn(nd2, y2c, __fma_rn(b2, y1b, yb)));
        const double yd = __fma_rn(nd1, y1d, __fma_rn(nd2, y2d, __fma_rn(b3, y1c, yc)));
        xp = x;
        y2a = y1a;
        y1a = ya;
        y2b = y1b;
        y1b = yb;
        y2c = y1c;
        y1c = yc;
        y2d = y1d;
        y1d = yd;
        acc = __fma_rn(yd, yd, acc);
    }
};

template <class Load>
__device__ void cascade64x2(const Load &sample, int64_t ka, int64_t kb, const FastBandCoeffs &kc,
                            const double *__restrict__ hann, int window, bool warp_frame, double &acc_a,
                            double &acc_b) {
    const double b0 = kc.beta64[0], b1 = kc.beta64[1], b2 = kc.beta64[2], b3 = kc.beta64[3];
    const double nd1 = -kc.d1, nd2 = -kc.d2;
    Cascade64 A, B;
    if (warp_frame) {
        // a warp holds two frames' 32 bands: lane j forms windowed samples
        // i0 + j of both frames, shuffled to the warp
        const int lane = threadIdx.x & 31;
        int i0 = 0;
        for (; i0 + 32 <= window; i0 += 32) {
            const double h = __ldg(hann + i0 + lane);
            const double xa = sample(ka + i0 + lane) * h, xb = sample(kb + i0 + lane) * h;
#pragma unroll 8
            for (int j = 0; j < 32; ++j) {
                A.step(__shfl_sync(0xffffffffu, xa, j), b0, b1, b2, b3, nd1, nd2);
                B.step(__shfl_sync(0xffffffffu, xb, j), b0, b1, b2, b3, nd1, nd2);
            }
        }
        const int rest = window - i0;
        const double h = lane < rest ? __ldg(hann + i0 + lane) : 0.0;
        const double xa = lane < rest ? sample(ka + i0 + lane) * h : 0.0;
        const double xb = lane < rest ? sample(kb + i0 + lane) * h : 0.0;
        for (int j = 0; j < rest; ++j) {
            A.step(__shfl_sync(0xffffffffu, xa, j), b0, b1, b2, b3, nd1, nd2);
            B.step(__shfl_sync(0xffffffffu, xb, j), b0, b1, b2, b3, nd1, nd2);
        }
    } else {
#pragma unroll 2
        for (int i = 0; i < window; ++i) {
            const double h = __ldg(hann + i);
            A.step(sample(ka + i) * h, b0, b1, b2, b3, nd1, nd2);
            B.step(sample(kb + i) * h, b0, b1, b2, b3, nd1, nd2);
        }
    }
    acc_a = A.acc;
    acc_b = B.acc;
}

// CTA: F frames x nb bands, two frames per thread (threads = F/2 x nb).
// Thread t: band t % nb, frames frame0 + 2 (t / nb) and the next.
__global__ void __launch_bounds__(256, 2) gammatone_f64fma_kernel(const SpecJob *__restrict__ jobs,
                                                               const Tile *__restrict__ tiles,
                                                               const FastBandCoeffs *__restrict__ coeffs, int nb,
                                                               const double *__restrict__ hann, int window, int hop) {
    const Tile tile = tiles[blockIdx.x];
    const int pair = threadIdx.x / nb;
    const int band = threadIdx.x - pair * nb;
    const SpecJob job = jobs[tile.job];
    const int64_t f = (int64_t)tile.frame0 + 2 * pair;
    if (f >= job.nf) return;
    const FastBandCoeffs &kc = coeffs[band];
    const int64_t ka = f * hop, kb = ka + hop;
    const VSig sig = job.sig;
    double acc_a, acc_b;
    // With 32 bands a warp is one frame pair, and window_inside (over both
    // frames) is the same for all its lanes, so the shuffles see the whole
    // warp.
    const bool warp_frame = nb == 32;
    if (window_inside(sig, ka, hop + window))
        cascade64x2(Direct{sig.base - sig.head}, ka, kb, kc, hann, window, warp_frame, acc_a, acc_b);
    else
        cascade64x2(Checked{sig}, ka, kb, kc, hann, window, warp_frame, acc_a, acc_b);
    const double inv_n = 1.0 / (double)window;
    double *out = job.out + (int64_t)band * job.nf;
    out[f] = sqrt(acc_a * inv_n) * kc.post64;
    if (f + 1 < job.nf) out[f + 1] = sqrt(acc_b * inv_n) * kc.post64;
}

}  // namespace

int gammatone_fast_frames_per_cta() { return kFramesPerBlock * kBlocksPerCta; }

void fill_fast_band_coeffs(const BandCoeffs *run, const double *cf, int nb, FastBandCoeffs *out) {
    // Direct form I for band groups whose highest centre frequency is below
    // 3 kHz (the exact split is not critical: both forms stay far inside
    // the fast form's tolerance near the boundary).
    for (int g = 0; g * 8 < nb; ++g) {
        const int hi = g * 8 + 7 < nb ? g * 8 + 7 : nb - 1;
        const int32_t direct_i = cf[hi] < 3000.0 ? 1 : 0;
        for (int b = g * 8; b <= hi; ++b) {
            const BandCoeffs &c = run[b];
            FastBandCoeffs &k = out[b];
            k.n0 = c.s1n0;
            k.n1 = c.s1n1;
            k.d1 = c.d1;
            k.d2 = c.d2;
            const double a0 = c.ca0;
            k.post = fabs(a0 * a0 * a0);
            k.beta[0] = (float)(c.s2n1 / a0);
            k.beta[1] = (float)(c.s3n1 / a0);
            k.beta[2] = (float)(c.s4n1 / a0);
            k.p1h = (float)c.d1;
            k.p1l = (float)(c.d1 - (double)k.p1h);
            k.p2h = (float)c.d2;
            k.p2l = (float)(c.d2 - (double)k.p2h);
            k.direct_i = direct_i;
            k.beta64[0] = c.s1n1 / c.s1n0;
            k.beta64[1] = c.s2n1 / a0;
            k.beta64[2] = c.s3n1 / a0;
            k.beta64[3] = c.s4n1 / a0;
            k.post64 = fabs(c.s1n0 * a0 * a0 * a0);
        }
    }
}

void launch_gammatone_fast(const SpecJob *d_jobs, const void *d_tiles, int ntiles, const FastBandCoeffs *d_coeffs,
                           int nb, const double *d_hann, int window, int hop, cudaStream_t s) {
    if (ntiles <= 0) return;
    const int threads = ((nb + 7) / 8) * kBlocksPerCta * 32;
    gammatone_fast_kernel<<<ntiles, threads, 0, s>>>(d_jobs, static_cast<const Tile *>(d_tiles), d_coeffs, nb,
                                                    d_hann, window, hop);
    launch_counter() += 1;
}

}  // namespace vqb

namespace vqb {

std::vector<int> gammatone_f64fma_frames_candidates(int nb) {
    const int f = 2 * (256 / nb);  // two frames per thread, 256 threads
    return {f, f / 2, f / 4};
}

void launch_gammatone_f64fma(const SpecJob *d_jobs, const void *d_tiles, int ntiles, const FastBandCoeffs *d_coeffs,
                             int nb, const double *d_hann, int window, int hop, int frames_per_cta, cudaStream_t s) {
    if (ntiles <= 0) return;
    const int threads = (frames_per_cta / 2) * nb;
    gammatone_f64fma_kernel<<<ntiles, threads, 0, s>>>(d_jobs, static_cast<const Tile *>(d_tiles), d_coeffs, nb,
                                                      d_hann, window, hop);
    launch_counter() += 1;
}

}  // namespace vqb
