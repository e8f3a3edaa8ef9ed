// Gammatone filterbank spectrograms of the two fast forms. Both compute the
// same cascade of four biquads per (frame, band) as the exact kernel
// (reference src/gammatone.zig:268-306) without its operation order.
//
// f64 FMA form (gammatone_f64fma_kernel): each biquad in direct form I with
// its numerator normalised to 1 + beta z^-1 (the four numerator gains and
// the band gain become one f64 factor on the RMS), so a stage is three FMAs:
// y = v + beta v[-1] - d2 y[-2] - d1 y[-1]. 13 FMAs and one multiply per
// sample instead of the exact form's 31 separately rounded operations; the
// results stay within ~1e-13 of the exact form in MOS. Two kernels compute
// it with the same bits: by default the f32 form's kernel below with all
// four stages in f64 (its staged shared-memory tiles, one 16-byte load per
// step for a thread's two frames), and gammatone_f64fma_kernel, whose
// thread and warp layout is the exact kernel's (a lane forms one windowed
// sample and the warp reads it by shuffle); the autotuner measures both.
//
// f32 form (gammatone_fast_kernel) splits the cascade across the two
// arithmetic pipes of an SM:
//
// * stages 1 and 2 run in f64 with FMA on the FP64 pipe, direct form I with
//   unit-leading numerators (3 FMAs a stage). Stage 1 sees the raw windowed
//   signal, whose out-of-band content is far larger than the band's output;
//   f32 state there would carry rounding of that content into the result.
// * stages 3 and 4 run in f32 on the FP32 pipe, two frames per thread as
//   packed f32x2 FMAs. Their pole coefficients are carried as hi + lo f32
//   pairs: rounding the poles to a single f32 shifts the upper bands'
//   responses enough to move MOS by ~6e-7. Bands whose centre frequencies
//   are low (poles near z = 1) use the direct form I recurrence, the rest
//   the transposed direct form II; each kept the smaller error in a sweep
//   over both. All numerator gains go into one f64 factor on the RMS.
// * the squared outputs are summed in f32 over runs of 16 samples and the
//   runs are added in f64.
// * the lowest band group (8 bands) runs all four stages in f64, as the
//   FP64-FMA form does: its poles sit nearest the unit circle, where f32
//   state noise grows most, and the spectrogram preparation (per-frame
//   floors, joint minimum) carries that error into every band. This is the
//   compensated state such bands need; on this part an f64 stage (3 FMAs on
//   the half-rate FP64 pipe) costs less than a double-single one (~20 f32
//   operations).
//
// Per frame-sample that is 6 FP64 FMAs (16 lanes per SM sub-partition) and
// 11-13 FP32 FMAs (32 lanes), which keeps both pipes about equally busy.
// The CTA's 16 frames are Hann-windowed once per 64-sample tile into shared
// memory (double-buffered; the next tile's samples are loaded into registers
// while the current one is filtered), so a thread reads its two frames'
// windowed samples with one 16-byte load per step.
//
// A warp holds 8 bands x 4 frame pairs: lanes of a frame pair read the same
// shared-memory word (a broadcast), and every band of a warp takes the same
// form (the host groups bands by 8). A CTA holds ceil(nb/8) band groups x 2
// frame blocks of 8 frames.
#include <algorithm>

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
constexpr int kCtaFrames = kFramesPerBlock * kBlocksPerCta;
constexpr int kRun = 16;             // f32 partial-sum run length
constexpr int kTileS = 64;           // samples per shared-memory tile
constexpr int kRowPad = kCtaFrames + 2;  // doubles per tile row (2-way write conflicts, 16-byte reads)

__device__ inline float2 f2(float v) { return make_float2(v, v); }

// 8-byte asynchronous global-to-shared copy; bytes = 0 writes zeros.
__device__ inline void cp_async8(double *dst, const double *src, int bytes) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(src), "r"(bytes) : "memory");
}
__device__ inline void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ inline void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

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

// Stages 1 and 2 of one frame in f64, direct form I with unit-leading
// numerators: y = x + b0 x[-1] - d2 y[-2] - d1 y[-1], then the same on y.
struct F64Pair {
    double x1 = 0.0, y1 = 0.0, y2 = 0.0, z1 = 0.0, z2 = 0.0;
    __device__ inline double step(double x, double b0, double b1, double nd1, double nd2) {
        const double y = __fma_rn(nd1, y1, __fma_rn(nd2, y2, __fma_rn(b0, x1, x)));
        const double z = __fma_rn(nd1, z1, __fma_rn(nd2, z2, __fma_rn(b1, y1, y)));
        x1 = x;
        y2 = y1;
        y1 = y;
        z2 = z1;
        z1 = z;
        return z;
    }
};

// The FP64-FMA form's four stages of one frame, direct form I with
// unit-leading numerators, and its sum of squares. Both kernels of that form
// run two frames per thread (the second hop samples later): two independent
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

template <bool kDirectI>
__device__ inline void filter_tile(const double (*__restrict__ wx)[kRowPad], int q, int count,
                                   const FastBandCoeffs &k, F64Pair &A, F64Pair &B, F32Stage (&st)[2],
                                   double &acc_a, double &acc_b) {
    const double b0 = k.beta64[0], b1 = k.beta64[1], nd1 = -k.d1, nd2 = -k.d2;
    const float2 c3 = f2(k.beta[0]), c4 = f2(k.beta[1]);
    const float2 np1h = f2(-k.p1h), np1l = f2(-k.p1l), np2h = f2(-k.p2h), np2l = f2(-k.p2l);
    auto step = [&](int i, float2 &part) {
        const double2 w = *reinterpret_cast<const double2 *>(&wx[i][q]);
        const double za = A.step(w.x, b0, b1, nd1, nd2);
        const double zb = B.step(w.y, b0, b1, nd1, nd2);
        float2 v = make_float2(__double2float_rn(za), __double2float_rn(zb));
        v = stage32<kDirectI>(v, st[0], c3, np1h, np1l, np2h, np2l);
        v = stage32<kDirectI>(v, st[1], c4, np1h, np1l, np2h, np2l);
        part = __ffma2_rn(v, v, part);
    };
    if (count == kTileS) {
#pragma unroll 1
        for (int r = 0; r < kTileS / kRun; ++r) {
            float2 part = f2(0.f);
#pragma unroll 4
            for (int j = 0; j < kRun; ++j) step(r * kRun + j, part);
            acc_a += (double)part.x;
            acc_b += (double)part.y;
        }
    } else {
        float2 part = f2(0.f);
        for (int i = 0; i < count; ++i) step(i, part);
        acc_a += (double)part.x;
        acc_b += (double)part.y;
    }
}

// The same tile position filtered by the FP64-FMA form: all four stages in
// f64, the squares summed in f64 per sample. The windowed samples are the
// products the unstaged kernel forms (sample x Hann value, zero outside the
// signal), so both kernels give the same bits.
__device__ inline void filter_tile64(const double (*__restrict__ wx)[kRowPad], int q, int count,
                                     const FastBandCoeffs &k, Cascade64 &A, Cascade64 &B) {
    const double b0 = k.beta64[0], b1 = k.beta64[1], b2 = k.beta64[2], b3 = k.beta64[3];
    const double nd1 = -k.d1, nd2 = -k.d2;
    auto step = [&](int i) {
        const double2 w = *reinterpret_cast<const double2 *>(&wx[i][q]);
        A.step(w.x, b0, b1, b2, b3, nd1, nd2);
        B.step(w.y, b0, b1, b2, b3, nd1, nd2);
    };
    if (count == kTileS) {
#pragma unroll 4
        for (int i = 0; i < kTileS; ++i) step(i);
    } else {
        for (int i = 0; i < count; ++i) step(i);
    }
}

// One tile (16 frames x all bands of one job) of the FP32 form (kF64: of the FP64-FMA form). raw, wx:
// the CTA's shared-memory staging (raw[2][16][kTileS] signal samples,
// frame-major; wx[2][kTileS][kRowPad] windowed samples, sample-major).
template <int kThreads, bool kF64>
__device__ __forceinline__ void fast_tile(const Tile tile, const SpecJob *__restrict__ jobs,
                                          const FastBandCoeffs *__restrict__ coeffs, int nb,
                                          const double *__restrict__ hann, int window, int hop,
                                          double (*raw)[kCtaFrames][kTileS], double (*wx)[kTileS][kRowPad]) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int groups = (nb + 7) >> 3;
    const int g = warp % groups, fblock = warp / groups;
    const int band_raw = g * 8 + (lane & 7);
    const int band = band_raw < nb ? band_raw : nb - 1;  // idle lanes filter a real band, never write
    const int q = fblock * kFramesPerBlock + 2 * (lane >> 3);
    const SpecJob job = jobs[tile.job];
    const VSig sig = job.sig;
    const int64_t f = (int64_t)tile.frame0 + q;
    const FastBandCoeffs k = coeffs[band];

    // Tiles of kTileS samples of the CTA's frames: entry e = (frame c =
    // e / kTileS, sample i = e % kTileS), so consecutive threads copy
    // consecutive samples of a frame. Samples outside the signal's stored
    // range or past the window are zero-filled by the copy itself.
    constexpr int kFills = (kCtaFrames * kTileS + kThreads - 1) / kThreads;
    auto fetch = [&](int i0, int buf) {
#pragma unroll
        for (int m = 0; m < kFills; ++m) {
            const int e = threadIdx.x + m * kThreads;
            if (e < kCtaFrames * kTileS) {
                const int c = e / kTileS, i = e - c * kTileS;
                const int64_t j = ((int64_t)tile.frame0 + c) * hop + i0 + i - sig.head;
                const bool in = i0 + i < window && (uint64_t)j < (uint64_t)sig.avail;
                cp_async8(&raw[buf][c][i], in ? sig.base + j : sig.base, in ? 8 : 0);
            }
        }
        cp_async_commit();
    };
    auto windowed = [&](int i0, int buf) {
#pragma unroll
        for (int m = 0; m < kFills; ++m) {
            const int e = threadIdx.x + m * kThreads;
            if (e < kCtaFrames * kTileS) {
                const int c = e / kTileS, i = e - c * kTileS;
                wx[buf][i][c] = i0 + i < window ? raw[buf][c][i] * __ldg(hann + i0 + i) : 0.0;
            }
        }
    };
    fetch(0, 0);
    cp_async_wait_all();
    __syncthreads();
    windowed(0, 0);
    if (kTileS < window) fetch(kTileS, 1);

    F64Pair A, B;
    F32Stage st[2];
#pragma unroll
    for (int s = 0; s < 2; ++s) st[s] = F32Stage{f2(0.f), f2(0.f), f2(0.f)};
    Cascade64 CA, CB;  // kF64
    double acc_a = 0.0, acc_b = 0.0;
    // One CTA barrier a tile. At tile t: tile t+1's copies (issued a tile
    // earlier) are waited for; behind the barrier every thread is done
    // filtering tile t-1 (whose windowed buffer tile t+1 takes) and done
    // windowing tile t (whose copy buffer tile t+2 takes); then tile t+1 is
    // windowed, tile t+2's copies are issued, and tile t is filtered.
    int buf = 0;
    for (int i0 = 0; i0 < window; i0 += kTileS) {
        const int next = i0 + kTileS;
        if (next < window) cp_async_wait_all();
        __syncthreads();
        if (next < window) windowed(next, buf ^ 1);
        if (next + kTileS < window) fetch(next + kTileS, buf);
        const int count = window - i0 < kTileS ? window - i0 : kTileS;
        if (kF64 || k.arith == kArithF64)
            filter_tile64(wx[buf], q, count, k, CA, CB);
        else if (k.arith == kArithF32Df1)
            filter_tile<true>(wx[buf], q, count, k, A, B, st, acc_a, acc_b);
        else
            filter_tile<false>(wx[buf], q, count, k, A, B, st, acc_a, acc_b);
        buf ^= 1;
    }
    if (kF64 || k.arith == kArithF64) {
        acc_a = CA.acc;
        acc_b = CB.acc;
    }
    if (band_raw < nb && f < job.nf) {
        const double inv_n = 1.0 / (double)window;
        double *out = job.out + (int64_t)band * job.nf;
        out[f] = sqrt(acc_a * inv_n) * k.post64;
        if (f + 1 < job.nf) out[f + 1] = sqrt(acc_b * inv_n) * k.post64;
    }
}

// kThreads = 64 x ceil(nb / 8): 256 for 32 bands, 192 for 21. kCtasPerSm
// sets the register budget: 2 (128 registers at 256 threads), which the f32
// form needs since its lowest band group's warps hold the all-f64 cascade
// (budgets of 3 or 4 CTAs spill over 1 KB a thread). kPersistent: a grid of
// kCtasPerSm CTAs per SM takes tiles from a device-side work queue (an
// atomic counter over the tile list, zero at launch) instead of one CTA per
// tile; every tile is computed the same either way. kF64: the FP64-FMA form
// on the same staged tiles.
template <int kThreads, int kCtasPerSm, bool kPersistent, bool kF64 = false>
__global__ void __launch_bounds__(kThreads, kCtasPerSm * 256 / kThreads) gammatone_fast_kernel(
    const SpecJob *__restrict__ jobs, const Tile *__restrict__ tiles, int ntiles, int *__restrict__ queue,
    const FastBandCoeffs *__restrict__ coeffs, int nb, const double *__restrict__ hann, int window, int hop) {
    __shared__ __align__(16) double raw[2][kCtaFrames][kTileS];
    __shared__ __align__(16) double wx[2][kTileS][kRowPad];
    if constexpr (!kPersistent) {
        fast_tile<kThreads, kF64>(tiles[blockIdx.x], jobs, coeffs, nb, hann, window, hop, raw, wx);
    } else {
        __shared__ int next;
        for (;;) {
            if (threadIdx.x == 0) next = atomicAdd(queue, 1);
            __syncthreads();
            const int ti = next;
            if (ti >= ntiles) return;  // the same for the whole CTA
            fast_tile<kThreads, kF64>(tiles[ti], jobs, coeffs, nb, hann, window, hop, raw, wx);
            __syncthreads();  // staging buffers and `next` free for the next tile
        }
    }
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
    // The lowest band group runs all four stages in f64: its poles sit
    // nearest the unit circle (1 - r = 0.004 .. 0.011 at 48 kHz), where f32
    // state noise is amplified most, and through the per-frame floors and
    // the joint minimum of the spectrogram preparation that error reaches
    // every band (with f32 stages there, MOS moved by up to 4e-6 on
    // low-SNR 48 kHz pairs; with f64 there, by at most 4e-7). Above it,
    // direct form I for band groups whose highest centre frequency is below
    // 3 kHz, else the transposed form (the exact split is not critical:
    // both forms stay far inside the fast form's tolerance near the
    // boundary).
    for (int g = 0; g * 8 < nb; ++g) {
        const int hi = g * 8 + 7 < nb ? g * 8 + 7 : nb - 1;
        const int32_t arith = g == 0 ? kArithF64 : cf[hi] < 3000.0 ? kArithF32Df1 : kArithF32Df2t;
        for (int b = g * 8; b <= hi; ++b) {
            const BandCoeffs &c = run[b];
            FastBandCoeffs &k = out[b];
            const double a0 = c.ca0;
            k.d1 = c.d1;
            k.d2 = c.d2;
            k.beta64[0] = c.s1n1 / c.s1n0;
            k.beta64[1] = c.s2n1 / a0;
            k.beta64[2] = c.s3n1 / a0;
            k.beta64[3] = c.s4n1 / a0;
            k.post64 = fabs(c.s1n0 * a0 * a0 * a0);
            k.beta[0] = (float)k.beta64[2];
            k.beta[1] = (float)k.beta64[3];
            k.p1h = (float)c.d1;
            k.p1l = (float)(c.d1 - (double)k.p1h);
            k.p2h = (float)c.d2;
            k.p2l = (float)(c.d2 - (double)k.p2h);
            k.arith = arith;
        }
    }
}

// Launch shapes: CTAs per SM (register budget) + 100 for the persistent
// work-queue form. The persistent shape measured ~4.5% slower inside the
// four-lane batch pipeline (its resident CTAs hold SMs the other lanes'
// kernels would take), so it is selected only by VISQOL_TUNE_3.
std::vector<int> gammatone_fast_shape_candidates() { return {2}; }
std::vector<int> gammatone_fast_shapes() { return {2, 102}; }

namespace {
int sm_count() {
    int dev = 0, n = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    return n > 0 ? n : 1;
}
}  // namespace

void launch_gammatone_fast(const SpecJob *d_jobs, const void *d_tiles, int ntiles, const FastBandCoeffs *d_coeffs,
                           int nb, const double *d_hann, int window, int hop, int shape, int *d_queue,
                           cudaStream_t s) {
    if (ntiles <= 0) return;
    const Tile *t = static_cast<const Tile *>(d_tiles);
    const int ctas = shape % 100;
    const bool persistent = shape >= 100 && d_queue;
    const int grid = persistent ? std::min(ntiles, sm_count() * ctas) : ntiles;
#define VQB_FAST(T, C, P)                                                                                    \
    gammatone_fast_kernel<T, C, P><<<grid, T, 0, s>>>(d_jobs, t, ntiles, d_queue, d_coeffs, nb, d_hann, window, \
                                                      hop)
#define VQB_FAST_T(T)         \
    if (persistent)           \
        VQB_FAST(T, 2, true); \
    else                      \
        VQB_FAST(T, 2, false);
    if (nb > 24) {
        VQB_FAST_T(256)
    } else if (nb > 16) {
        VQB_FAST_T(192)
    } else if (nb > 8) {
        VQB_FAST_T(128)
    } else {
        VQB_FAST_T(64)
    }
#undef VQB_FAST_T
#undef VQB_FAST
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

// The staged kernel first: it measured 0.82 of the FP64 FMA pipe's peak in
// isolation at 32 bands against 0.75 for the unstaged one.
std::vector<int> gammatone_f64_staged_candidates() { return {1, 0}; }

void launch_gammatone_f64_staged(const SpecJob *d_jobs, const void *d_tiles, int ntiles,
                                 const FastBandCoeffs *d_coeffs, int nb, const double *d_hann, int window, int hop,
                                 cudaStream_t s) {
    if (ntiles <= 0) return;
    const Tile *t = static_cast<const Tile *>(d_tiles);
#define VQB_F64S(T) \
    gammatone_fast_kernel<T, 2, false, true><<<ntiles, T, 0, s>>>(d_jobs, t, ntiles, nullptr, d_coeffs, nb, d_hann, \
                                                                  window, hop)
    if (nb > 24)
        VQB_F64S(256);
    else if (nb > 16)
        VQB_F64S(192);
    else if (nb > 8)
        VQB_F64S(128);
    else
        VQB_F64S(64);
#undef VQB_F64S
    launch_counter() += 1;
}

}  // namespace vqb
