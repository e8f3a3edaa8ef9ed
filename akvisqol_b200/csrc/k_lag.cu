// Fused FFT cross-correlation lag search (reference src/xcorr.zig:197-251),
// three passes over the n-point complex buffer instead of one per stage group:
//
//   1. pack + global DIF stages: view the n = R * 4096 points as R rows of
//      4096 columns. The DIF stages with spans n .. 8192 only combine points
//      of one column, so a CTA loads `cols` whole columns (R x cols points,
//      64 KB), forms the envelopes on the fly from the signals, runs those
//      stages in shared memory and writes z once.
//   2. block stages + cross spectrum: the remaining DIF stages (spans
//      4096 .. 2) stay inside 4096-point blocks, and in bit-reversed order a
//      block's cross-spectrum partners Z[-k] all sit in one mirror block
//      (position u of block b pairs with 4095 - u of block b'), so a CTA loads
//      a block and its mirror, finishes the forward transform, forms the
//      cross terms, and runs the inverse's block stages (spans 2 .. 4096).
//   3. global DIT stages + argmax: columns again; after the last stage each
//      CTA reduces |Re| over its lags in the CPU's scan order and writes one
//      candidate; a final kernel picks the first maximum.
//
// Butterflies and twiddles are those of the radix-2 DIF/DIT (reference
// src/dsp/fft.zig:127-166); every schedule of them gives the same bits.
//
// The passes are written once for two complex types. double2 is the exact
// search: every product and sum rounded separately, the CPU's results bit
// for bit. float2 is the f32-nominated search every form runs (reference
// src/xcorr.zig:270-340, its GPU flow src/gpu/engine.zig:445-540): the same
// schedule in f32 with FMA, half the bytes per pass. Its correlation is within
// tol(n) n (|a|^2 + |b|^2) of the exact one, tol(n) = 8 eps_f32 log2(n)
// (src/gpu/engine.zig:820-822), so every lag whose |Re| lies within twice
// that of the largest is nominated (each inverse CTA keeps those within the
// slack of its own maximum, a superset), at most kLagCandCap of them per
// search; they are rescored by f64 dot products of the envelopes and the
// first maximum in ascending lag wins. A search with more candidates (long
// runs of near-equal correlation: silence, periodic signals), or whose two
// best rescored lags are a near-tie, reports it, and the host reruns it with
// the exact search, so the lag is always the exact search's.
#include <algorithm>
#include <cfloat>
#include <type_traits>

#include "device.cuh"
#include "kernels.h"

namespace vqb {

namespace {

constexpr int kB = 4096;        // block (and column-tile) points
constexpr int kThreads = 256;

__device__ inline double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ inline double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ inline double2 cmul(double2 x, double2 w) {
    return make_double2(x.x * w.x - x.y * w.y, x.x * w.y + x.y * w.x);
}
__device__ inline double2 cmul_conj(double2 x, double2 w) {
    const double wi = -w.y;
    return make_double2(x.x * w.x - x.y * wi, x.x * wi + x.y * w.x);
}
__device__ inline double2 cross_term(double2 x, double2 zy) {
    const double2 y = make_double2(zy.x, -zy.y);
    const double2 sum = make_double2(x.x + y.x, x.y + y.y);
    const double2 dif_c = make_double2(x.x - y.x, -(x.y - y.y));
    const double2 idc = make_double2(-dif_c.y, dif_c.x);
    return make_double2(0.25 * (sum.x * idc.x - sum.y * idc.y), 0.25 * (sum.x * idc.y + sum.y * idc.x));
}

// f32: products and sums fused where they chain.
__device__ inline float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ inline float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ inline float2 cmul(float2 x, float2 w) {
    return make_float2(__fmaf_rn(x.x, w.x, -(x.y * w.y)), __fmaf_rn(x.x, w.y, x.y * w.x));
}
__device__ inline float2 cmul_conj(float2 x, float2 w) {
    return make_float2(__fmaf_rn(x.x, w.x, x.y * w.y), __fmaf_rn(x.y, w.x, -(x.x * w.y)));
}
__device__ inline float2 cross_term(float2 x, float2 zy) {
    const float2 sum = make_float2(x.x + zy.x, x.y - zy.y);
    const float2 idc = make_float2(x.y + zy.y, x.x - zy.x);  // i * conj(x - conj(zy))
    return make_float2(0.25f * __fmaf_rn(sum.x, idc.x, -(sum.y * idc.y)),
                       0.25f * __fmaf_rn(sum.x, idc.y, sum.y * idc.x));
}

template <class C>
__device__ inline C *zbuf(const LagJob &j);
template <>
__device__ inline double2 *zbuf<double2>(const LagJob &j) {
    return j.z;
}
template <>
__device__ inline float2 *zbuf<float2>(const LagJob &j) {
    return j.z32;
}

// 16-byte asynchronous global-to-shared copy (both addresses 16-byte aligned).
__device__ inline void cp_async16(double2 *dst, const double2 *src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
}

__host__ __device__ inline int64_t pow2_at_least(int64_t x) {
    int64_t n = 1;
    while (n < x) n <<= 1;
    return n;
}

// Envelope parameters of one signal: mean and +-nyquist/N.
struct EnvParams {
    double mean, q;
};

__device__ inline EnvParams env_params(const VSig &s, const double *stats) {
    EnvParams p{0.0, 0.0};
    if (s.len > 0) {
        p.mean = stats[0] / (double)s.len;
        const int64_t N = pow2_at_least(s.len) > 32 ? pow2_at_least(s.len) : 32;
        p.q = stats[1] / (double)N;
    }
    return p;
}

// upperEnvelope (reference src/envelope.zig:45-52) at sample i.
__device__ inline double env_of(double x, const EnvParams &p, int64_t i) {
    const double pc = x - p.mean;
    const double nt = (i & 1) ? -p.q : p.q;
    return fabs(2.0 * (pc - nt) - 0.000001) + p.mean;
}
__device__ inline double env_at(const VSig &s, const EnvParams &p, int64_t i) { return env_of(vsig_at(s, i), p, i); }

template <bool RAW>
__device__ inline double2 packed(const LagJob &job, const EnvParams &pa, const EnvParams &pb, int64_t i) {
    double re = 0.0, im = 0.0;
    if (i < job.a.len) re = RAW ? vsig_at(job.a, i) : env_at(job.a, pa, i);
    if (i < job.b.len) im = RAW ? vsig_at(job.b, i) : env_at(job.b, pb, i);
    return make_double2(re, im);
}

// Point i of z in the search's type; the f32 search also sums the squares
// of the f64 envelope values (its nomination slack scales with them).
template <class C>
__device__ inline C as_point(double2 v, double &ea, double &eb) {
    if constexpr (std::is_same<C, float2>::value) {
        ea += v.x * v.x;
        eb += v.y * v.y;
        return make_float2((float)v.x, (float)v.y);
    } else {
        return v;
    }
}

template <class C, bool RAW>
__device__ inline C pack_point(const LagJob &job, const EnvParams &pa, const EnvParams &pb, int64_t i, double &ea,
                               double &eb) {
    const double2 v = packed<RAW>(job, pa, pb, i);
    if constexpr (std::is_same<C, float2>::value) {
        ea += v.x * v.x;
        eb += v.y * v.y;
        return make_float2((float)v.x, (float)v.y);
    } else {
        return v;
    }
}

// Sum of a double over the CTA in a fixed order (each warp by shuffles, then
// the warps in index order), returned to every thread.
__device__ inline double block_sum(double v) {
    __shared__ double warp_sum[32];
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    __syncthreads();  // warp_sum free (an earlier call may still be reading it)
    if ((threadIdx.x & 31) == 0) warp_sum[threadIdx.x >> 5] = v;
    __syncthreads();
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += warp_sum[w];
    return t;
}

// The f32 forward CTAs' envelope energies, summed.
template <class C>
__device__ inline void store_energy(const LagJob &job, double ea, double eb) {
    if constexpr (std::is_same<C, float2>::value) {
        ea = block_sum(ea);
        eb = block_sum(eb);
        if (threadIdx.x == 0) job.energy[blockIdx.x] = make_double2(ea, eb);
    }
}

// G column stages on x[t * cols + c] (t < R = 2^G rows); DIT reverses the
// stage order. Stage l has span n >> l; the twiddle of the lower point (t, c)
// is W_{n>>l}^j = top[j << l], j = m * 4096 + c0 + c with m = t mod 2h
// (h = R >> (l+1)). tcol holds those twiddles stage-major,
// tcol[off(l) + m * 4096 + col] = top[(m * 4096 + col) << l], so a CTA's
// columns read contiguous runs. Stages go in pairs (radix 4, one barrier)
// with a radix-2 stage where G is odd.
__device__ inline int64_t tcol_off(int G, int l) {
    // sum over l' < l of (R >> (l'+1)) * 4096
    const int64_t R = (int64_t)1 << G;
    return (R - (R >> l)) * kB;
}

template <class C, bool DIT>
__device__ inline void column_stage2(C *x, int G, int l, int cols, int64_t c0, const C *__restrict__ tcol) {
    const int R = 1 << G, h = R >> (l + 1);
    const C *tw = tcol + tcol_off(G, l) + c0;
    for (int bf = threadIdx.x; bf < (R >> 1) * cols; bf += blockDim.x) {
        const int pr = bf / cols, c = bf - pr * cols;
        const int m = pr % h;
        const int t = (pr / h) * 2 * h + m;
        const C w = tw[(int64_t)m * kB + c];
        C *pa = x + t * cols + c, *pb = x + (t + h) * cols + c;
        const C a = *pa;
        if (!DIT) {
            const C b = *pb;
            *pa = cadd(a, b);
            *pb = cmul(csub(a, b), w);
        } else {
            const C b = cmul_conj(*pb, w);
            *pa = cadd(a, b);
            *pb = csub(a, b);
        }
    }
}

// Stages l (span S) and l+1 (span S/2) on 4-row groups t0 + {0,q,2q,3q},
// q = R >> (l+2): stage l pairs (0,2),(1,3) with twiddle rows m and m+q,
// stage l+1 pairs (0,1),(2,3) with row m. DIT runs stage l+1 first.
template <class C, bool DIT>
__device__ inline void column_stage4(C *x, int G, int l, int cols, int64_t c0, const C *__restrict__ tcol) {
    const int R = 1 << G, q = R >> (l + 2);
    const C *tw1 = tcol + tcol_off(G, l) + c0, *tw2 = tcol + tcol_off(G, l + 1) + c0;
    for (int g = threadIdx.x; g < (R >> 2) * cols; g += blockDim.x) {
        const int pr = g / cols, c = g - pr * cols;
        const int m = pr % q;
        const int t0 = (pr / q) * 4 * q + m;
        C *p0 = x + t0 * cols + c, *p1 = p0 + q * cols, *p2 = p1 + q * cols, *p3 = p2 + q * cols;
        C x0 = *p0, x1 = *p1, x2 = *p2, x3 = *p3;
        const C wa = tw1[(int64_t)m * kB + c], wb = tw1[(int64_t)(m + q) * kB + c];
        const C w2 = tw2[(int64_t)m * kB + c];
        C a, b;
        if (!DIT) {
            a = x0, b = x2;
            x0 = cadd(a, b);
            x2 = cmul(csub(a, b), wa);
            a = x1, b = x3;
            x1 = cadd(a, b);
            x3 = cmul(csub(a, b), wb);
            a = x0, b = x1;
            x0 = cadd(a, b);
            x1 = cmul(csub(a, b), w2);
            a = x2, b = x3;
            x2 = cadd(a, b);
            x3 = cmul(csub(a, b), w2);
        } else {
            a = x0, b = cmul_conj(x1, w2);
            x0 = cadd(a, b);
            x1 = csub(a, b);
            a = x2, b = cmul_conj(x3, w2);
            x2 = cadd(a, b);
            x3 = csub(a, b);
            a = x0, b = cmul_conj(x2, wa);
            x0 = cadd(a, b);
            x2 = csub(a, b);
            a = x1, b = cmul_conj(x3, wb);
            x1 = cadd(a, b);
            x3 = csub(a, b);
        }
        *p0 = x0, *p1 = x1, *p2 = x2, *p3 = x3;
    }
}

template <class C, bool DIT>
__device__ inline void column_stages(C *x, int G, int cols, int64_t c0, const C *__restrict__ tcol) {
    if (!DIT) {
        int l = 0;
        for (; l + 1 < G; l += 2) {
            column_stage4<C, false>(x, G, l, cols, c0, tcol);
            __syncthreads();
        }
        if (l < G) {
            column_stage2<C, false>(x, G, l, cols, c0, tcol);
            __syncthreads();
        }
    } else {
        int l = G - 1;
        if (G & 1) {
            column_stage2<C, true>(x, G, l, cols, c0, tcol);
            __syncthreads();
            --l;
        }
        for (; l >= 1; l -= 2) {
            column_stage4<C, true>(x, G, l - 1, cols, c0, tcol);
            __syncthreads();
        }
    }
}

// Pass 1: pack + DIF column stages. grid (n / (R*cols) ... = 4096/cols, jobs).
template <class C, bool RAW>
__global__ void __launch_bounds__(kThreads, 3) fwd_columns(const LagJob *__restrict__ jobs, int G,
                                                        const C *__restrict__ tcol) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *sm = reinterpret_cast<C *>(smem_raw);
    const LagJob job = jobs[blockIdx.y];
    const int cols = kB >> G > 0 ? (kB >> G) : 1;
    const int64_t c0 = (int64_t)blockIdx.x * cols;
    EnvParams pa{}, pb{};
    if (!RAW) {
        pa = env_params(job.a, job.stats_a);
        pb = env_params(job.b, job.stats_b);
    }
    // R * cols = kB points, a fixed 16 per thread: four at a time keeps
    // eight signal loads in flight within the three-CTA register budget.
    double ea = 0.0, eb = 0.0;
#pragma unroll 4
    for (int k = 0; k < kB / kThreads; ++k) {
        const int e = threadIdx.x + k * kThreads;
        const int t = e / cols, c = e - t * cols;
        sm[e] = pack_point<C, RAW>(job, pa, pb, (int64_t)t * kB + c0 + c, ea, eb);
    }
    __syncthreads();
    column_stages<C, false>(sm, G, cols, c0, tcol);
    C *z = zbuf<C>(job);
#pragma unroll 4
    for (int k = 0; k < kB / kThreads; ++k) {
        const int e = threadIdx.x + k * kThreads;
        const int t = e / cols, c = e - t * cols;
        z[(int64_t)t * kB + c0 + c] = sm[e];
    }
    store_energy<C>(job, ea, eb);
}

// Radix-4/radix-2 block stages of one B-point block in shared memory
// (tw[k] = W_B^k); the same stage plans as the stand-alone block passes.
template <class C>
__device__ inline void dif2(C *sm, int B, int s, const C *tw) {
    const int h = s >> 1, step = B / s;
    for (int bf = threadIdx.x; bf < (B >> 1); bf += blockDim.x) {
        const int blk = bf / h, j = bf - blk * h;
        const int i0 = blk * s + j;
        const C a = sm[i0], b = sm[i0 + h];
        sm[i0] = cadd(a, b);
        sm[i0 + h] = cmul(csub(a, b), tw[j * step]);
    }
}
template <class C>
__device__ inline void dit2(C *sm, int B, int s, const C *tw) {
    const int h = s >> 1, step = B / s;
    for (int bf = threadIdx.x; bf < (B >> 1); bf += blockDim.x) {
        const int blk = bf / h, j = bf - blk * h;
        const int i0 = blk * s + j;
        const C a = sm[i0];
        const C b = cmul_conj(sm[i0 + h], tw[j * step]);
        sm[i0] = cadd(a, b);
        sm[i0 + h] = csub(a, b);
    }
}
template <class C>
__device__ inline void dif4(C *sm, int B, int s, const C *tw) {
    const int q = s >> 2, st1 = B / s, st2 = 2 * st1;
    for (int g = threadIdx.x; g < (B >> 2); g += blockDim.x) {
        const int blk = g / q, j = g - blk * q;
        const int b0 = blk * s + j;
        C x0 = sm[b0], x1 = sm[b0 + q], x2 = sm[b0 + 2 * q], x3 = sm[b0 + 3 * q];
        C a = x0, b = x2;
        x0 = cadd(a, b);
        x2 = cmul(csub(a, b), tw[j * st1]);
        a = x1, b = x3;
        x1 = cadd(a, b);
        x3 = cmul(csub(a, b), tw[(j + q) * st1]);
        const C w = tw[j * st2];
        a = x0, b = x1;
        x0 = cadd(a, b);
        x1 = cmul(csub(a, b), w);
        a = x2, b = x3;
        x2 = cadd(a, b);
        x3 = cmul(csub(a, b), w);
        sm[b0] = x0, sm[b0 + q] = x1, sm[b0 + 2 * q] = x2, sm[b0 + 3 * q] = x3;
    }
}
template <class C>
__device__ inline void dit4(C *sm, int B, int s, const C *tw) {
    const int q = s >> 2, st1 = B / s, st2 = 2 * st1;
    for (int g = threadIdx.x; g < (B >> 2); g += blockDim.x) {
        const int blk = g / q, j = g - blk * q;
        const int b0 = blk * s + j;
        C x0 = sm[b0], x1 = sm[b0 + q], x2 = sm[b0 + 2 * q], x3 = sm[b0 + 3 * q];
        const C w = tw[j * st2];
        C a = x0, b = cmul_conj(x1, w);
        x0 = cadd(a, b);
        x1 = csub(a, b);
        a = x2, b = cmul_conj(x3, w);
        x2 = cadd(a, b);
        x3 = csub(a, b);
        a = x0, b = cmul_conj(x2, tw[j * st1]);
        x0 = cadd(a, b);
        x2 = csub(a, b);
        a = x1, b = cmul_conj(x3, tw[(j + q) * st1]);
        x1 = cadd(a, b);
        x3 = csub(a, b);
        sm[b0] = x0, sm[b0 + q] = x1, sm[b0 + 2 * q] = x2, sm[b0 + 3 * q] = x3;
    }
}

// Both blocks' stages advance together (one barrier per stage pair).
template <class C>
__device__ inline void blocks_dif(C *s0, C *s1, int B, const C *tw) {
    int stages = 0;
    for (int r = B; r > 1; r >>= 1) ++stages;
    int s = B;
    for (; stages >= 2; stages -= 2, s >>= 2) {
        dif4(s0, B, s, tw);
        if (s1) dif4(s1, B, s, tw);
        __syncthreads();
    }
    if (stages == 1) {
        dif2(s0, B, 2, tw);
        if (s1) dif2(s1, B, 2, tw);
        __syncthreads();
    }
}
template <class C>
__device__ inline void blocks_dit(C *s0, C *s1, int B, const C *tw) {
    int stages = 0;
    for (int r = B; r > 1; r >>= 1) ++stages;
    int s = 4;
    if (stages & 1) {
        dit2(s0, B, 2, tw);
        if (s1) dit2(s1, B, 2, tw);
        __syncthreads();
        s = 8;
    }
    for (; s <= B; s <<= 2) {
        dit4(s0, B, s, tw);
        if (s1) dit4(s1, B, s, tw);
        __syncthreads();
    }
}

// Pass 2 on the 4096-point blocks, in registers: each radix-2 stage group of
// four (spans S0 .. S0/8) runs on 16 points per thread (point j + m*S0/16 of
// an S0-block, m = 0..15), so the 12 DIF stages, the cross terms and the 12
// DIT stages take three register passes each way with four shared-memory
// round trips in all (the first and last passes read and write global
// memory directly). Shared memory holds the two blocks padded by one point
// per 16 (position e at e + e/16), which keeps all three access patterns
// (stride 256, 16 and 1 points) free of bank conflicts. Twiddles come from
// the stage-major table tst[(4096 - S) + k] = W_S^k, contiguous per stage.
//
// CTA 0: block 0 (partners inside it, reference pairing
// src/xcorr.zig:211-229); CTA 1: block 1 (u <-> B-1-u); CTA k >= 2: blocks
// b and b' = 3*hb - 1 - b for the (k-1)-th pair, hb = 2 * floor_pow2(k-1).
// Threads 0..255 own the first block, 256..511 the second.
constexpr int kMidThreads = 512;
constexpr int kPadB = kB + kB / 16;

__device__ inline int padi(int e) { return e + (e >> 4); }

// x W_16^k, or x conj(W_16^k) (CONJ), W_16^k = e^{-2 pi i k / 16}, k < 8:
// the f32 search's span-16 stages take their twiddles as constants, the
// products by 1 and -i as exchanges and the ones by W_16^2 and W_16^6 as a
// sum and a difference scaled once. k is a constant once the stage loops
// are unrolled, so the switch folds.
__device__ inline float2 w16_mul(float2 x, int k, bool conj) {
    constexpr float c1 = 0.92387953251128674f, s1 = 0.38268343236508978f, h = 0.70710678118654752f;
    float wr = 1.0f, wi = 0.0f;
    switch (k) {
        case 0:
            return x;
        case 2:
            return conj ? make_float2(h * (x.x - x.y), h * (x.x + x.y)) : make_float2(h * (x.x + x.y), h * (x.y - x.x));
        case 4:
            return conj ? make_float2(-x.y, x.x) : make_float2(x.y, -x.x);
        case 6:
            return conj ? make_float2(-h * (x.x + x.y), h * (x.x - x.y))
                        : make_float2(h * (x.y - x.x), -h * (x.x + x.y));
        case 1: wr = c1, wi = -s1; break;
        case 3: wr = s1, wi = -c1; break;
        case 5: wr = -s1, wi = -c1; break;
        default: wr = -c1, wi = -s1; break;
    }
    if (conj) wi = -wi;
    return make_float2(__fmaf_rn(x.x, wr, -(x.y * wi)), __fmaf_rn(x.x, wi, x.y * wr));
}

template <class C, int S0>
__device__ inline void dif16(C (&x)[16], int j, const C *__restrict__ tst) {
    constexpr int q = S0 / 16;
    // spans 16 .. 2 (j = 0) of the f32 search: constant twiddles
    constexpr bool konst = S0 == 16 && std::is_same<C, float2>::value;
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        const int half = 8 >> r;
        const C *tw = tst + (kB - (S0 >> r));
#pragma unroll
        for (int m = 0; m < 16; ++m) {
            if (m & half) continue;
            const C a = x[m], b = x[m + half];
            x[m] = cadd(a, b);
            if constexpr (konst) {
                x[m + half] = w16_mul(csub(a, b), (m & (half - 1)) << r, false);
            } else {
                const C w = __ldg(tw + j + (m & (half - 1)) * q);
                x[m + half] = cmul(csub(a, b), w);
            }
        }
    }
}

template <class C, int S0>
__device__ inline void dit16(C (&x)[16], int j, const C *__restrict__ tst) {
    constexpr int q = S0 / 16;
    constexpr bool konst = S0 == 16 && std::is_same<C, float2>::value;
#pragma unroll
    for (int r = 3; r >= 0; --r) {
        const int half = 8 >> r;
        const C *tw = tst + (kB - (S0 >> r));
#pragma unroll
        for (int m = 0; m < 16; ++m) {
            if (m & half) continue;
            C b;
            if constexpr (konst) {
                b = w16_mul(x[m + half], (m & (half - 1)) << r, true);
            } else {
                const C w = __ldg(tw + j + (m & (half - 1)) * q);
                b = cmul_conj(x[m + half], w);
            }
            const C a = x[m];
            x[m] = cadd(a, b);
            x[m + half] = csub(a, b);
        }
    }
}

template <class C>
__global__ void __launch_bounds__(kMidThreads, sizeof(C) == 8 ? 2 : 1) middle_blocks(const LagJob *__restrict__ jobs,
                                                                const C *__restrict__ tst) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *sm = reinterpret_cast<C *>(smem_raw);
    const LagJob job = jobs[blockIdx.y];
    const int k = blockIdx.x;
    int64_t b0 = 0, b1 = -1;
    if (k == 1) {
        b0 = 1;
    } else if (k >= 2) {
        const int64_t i = k - 1;
        const int64_t p = (int64_t)1 << (63 - __clzll(i));
        const int64_t hb = 2 * p;
        b0 = i + p;
        b1 = 3 * hb - 1 - b0;
    }
    const int half = threadIdx.x >> 8, t = threadIdx.x & 255;
    const bool active = half == 0 || b1 >= 0;
    C *own = sm + half * kPadB;
    C *z = zbuf<C>(job) + (half == 1 && b1 >= 0 ? b1 : b0) * kB;
    C x[16];
    // DIF spans 4096 .. 512: points t + 256 m
    if (active) {
#pragma unroll
        for (int m = 0; m < 16; ++m) x[m] = z[t + 256 * m];
        dif16<C, 4096>(x, t, tst);
#pragma unroll
        for (int m = 0; m < 16; ++m) own[padi(t + 256 * m)] = x[m];
    }
    __syncthreads();
    // DIF spans 256 .. 32: points (t/16)*256 + t%16 + 16 m
    const int base2 = (t >> 4) * 256 + (t & 15);
    if (active) {
#pragma unroll
        for (int m = 0; m < 16; ++m) x[m] = own[padi(base2 + 16 * m)];
        dif16<C, 256>(x, t & 15, tst);
#pragma unroll
        for (int m = 0; m < 16; ++m) own[padi(base2 + 16 * m)] = x[m];
    }
    __syncthreads();
    // DIF spans 16 .. 2: points 16 t + m
    if (active) {
#pragma unroll
        for (int m = 0; m < 16; ++m) x[m] = own[padi(16 * t + m)];
        dif16<C, 16>(x, 0, tst);
#pragma unroll
        for (int m = 0; m < 16; ++m) own[padi(16 * t + m)] = x[m];
    }
    __syncthreads();
    // cross terms: each point with its partner's forward value
    if (active) {
#pragma unroll
        for (int m = 0; m < 16; ++m) {
            const int u = 16 * t + m;
            C zp;
            if (b1 >= 0) {
                zp = sm[(1 - half) * kPadB + padi(kB - 1 - u)];
            } else if (k == 1) {
                zp = own[padi(kB - 1 - u)];
            } else {
                int p = u;
                if (u >= 2) {
                    const int h = 1 << (31 - __clz(u));
                    p = 3 * h - 1 - u;
                }
                zp = own[padi(p)];
            }
            x[m] = cross_term(x[m], zp);
        }
    }
    __syncthreads();
    // DIT spans 2 .. 16, then 32 .. 256, then 512 .. 4096 (to global memory)
    if (active) {
        dit16<C, 16>(x, 0, tst);
#pragma unroll
        for (int m = 0; m < 16; ++m) own[padi(16 * t + m)] = x[m];
    }
    __syncthreads();
    if (active) {
#pragma unroll
        for (int m = 0; m < 16; ++m) x[m] = own[padi(base2 + 16 * m)];
        dit16<C, 256>(x, t & 15, tst);
#pragma unroll
        for (int m = 0; m < 16; ++m) own[padi(base2 + 16 * m)] = x[m];
    }
    __syncthreads();
    if (active) {
#pragma unroll
        for (int m = 0; m < 16; ++m) x[m] = own[padi(t + 256 * m)];
        dit16<C, 4096>(x, t, tst);
#pragma unroll
        for (int m = 0; m < 16; ++m) z[t + 256 * m] = x[m];
    }
}

struct Best {
    double v;
    int64_t key;
};
__device__ inline Best better(Best a, Best b) {
    if (b.v > a.v) return b;
    if (b.v == a.v && b.key < a.key) return b;
    return a;
}
// Position i's key in the CPU's scan order (negative lags first), or -1.
__device__ inline int64_t lag_key(int64_t i, int64_t n, int64_t max_lag) {
    if (i >= n - max_lag) return i - (n - max_lag);
    if (i <= max_lag) return max_lag + i;
    return -1;
}

__device__ inline void block_best(Best best, double *pv, int64_t *pk, int64_t slot) {
    for (int off = 16; off > 0; off >>= 1) {
        Best o{__shfl_down_sync(0xffffffffu, best.v, off), __shfl_down_sync(0xffffffffu, best.key, off)};
        best = better(best, o);
    }
    __shared__ Best warp_best[kThreads / 32];
    if ((threadIdx.x & 31) == 0) warp_best[threadIdx.x >> 5] = best;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) best = better(best, warp_best[w]);
        pv[slot] = best.v;
        pk[slot] = best.key;
    }
}

// Pass 3: DIT column stages, then this CTA's lag candidates.
__global__ void __launch_bounds__(kThreads) inv_columns_argmax(const LagJob *__restrict__ jobs, int G,
                                                               const double2 *__restrict__ tcol, double *pv,
                                                               int64_t *pk, int parts) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2 *sm = reinterpret_cast<double2 *>(smem_raw);
    const LagJob job = jobs[blockIdx.y];
    const int cols = kB >> G > 0 ? (kB >> G) : 1;
    const int64_t c0 = (int64_t)blockIdx.x * cols;
    // The tile arrives by asynchronous 16-byte copies: all 16 of a thread's
    // loads in flight at once, none staged through registers.
#pragma unroll
    for (int k = 0; k < kB / kThreads; ++k) {
        const int e = threadIdx.x + k * kThreads;
        const int t = e / cols, c = e - t * cols;
        cp_async16(sm + e, job.z + (int64_t)t * kB + c0 + c);
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    __syncthreads();
    column_stages<double2, true>(sm, G, cols, c0, tcol);
    const int64_t n = job.n, max_lag = job.biggest - 1;
    Best best{-INFINITY, INT64_MAX};
    for (int e = threadIdx.x; e < kB; e += blockDim.x) {
        const int t = e / cols, c = e - t * cols;
        const int64_t key = lag_key((int64_t)t * kB + c0 + c, n, max_lag);
        if (key >= 0) best = better(best, Best{fabs(sm[e].x), key});
    }
    block_best(best, pv, pk, (int64_t)blockIdx.y * parts + blockIdx.x);
}

// Register forms of passes 1 and 3 for R = 2^G rows, 4 <= G <= 11 (signals up to 2^22 samples). Thread
// q of a column (c, q: c fastest, so rows are coalesced) keeps 16 points of
// column c in registers, and the G column stages run in groups of four:
//
//   group A (spans R/2 .. R/16):    rows q + (R/16) m
//   group B (spans R/32 .. R/256):  rows b (R/16) + q' + (R/256) m, with
//                                   q = b (R/256) + q'   (only if G > 8)
//   tail (spans <= 8):              rows 16 q + m
//
// with one shared-memory exchange between groups. Each stage's butterflies
// are the radix-2 ones of the shared-memory passes, with the same twiddles
// (stage l, lower row t: tcol[off(l) + (t mod 2h) 4096 + col]), so the
// results are the same bits; a group costs one barrier instead of one per
// stage pair.
template <class C, int G, bool DIT>
__device__ inline void column_group4(C (&x)[16], int l0, int stride, int base_mod, const C *__restrict__ tcol,
                                     int64_t col) {
#pragma unroll
    for (int kk = 0; kk < 4; ++kk) {
        const int k = DIT ? 3 - kk : kk;
        const int l = l0 + k, half = 8 >> k;
        const C *tw = tcol + tcol_off(G, l) + col;
#pragma unroll
        for (int m = 0; m < 16; ++m) {
            if (m & half) continue;
            const C w = __ldg(tw + (int64_t)(base_mod + stride * (m & (half - 1))) * kB);
            const C a = x[m];
            if (!DIT) {
                const C b = x[m + half];
                x[m] = cadd(a, b);
                x[m + half] = cmul(csub(a, b), w);
            } else {
                const C b = cmul_conj(x[m + half], w);
                x[m] = cadd(a, b);
                x[m + half] = csub(a, b);
            }
        }
    }
}

// Stages l0 .. G-1, whose spans h = R >> (l+1) are at most 8, on rows
// 16 q + m (t mod 2h = m mod 2h).
template <class C, int G, bool DIT>
__device__ inline void column_tail(C (&x)[16], int l0, const C *__restrict__ tcol, int64_t col) {
    constexpr int R = 1 << G;
#pragma unroll
    for (int kk = 0; kk < 4; ++kk) {
        const int l = DIT ? G - 1 - kk : l0 + kk;
        if (l < l0 || l >= G) continue;
        const int h = R >> (l + 1);
        const C *tw = tcol + tcol_off(G, l) + col;
#pragma unroll
        for (int m = 0; m < 16; ++m) {
            if (m & h) continue;
            const C w = __ldg(tw + (int64_t)(m & (h - 1)) * kB);
            const C a = x[m];
            if (!DIT) {
                const C b = x[m + h];
                x[m] = cadd(a, b);
                x[m + h] = cmul(csub(a, b), w);
            } else {
                const C b = cmul_conj(x[m + h], w);
                x[m] = cadd(a, b);
                x[m + h] = csub(a, b);
            }
        }
    }
}

// Row of register m in group A, group B and the tail, for thread q.
template <int G>
__device__ inline int row_a(int q, int m) { return q + ((1 << G) / 16) * m; }
template <int G>
__device__ inline int row_b(int q, int m) {
    constexpr int R = 1 << G, s = R / 256 > 0 ? R / 256 : 1;
    return (q / s) * (R / 16) + (q % s) + s * m;
}
__device__ inline int row_t(int q, int m) { return 16 * q + m; }

template <class C, int G, bool RAW>
__global__ void __launch_bounds__(kThreads, 2) fwd_columns_reg(const LagJob *__restrict__ jobs,
                                                            const C *__restrict__ tcol) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *sm = reinterpret_cast<C *>(smem_raw);
    constexpr int R = 1 << G, cols = kB >> G;
    const LagJob job = jobs[blockIdx.y];
    const int c = threadIdx.x % cols, q = threadIdx.x / cols;
    const int64_t col = (int64_t)blockIdx.x * cols + c;
    EnvParams pa{}, pb{};
    if (!RAW) {
        pa = env_params(job.a, job.stats_a);
        pb = env_params(job.b, job.stats_b);
    }
    C x[16];
    double ea = 0.0, eb = 0.0;
#pragma unroll
    for (int m = 0; m < 16; ++m) x[m] = pack_point<C, RAW>(job, pa, pb, (int64_t)row_a<G>(q, m) * kB + col, ea, eb);
    column_group4<C, G, false>(x, 0, R / 16, q, tcol, col);
    C *z = zbuf<C>(job);
    if (G > 4) {
#pragma unroll
        for (int m = 0; m < 16; ++m) sm[row_a<G>(q, m) * cols + c] = x[m];
        __syncthreads();
        if (G > 8) {
            constexpr int s = R / 256 > 0 ? R / 256 : 1;
#pragma unroll
            for (int m = 0; m < 16; ++m) x[m] = sm[row_b<G>(q, m) * cols + c];
            column_group4<C, G, false>(x, 4, s, q % s, tcol, col);
#pragma unroll
            for (int m = 0; m < 16; ++m) sm[row_b<G>(q, m) * cols + c] = x[m];
            __syncthreads();
        }
#pragma unroll
        for (int m = 0; m < 16; ++m) x[m] = sm[row_t(q, m) * cols + c];
        column_tail<C, G, false>(x, G > 8 ? 8 : 4, tcol, col);
#pragma unroll
        for (int m = 0; m < 16; ++m) z[(int64_t)row_t(q, m) * kB + col] = x[m];
    } else {
#pragma unroll
        for (int m = 0; m < 16; ++m) z[(int64_t)row_a<G>(q, m) * kB + col] = x[m];
    }
    store_energy<C>(job, ea, eb);
}

// 8-byte asynchronous copy to shared memory; `in` false writes zeros (no
// bytes are read; src must still be a global address).
__device__ inline void cp_async8z(double *dst, const double *src, bool in) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(src), "r"(in ? 8 : 0) : "memory");
}

// Pass 1 as fwd_columns_reg, with the CTA's 4096 (a, b) samples first staged
// in shared memory by asynchronous copies (16 a thread, consecutive threads
// on consecutive columns of a row, zero outside the stored samples): every
// load is in flight at once and none holds a register, where the register
// form's loads queue behind its 128-register budget. The values, and so the
// results, are the register form's. The stage is then the exchange buffer.
template <class C, int G, bool RAW>
__global__ void __launch_bounds__(kThreads, sizeof(C) == 8 ? 3 : 2) fwd_columns_staged(const LagJob *__restrict__ jobs,
                                                               const C *__restrict__ tcol) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *sm = reinterpret_cast<C *>(smem_raw);
    double2 *stage = reinterpret_cast<double2 *>(smem_raw);  // [row][col] of the tile
    constexpr int R = 1 << G, cols = kB >> G;
    const LagJob job = jobs[blockIdx.y];
    const int c = threadIdx.x % cols, q = threadIdx.x / cols;
    const int64_t c0 = (int64_t)blockIdx.x * cols, col = c0 + c;
    C *z = zbuf<C>(job);
    const double *guard = reinterpret_cast<const double *>(z);
#pragma unroll
    for (int k = 0; k < kB / kThreads; ++k) {
        const int e = threadIdx.x + k * kThreads;
        const int t = e / cols, cc = e - t * cols;
        const int64_t i = (int64_t)t * kB + c0 + cc;
        const int64_t ja = i - job.a.head, jb = i - job.b.head;
        const bool ina = i < job.a.len && (uint64_t)ja < (uint64_t)job.a.avail;
        const bool inb = i < job.b.len && (uint64_t)jb < (uint64_t)job.b.avail;
        cp_async8z(&stage[e].x, ina ? job.a.base + ja : guard, ina);
        cp_async8z(&stage[e].y, inb ? job.b.base + jb : guard, inb);
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    EnvParams pa{}, pb{};
    if (!RAW) {
        pa = env_params(job.a, job.stats_a);
        pb = env_params(job.b, job.stats_b);
    }
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    __syncthreads();
    C x[16];
    double ea = 0.0, eb = 0.0;
    if constexpr (std::is_same<C, float2>::value && !RAW) {
        // The f32 search forms the envelopes in f32: a few f32 ulps of each
        // value, |delta corr| <= ~3 eps_f32 (|a|^2 + |b|^2), far inside the
        // nomination slack; the rescoring uses the f64 envelopes.
        const float ma = (float)pa.mean, qa = (float)pa.q, mb = (float)pb.mean, qb = (float)pb.q;
        float ea32 = 0.0f, eb32 = 0.0f;
#pragma unroll
        for (int m = 0; m < 16; ++m) {
            const int64_t i = (int64_t)row_a<G>(q, m) * kB + col;
            const double2 v = stage[row_a<G>(q, m) * cols + c];
            float re = 0.0f, im = 0.0f;
            if (i < job.a.len) re = fabsf(__fmaf_rn(2.0f, ((float)v.x - ma) - ((i & 1) ? -qa : qa), -1e-6f)) + ma;
            if (i < job.b.len) im = fabsf(__fmaf_rn(2.0f, ((float)v.y - mb) - ((i & 1) ? -qb : qb), -1e-6f)) + mb;
            ea32 = __fmaf_rn(re, re, ea32);
            eb32 = __fmaf_rn(im, im, eb32);
            x[m] = make_float2(re, im);
        }
        ea = ea32;
        eb = eb32;
    } else {
#pragma unroll
        for (int m = 0; m < 16; ++m) {
            const int64_t i = (int64_t)row_a<G>(q, m) * kB + col;
            const double2 v = stage[row_a<G>(q, m) * cols + c];
            double re = 0.0, im = 0.0;
            if (i < job.a.len) re = RAW ? v.x : env_of(v.x, pa, i);
            if (i < job.b.len) im = RAW ? v.y : env_of(v.y, pb, i);
            x[m] = as_point<C>(make_double2(re, im), ea, eb);
        }
    }
    __syncthreads();  // the stage becomes the exchange buffer
    column_group4<C, G, false>(x, 0, R / 16, q, tcol, col);
    if (G > 4) {
#pragma unroll
        for (int m = 0; m < 16; ++m) sm[row_a<G>(q, m) * cols + c] = x[m];
        __syncthreads();
        if (G > 8) {
            constexpr int s = R / 256 > 0 ? R / 256 : 1;
#pragma unroll
            for (int m = 0; m < 16; ++m) x[m] = sm[row_b<G>(q, m) * cols + c];
            column_group4<C, G, false>(x, 4, s, q % s, tcol, col);
#pragma unroll
            for (int m = 0; m < 16; ++m) sm[row_b<G>(q, m) * cols + c] = x[m];
            __syncthreads();
        }
#pragma unroll
        for (int m = 0; m < 16; ++m) x[m] = sm[row_t(q, m) * cols + c];
        column_tail<C, G, false>(x, G > 8 ? 8 : 4, tcol, col);
#pragma unroll
        for (int m = 0; m < 16; ++m) z[(int64_t)row_t(q, m) * kB + col] = x[m];
    } else {
#pragma unroll
        for (int m = 0; m < 16; ++m) z[(int64_t)row_a<G>(q, m) * kB + col] = x[m];
    }
    store_energy<C>(job, ea, eb);
}

template <int G>
__global__ void __launch_bounds__(kThreads, 2) inv_columns_reg(const LagJob *__restrict__ jobs,
                                                            const double2 *__restrict__ tcol, double *pv,
                                                            int64_t *pk, int parts) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2 *sm = reinterpret_cast<double2 *>(smem_raw);
    constexpr int R = 1 << G, cols = kB >> G;
    const LagJob job = jobs[blockIdx.y];
    const int c = threadIdx.x % cols, q = threadIdx.x / cols;
    const int64_t col = (int64_t)blockIdx.x * cols + c;
    double2 x[16];
    if (G > 4) {
#pragma unroll
        for (int m = 0; m < 16; ++m) x[m] = job.z[(int64_t)row_t(q, m) * kB + col];
        column_tail<double2, G, true>(x, G > 8 ? 8 : 4, tcol, col);
#pragma unroll
        for (int m = 0; m < 16; ++m) sm[row_t(q, m) * cols + c] = x[m];
        __syncthreads();
        if (G > 8) {
            constexpr int s = R / 256 > 0 ? R / 256 : 1;
#pragma unroll
            for (int m = 0; m < 16; ++m) x[m] = sm[row_b<G>(q, m) * cols + c];
            column_group4<double2, G, true>(x, 4, s, q % s, tcol, col);
#pragma unroll
            for (int m = 0; m < 16; ++m) sm[row_b<G>(q, m) * cols + c] = x[m];
            __syncthreads();
        }
#pragma unroll
        for (int m = 0; m < 16; ++m) x[m] = sm[row_a<G>(q, m) * cols + c];
    } else {
#pragma unroll
        for (int m = 0; m < 16; ++m) x[m] = job.z[(int64_t)row_a<G>(q, m) * kB + col];
    }
    column_group4<double2, G, true>(x, 0, R / 16, q, tcol, col);
    const int64_t n = job.n, max_lag = job.biggest - 1;
    Best best{-INFINITY, INT64_MAX};
#pragma unroll
    for (int m = 0; m < 16; ++m) {
        const int64_t key = lag_key((int64_t)row_a<G>(q, m) * kB + col, n, max_lag);
        if (key >= 0) best = better(best, Best{fabs(x[m].x), key});
    }
    block_best(best, pv, pk, (int64_t)blockIdx.y * parts + blockIdx.x);
}

// Single-block transforms (n <= 4096): pack, DIF, cross, DIT, argmax in one CTA.
template <bool RAW>
__global__ void __launch_bounds__(kThreads) small_lag(const LagJob *__restrict__ jobs, const double2 *__restrict__ tw,
                                                      double *pv, int64_t *pk) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2 *sm = reinterpret_cast<double2 *>(smem_raw);
    const LagJob job = jobs[blockIdx.y];
    const int B = (int)job.n;
    EnvParams pa{}, pb{};
    if (!RAW) {
        pa = env_params(job.a, job.stats_a);
        pb = env_params(job.b, job.stats_b);
    }
    for (int u = threadIdx.x; u < B; u += blockDim.x) sm[u] = packed<RAW>(job, pa, pb, u);
    __syncthreads();
    blocks_dif<double2>(sm, nullptr, B, tw);
    for (int i = threadIdx.x; i < (B > 1 ? B / 2 : 1); i += blockDim.x) {
        if (i == 0) {
            sm[0] = cross_term(sm[0], sm[0]);
            if (B > 1) sm[1] = cross_term(sm[1], sm[1]);
            continue;
        }
        const int p = 1 << (31 - __clz(i));
        const int h = 2 * p;
        const int a = i + p, b = 3 * h - 1 - a;
        const double2 za = sm[a], zb = sm[b];
        sm[a] = cross_term(za, zb);
        sm[b] = cross_term(zb, za);
    }
    __syncthreads();
    blocks_dit<double2>(sm, nullptr, B, tw);
    const int64_t max_lag = job.biggest - 1;
    Best best{-INFINITY, INT64_MAX};
    for (int u = threadIdx.x; u < B; u += blockDim.x) {
        const int64_t key = lag_key(u, B, max_lag);
        if (key >= 0) best = better(best, Best{fabs(sm[u].x), key});
    }
    block_best(best, pv, pk, blockIdx.y);
}

// One warp per job: lanes stride over the candidates, then a shuffle
// reduction (`better` is associative and commutative: the largest value,
// ties to the smallest key, i.e. the CPU scan's first maximum).
__global__ void pick_lag(const LagJob *__restrict__ jobs, int njobs, const double *pv, const int64_t *pk, int parts) {
    const int j = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (j >= njobs) return;
    Best best{-INFINITY, INT64_MAX};
    for (int p = lane; p < parts; p += 32)
        best = better(best, Best{pv[(int64_t)j * parts + p], pk[(int64_t)j * parts + p]});
    for (int off = 16; off > 0; off >>= 1) {
        Best o{__shfl_down_sync(0xffffffffu, best.v, off), __shfl_down_sync(0xffffffffu, best.key, off)};
        best = better(best, o);
    }
    if (lane == 0) *jobs[j].lag_out = best.key == INT64_MAX ? 0 : best.key - (jobs[j].biggest - 1);
}

// ---- f32 search: nomination, pick, f64 rescoring ---------------------------

// Twice the f32 correlation's error bound, 2 tol(n) n (|a|^2 + |b|^2) with
// tol(n) = 8 eps_f32 log2(n) (reference refineSlack src/xcorr.zig:302-308,
// lagTolerance src/gpu/engine.zig:820-822), from the forward CTAs' energy
// sums. Every thread gets the same value (a fixed summation order).
__device__ inline double job_slack(const LagJob &job, int parts) {
    if (job.slack_fixed > 0.0) return job.slack_fixed;
    double e = 0.0;
    for (int p = threadIdx.x; p < parts; p += blockDim.x) e += job.energy[p].x + job.energy[p].y;
    e = block_sum(e);
    int lg = 0;
    for (int64_t r = job.n; r > 1; r >>= 1) ++lg;
    const double tol = 8.0 * (double)FLT_EPSILON * (double)lg;
    return 2.0 * tol * e * (double)job.n;
}

__device__ inline float block_max(float v) {
    __shared__ float warp_max[32];
    for (int off = 16; off > 0; off >>= 1) v = fmaxf(v, __shfl_down_sync(0xffffffffu, v, off));
    __syncthreads();
    if ((threadIdx.x & 31) == 0) warp_max[threadIdx.x >> 5] = v;
    __syncthreads();
    float t = -INFINITY;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t = fmaxf(t, warp_max[w]);
    return t;
}

// This CTA's nomination record: its largest |Re| over valid lags (key >= 0)
// and every lag within `slack` of it (a superset of the search's candidates
// here, since the search's largest is at least this CTA's).
__device__ inline void block_nominate(const float (&v)[16], const int32_t (&key)[16], double slack, LagCands *out) {
    float top = -INFINITY;
#pragma unroll
    for (int m = 0; m < 16; ++m)
        if (key[m] >= 0) top = fmaxf(top, v[m]);
    top = block_max(top);
    __shared__ int count;
    if (threadIdx.x == 0) count = 0;
    __syncthreads();
    const double floor = (double)top - slack;
#pragma unroll
    for (int m = 0; m < 16; ++m) {
        if (key[m] >= 0 && (double)v[m] >= floor) {
            const int i = atomicAdd(&count, 1);
            if (i < kLagCandCap) {
                out->v[i] = v[m];
                out->key[i] = key[m];
            }
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        out->top = top;
        out->count = count;
    }
}

// 8-byte asynchronous global-to-shared copy (both addresses 8-byte aligned).
__device__ inline void cp_async8(float2 *dst, const float2 *src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
}

// Pass 3 of the f32 search, shared-memory column form (any G): DIT column
// stages, then this CTA's nomination record. parts: CTAs per job.
__global__ void __launch_bounds__(kThreads) inv_columns_nominate(const LagJob *__restrict__ jobs, int G,
                                                                 const float2 *__restrict__ tcol, int parts) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2 *sm = reinterpret_cast<float2 *>(smem_raw);
    const LagJob job = jobs[blockIdx.y];
    const int cols = kB >> G > 0 ? (kB >> G) : 1;
    const int64_t c0 = (int64_t)blockIdx.x * cols;
#pragma unroll
    for (int k = 0; k < kB / kThreads; ++k) {
        const int e = threadIdx.x + k * kThreads;
        const int t = e / cols, c = e - t * cols;
        cp_async8(sm + e, job.z32 + (int64_t)t * kB + c0 + c);
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    __syncthreads();
    column_stages<float2, true>(sm, G, cols, c0, tcol);
    const double slack = job_slack(job, parts);
    const int64_t n = job.n, max_lag = job.biggest - 1;
    float v[16];
    int32_t key[16];
#pragma unroll
    for (int k = 0; k < kB / kThreads; ++k) {
        const int e = threadIdx.x + k * kThreads;
        const int t = e / cols, c = e - t * cols;
        const int64_t i = (int64_t)t * kB + c0 + c;
        v[k] = fabsf(sm[e].x);
        key[k] = (int32_t)lag_key(i, n, max_lag);
        if (job.corr_out) job.corr_out[i] = sm[e].x;
    }
    block_nominate(v, key, slack, job.cands + blockIdx.x);
}

// Pass 3 of the f32 search, register form (4 <= G <= 11). Four CTAs an SM
// (64 registers, no spills; 32 KB of exchange buffer each): the pass reads
// its 4096 points at once and then only computes, so more resident CTAs keep
// more loads in flight.
template <int G>
__global__ void __launch_bounds__(kThreads, 4) inv_columns_reg_nominate(const LagJob *__restrict__ jobs,
                                                                     const float2 *__restrict__ tcol, int parts) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2 *sm = reinterpret_cast<float2 *>(smem_raw);
    constexpr int R = 1 << G, cols = kB >> G;
    const LagJob job = jobs[blockIdx.y];
    const int c = threadIdx.x % cols, q = threadIdx.x / cols;
    const int64_t col = (int64_t)blockIdx.x * cols + c;
    float2 x[16];
    if (G > 4) {
#pragma unroll
        for (int m = 0; m < 16; ++m) x[m] = job.z32[(int64_t)row_t(q, m) * kB + col];
        column_tail<float2, G, true>(x, G > 8 ? 8 : 4, tcol, col);
#pragma unroll
        for (int m = 0; m < 16; ++m) sm[row_t(q, m) * cols + c] = x[m];
        __syncthreads();
        if (G > 8) {
            constexpr int s = R / 256 > 0 ? R / 256 : 1;
#pragma unroll
            for (int m = 0; m < 16; ++m) x[m] = sm[row_b<G>(q, m) * cols + c];
            column_group4<float2, G, true>(x, 4, s, q % s, tcol, col);
#pragma unroll
            for (int m = 0; m < 16; ++m) sm[row_b<G>(q, m) * cols + c] = x[m];
            __syncthreads();
        }
#pragma unroll
        for (int m = 0; m < 16; ++m) x[m] = sm[row_a<G>(q, m) * cols + c];
    } else {
#pragma unroll
        for (int m = 0; m < 16; ++m) x[m] = job.z32[(int64_t)row_a<G>(q, m) * kB + col];
    }
    column_group4<float2, G, true>(x, 0, R / 16, q, tcol, col);
    const double slack = job_slack(job, parts);
    const int64_t n = job.n, max_lag = job.biggest - 1;
    float v[16];
    int32_t key[16];
#pragma unroll
    for (int m = 0; m < 16; ++m) {
        const int64_t i = (int64_t)row_a<G>(q, m) * kB + col;
        v[m] = fabsf(x[m].x);
        key[m] = (int32_t)lag_key(i, n, max_lag);
        if (job.corr_out) job.corr_out[i] = x[m].x;
    }
    block_nominate(v, key, slack, job.cands + blockIdx.x);
}

// n <= 4096: the whole f32 search's transform and nomination in one CTA.
template <bool RAW>
__global__ void __launch_bounds__(kThreads) small_lag32(const LagJob *__restrict__ jobs, const float2 *__restrict__ tw) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2 *sm = reinterpret_cast<float2 *>(smem_raw);
    const LagJob job = jobs[blockIdx.y];
    const int B = (int)job.n;
    EnvParams pa{}, pb{};
    if (!RAW) {
        pa = env_params(job.a, job.stats_a);
        pb = env_params(job.b, job.stats_b);
    }
    double ea = 0.0, eb = 0.0;
    for (int u = threadIdx.x; u < B; u += blockDim.x) sm[u] = pack_point<float2, RAW>(job, pa, pb, u, ea, eb);
    ea = block_sum(ea);
    eb = block_sum(eb);
    if (threadIdx.x == 0) job.energy[0] = make_double2(ea, eb);
    __syncthreads();
    blocks_dif<float2>(sm, nullptr, B, tw);
    for (int i = threadIdx.x; i < (B > 1 ? B / 2 : 1); i += blockDim.x) {
        if (i == 0) {
            sm[0] = cross_term(sm[0], sm[0]);
            if (B > 1) sm[1] = cross_term(sm[1], sm[1]);
            continue;
        }
        const int p = 1 << (31 - __clz(i));
        const int h = 2 * p;
        const int a = i + p, b = 3 * h - 1 - a;
        const float2 za = sm[a], zb = sm[b];
        sm[a] = cross_term(za, zb);
        sm[b] = cross_term(zb, za);
    }
    __syncthreads();
    blocks_dit<float2>(sm, nullptr, B, tw);
    const double slack = job_slack(job, 1);
    const int64_t max_lag = job.biggest - 1;
    float v[16];
    int32_t key[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) {
        const int u = threadIdx.x + k * kThreads;
        key[k] = -1;
        v[k] = 0.f;
        if (u < B) {
            v[k] = fabsf(sm[u].x);
            key[k] = (int32_t)lag_key(u, B, max_lag);
            if (job.corr_out) job.corr_out[u] = sm[u].x;
        }
    }
    block_nominate(v, key, slack, job.cands);
}

// Nomination records of an approximate correlation supplied by the caller
// (approx = corr_out, n values, circular index order), 4096 values a CTA:
// the reference's refineLag input (src/xcorr.zig:278-300). grid (parts, 1).
__global__ void __launch_bounds__(kThreads) nominate_approx(const LagJob *__restrict__ jobs) {
    const LagJob job = jobs[0];
    const int64_t n = job.n, max_lag = job.biggest - 1;
    float v[16];
    int32_t key[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) {
        const int64_t i = (int64_t)blockIdx.x * kB + threadIdx.x + k * kThreads;
        key[k] = -1;
        v[k] = 0.f;
        if (i < n) {
            v[k] = fabsf(job.corr_out[i]);
            key[k] = (int32_t)lag_key(i, n, max_lag);
        }
    }
    block_nominate(v, key, job.slack_fixed, job.cands + blockIdx.x);
}

// The search's candidates: lags whose |Re| is within the slack of the
// largest (reference refineLag src/xcorr.zig:278-300), from the CTAs'
// records. Over kLagCandCap of them, or a CTA near the top whose own list
// overflowed, sets status 1 (the exact search decides). One CTA per job.
__global__ void __launch_bounds__(kThreads) pick_candidates(const LagJob *__restrict__ jobs, int parts) {
    const LagJob job = jobs[blockIdx.x];
    const double slack = job_slack(job, parts);
    float top = -INFINITY;
    for (int p = threadIdx.x; p < parts; p += blockDim.x) top = fmaxf(top, job.cands[p].top);
    top = block_max(top);
    const double floor = (double)top - slack;
    // the records at or above the floor (each holds at least one candidate,
    // its own maximum, so more than kLagCandCap of them is an overflow)
    __shared__ int count, over, nsel;
    __shared__ int sel[kLagCandCap];
    if (threadIdx.x == 0) count = 0, over = 0, nsel = 0;
    __syncthreads();
    for (int p = threadIdx.x; p < parts; p += blockDim.x) {
        if ((double)job.cands[p].top < floor) continue;
        const int k = atomicAdd(&nsel, 1);
        if (job.cands[p].count > kLagCandCap || k >= kLagCandCap)
            over = 1;
        else
            sel[k] = p;
    }
    __syncthreads();
    // a warp per record, its lanes over the record's candidates
    if (!over) {
        const int lane = threadIdx.x & 31, warps = blockDim.x >> 5;
        for (int r = threadIdx.x >> 5; r < nsel; r += warps) {
            const LagCands &c = job.cands[sel[r]];
            for (int i = lane; i < c.count; i += 32) {
                if ((double)c.v[i] < floor) continue;
                const int k = atomicAdd(&count, 1);
                if (k < kLagCandCap) job.cand_key[k] = c.key[i];
            }
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const int bad = over || count > kLagCandCap || count == 0;
        *job.status = bad;
        *job.ncand = bad ? 0 : count;
    }
}

constexpr int kRescoreChunk = 4096;  // b samples per rescoring CTA
constexpr int kRescoreSpan = 1024;   // widest candidate lag range staged with a chunk

// Partial dot products sum_j a[j + lag] b[j] of every candidate lag over
// this CTA's chunk of b (reference dotAtLag src/xcorr.zig:328-340; the
// summation order is this kernel's, fixed), of the envelopes (or raw
// signals), in f64: each thread adds its 16 products in order, the warps
// reduce by shuffles and the 8 warp sums are added in order. When the
// candidates lie within kRescoreSpan lags of each other (near-maxima of one
// peak, the usual case) the envelope of a over the chunk's window and of b
// over the chunk are formed once, into shared memory and registers, and
// every candidate reads them; otherwise each candidate takes its own pass,
// forming the values it needs. grid (chunks, jobs).
template <bool RAW>
__global__ void __launch_bounds__(kThreads) rescore_candidates(const LagJob *__restrict__ jobs, int nchunks) {
    __shared__ double win[kRescoreChunk + kRescoreSpan];
    __shared__ double part[kLagCandCap][kThreads / 32];
    __shared__ int32_t keys[kLagCandCap];
    constexpr int kPer = kRescoreChunk / kThreads;
    const LagJob job = jobs[blockIdx.y];
    if (*job.status != 0) return;
    const int count = *job.ncand;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    EnvParams pa{}, pb{};
    if (!RAW) {
        pa = env_params(job.a, job.stats_a);
        pb = env_params(job.b, job.stats_b);
    }
    const int64_t max_lag = job.biggest - 1;
    const int64_t j0 = (int64_t)blockIdx.x * kRescoreChunk;
    if (threadIdx.x < count) keys[threadIdx.x] = job.cand_key[threadIdx.x];
    __syncthreads();
    int kmin = INT32_MAX, kmax = INT32_MIN;
    for (int c = 0; c < count; ++c) {
        kmin = min(kmin, keys[c]);
        kmax = max(kmax, keys[c]);
    }
    // a warp's 32 partial sums, in lane order by halves, into lane 0
    auto warp_sum = [](double v) {
        for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
        return v;
    };
    if (count > 0 && kmax - kmin <= kRescoreSpan) {
        const int64_t ws = j0 + (int64_t)kmin - max_lag;  // a index of win[0]
        const int wlen = kRescoreChunk + (kmax - kmin);
        // a's stored samples over the window by asynchronous copies (all in
        // flight at once, zeros outside them), b's by plain loads meanwhile
        const double *guard = job.rescore;
        for (int e = threadIdx.x; e < wlen; e += kThreads) {
            const int64_t ia = ws + e, ja = ia - job.a.head;
            const bool in = ia >= 0 && ia < job.a.len && (uint64_t)ja < (uint64_t)job.a.avail;
            cp_async8z(win + e, in ? job.a.base + ja : guard, in);
        }
        asm volatile("cp.async.commit_group;\n" ::: "memory");
        double y[kPer];
#pragma unroll
        for (int k = 0; k < kPer; ++k) {
            const int64_t j = j0 + threadIdx.x + k * kThreads;
            y[k] = j < job.b.len ? vsig_at(job.b, j) : 0.0;
        }
        if (!RAW) {
#pragma unroll
            for (int k = 0; k < kPer; ++k) {
                const int64_t j = j0 + threadIdx.x + k * kThreads;
                if (j < job.b.len) y[k] = env_of(y[k], pb, j);
            }
        }
        asm volatile("cp.async.wait_all;\n" ::: "memory");
        // each thread forms the envelope of the window entries it copied
        for (int e = threadIdx.x; e < wlen; e += kThreads) {
            const int64_t ia = ws + e;
            if (ia < 0 || ia >= job.a.len)
                win[e] = 0.0;
            else if (!RAW)
                win[e] = env_of(win[e], pa, ia);
        }
        __syncthreads();
        for (int c = 0; c < count; ++c) {
            const double *w = win + (keys[c] - kmin) + threadIdx.x;
            double acc = 0.0;
#pragma unroll
            for (int k = 0; k < kPer; ++k) acc += w[k * kThreads] * y[k];
            acc = warp_sum(acc);
            if (lane == 0) part[c][warp] = acc;
        }
    } else {
        for (int c = 0; c < count; ++c) {
            const int64_t lag = (int64_t)keys[c] - max_lag;
            double acc = 0.0;
            for (int k = 0; k < kPer; ++k) {
                const int64_t j = j0 + threadIdx.x + k * kThreads, ia = j + lag;
                if (j < job.b.len && ia >= 0 && ia < job.a.len) {
                    const double y = RAW ? vsig_at(job.b, j) : env_at(job.b, pb, j);
                    const double x = RAW ? vsig_at(job.a, ia) : env_at(job.a, pa, ia);
                    acc += x * y;
                }
            }
            acc = warp_sum(acc);
            if (lane == 0) part[c][warp] = acc;
        }
    }
    __syncthreads();
    if (threadIdx.x < count) {
        double t = 0.0;
#pragma unroll
        for (int w = 0; w < kThreads / 32; ++w) t += part[threadIdx.x][w];
        job.rescore[(int64_t)threadIdx.x * nchunks + blockIdx.x] = t;
    }
}

// Rescored candidates closer than this fraction of |a|^2 + |b|^2 are a tie
// as far as the two searches can tell: each search's rounding error is
// below 1e-13 of it, real lags' differences are far above.
constexpr double kTieMargin = 1e-10;

// The best |dot| so far (value, lag key) and the second best value.
struct Top2 {
    Best first;
    double second;
};
__device__ inline bool prefers(Best x, Best y) { return x.v > y.v || (x.v == y.v && x.key < y.key); }
__device__ inline Top2 merge(Top2 a, Top2 b) {
    if (prefers(b.first, a.first)) return Top2{b.first, fmax(b.second, a.first.v)};
    return Top2{a.first, fmax(a.second, b.first.v)};
}

// The first maximum of |dot| in ascending lag (reference rescore
// src/xcorr.zig:311-325). Where the two best are within kTieMargin (a
// periodic signal's equal peaks), which of them the exact search picks is
// decided by its own rounding, so the job is left to it (status 1). One CTA
// per job: a warp per candidate adds its chunk partials (lanes strided, then
// a fixed shuffle order); parts: the job's energy records.
__global__ void __launch_bounds__(kThreads) pick_rescored(const LagJob *__restrict__ jobs, int njobs, int nchunks,
                                                          int parts) {
    const LagJob job = jobs[blockIdx.x];
    if (*job.status != 0) return;
    const int count = *job.ncand;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, warps = blockDim.x >> 5;
    double e = 0.0;
    for (int p = threadIdx.x; p < parts; p += blockDim.x) e += job.energy[p].x + job.energy[p].y;
    e = block_sum(e);
    __shared__ double dot[kLagCandCap];
    for (int c = warp; c < count; c += warps) {
        double d = 0.0;
        for (int k = lane; k < nchunks; k += 32) d += job.rescore[(int64_t)c * nchunks + k];
        for (int off = 16; off > 0; off >>= 1) d += __shfl_down_sync(0xffffffffu, d, off);
        if (lane == 0) dot[c] = d;
    }
    __syncthreads();
    if (warp != 0) return;
    Top2 top{Best{-INFINITY, INT64_MAX}, -INFINITY};
    for (int c = lane; c < count; c += 32) top = merge(top, Top2{Best{fabs(dot[c]), (int64_t)job.cand_key[c]}, -INFINITY});
    for (int off = 16; off > 0; off >>= 1) {
        Top2 o{Best{__shfl_down_sync(0xffffffffu, top.first.v, off), __shfl_down_sync(0xffffffffu, top.first.key, off)},
               __shfl_down_sync(0xffffffffu, top.second, off)};
        top = merge(top, o);
    }
    if (lane == 0) {
        if (top.first.v - top.second <= kTieMargin * e)
            *job.status = 1;
        else
            *job.lag_out = top.first.key - (job.biggest - 1);
    }
}

}  // namespace

void lag_init_attributes() {
    const int one = kB * (int)sizeof(double2);
    cudaFuncSetAttribute(fwd_columns<double2, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, one);
    cudaFuncSetAttribute(fwd_columns<double2, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, one);
    cudaFuncSetAttribute(inv_columns_argmax, cudaFuncAttributeMaxDynamicSharedMemorySize, one);
#define VQB_COLS_ATTR(GG)                                                                                 \
    cudaFuncSetAttribute(fwd_columns_reg<double2, GG, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, one);  \
    cudaFuncSetAttribute(fwd_columns_reg<double2, GG, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, one); \
    cudaFuncSetAttribute(fwd_columns_staged<double2, GG, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, one); \
    cudaFuncSetAttribute(fwd_columns_staged<double2, GG, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, one); \
    cudaFuncSetAttribute(fwd_columns_staged<float2, GG, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, one); \
    cudaFuncSetAttribute(fwd_columns_staged<float2, GG, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, one); \
    cudaFuncSetAttribute(inv_columns_reg<GG>, cudaFuncAttributeMaxDynamicSharedMemorySize, one);
    VQB_COLS_ATTR(4)
    VQB_COLS_ATTR(5)
    VQB_COLS_ATTR(6)
    VQB_COLS_ATTR(7)
    VQB_COLS_ATTR(8)
    VQB_COLS_ATTR(9)
    VQB_COLS_ATTR(10)
    VQB_COLS_ATTR(11)
#undef VQB_COLS_ATTR
    cudaFuncSetAttribute(small_lag<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, one);
    cudaFuncSetAttribute(small_lag<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, one);
    cudaFuncSetAttribute(middle_blocks<double2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)(2 * kPadB * sizeof(double2)));
}

bool fused_lag_supported(int64_t n) { return n >= 1 && n <= ((int64_t)kB << 12); }

size_t fused_lag_parts(int64_t n) {
    if (n <= kB) return 1;
    int G = 0;
    for (int64_t r = n / kB; r > 1; r >>= 1) ++G;
    const int cols = (kB >> G) > 0 ? (kB >> G) : 1;
    return (size_t)(kB / cols);
}

size_t column_twiddle_count(int64_t n) { return n <= kB ? 0 : (size_t)(n - kB); }

size_t block_stage_twiddle_count() { return kB - 1; }

void fill_block_stage_twiddles(const double2 *block, double2 *out) {
    // out[(4096 - S) + k] = W_S^k = block[k * 4096 / S], spans S = 4096 .. 2
    for (int S = kB; S >= 2; S >>= 1)
        for (int k2 = 0; k2 < S / 2; ++k2) out[(kB - S) + k2] = block[(size_t)k2 * (kB / S)];
}

void fill_column_twiddles(const double2 *top, int64_t n, double2 *out) {
    if (n <= kB) return;
    int G = 0;
    for (int64_t r = n / kB; r > 1; r >>= 1) ++G;
    const int64_t R = (int64_t)1 << G;
    size_t k = 0;
    for (int l = 0; l < G; ++l)
        for (int64_t m = 0; m < (R >> (l + 1)); ++m)
            for (int64_t col = 0; col < kB; ++col) out[k++] = top[(m * kB + col) << l];
}

bool fused_lag_register_columns(int64_t n) { return n >= ((int64_t)kB << 4) && n <= ((int64_t)kB << 11); }

void launch_fused_lag(const LagJob *d_jobs, int njobs, int64_t n, bool raw, const double2 *tcol,
                      const double2 *tw_block, const double2 *tst, double *pv, int64_t *pk, int columns,
                      cudaStream_t s) {
    if (njobs <= 0) return;
    const size_t one = (size_t)kB * sizeof(double2);
    if (n <= kB) {
        const size_t smem = (size_t)n * sizeof(double2);
        if (raw)
            small_lag<true><<<dim3(1, (unsigned)njobs), kThreads, smem, s>>>(d_jobs, tw_block, pv, pk);
        else
            small_lag<false><<<dim3(1, (unsigned)njobs), kThreads, smem, s>>>(d_jobs, tw_block, pv, pk);
        pick_lag<<<(njobs + 3) / 4, 128, 0, s>>>(d_jobs, njobs, pv, pk, 1);
        launch_counter() += 2;
        return;
    }
    int G = 0;
    for (int64_t r = n / kB; r > 1; r >>= 1) ++G;
    const int parts = (int)fused_lag_parts(n);
    const int64_t nblk = n / kB;
    const dim3 grid((unsigned)parts, (unsigned)njobs);
    const size_t reg_smem = G > 4 ? one : 0;
    // 0: the shared-memory column passes; 1: register passes; 2: register
    // passes with the forward samples staged in shared memory
    const int Gr = columns == 1 || columns == 2 ? G : 0;
    const bool staged = columns == 2;
    switch (Gr) {
#define VQB_COLS(GG)                                                                                       \
    case GG:                                                                                               \
        if (staged && raw)                                                                                 \
            fwd_columns_staged<double2, GG, true><<<grid, kThreads, one, s>>>(d_jobs, tcol);               \
        else if (staged)                                                                                   \
            fwd_columns_staged<double2, GG, false><<<grid, kThreads, one, s>>>(d_jobs, tcol);              \
        else if (raw)                                                                                      \
            fwd_columns_reg<double2, GG, true><<<grid, kThreads, reg_smem, s>>>(d_jobs, tcol);             \
        else                                                                                               \
            fwd_columns_reg<double2, GG, false><<<grid, kThreads, reg_smem, s>>>(d_jobs, tcol);            \
        break;
        VQB_COLS(4)
        VQB_COLS(5)
        VQB_COLS(6)
        VQB_COLS(7)
        VQB_COLS(8)
        VQB_COLS(9)
        VQB_COLS(10)
        VQB_COLS(11)
#undef VQB_COLS
    default:
        if (raw)
            fwd_columns<double2, true><<<grid, kThreads, one, s>>>(d_jobs, G, tcol);
        else
            fwd_columns<double2, false><<<grid, kThreads, one, s>>>(d_jobs, G, tcol);
    }
    middle_blocks<double2><<<dim3((unsigned)(nblk / 2 + 1), (unsigned)njobs), kMidThreads, 2 * kPadB * sizeof(double2), s>>>(
        d_jobs, tst);
    switch (Gr) {
#define VQB_COLS(GG)                                                                                       \
    case GG:                                                                                               \
        inv_columns_reg<GG><<<grid, kThreads, reg_smem, s>>>(d_jobs, tcol, pv, pk, parts);                \
        break;
        VQB_COLS(4)
        VQB_COLS(5)
        VQB_COLS(6)
        VQB_COLS(7)
        VQB_COLS(8)
        VQB_COLS(9)
        VQB_COLS(10)
        VQB_COLS(11)
#undef VQB_COLS
    default:
        inv_columns_argmax<<<grid, kThreads, one, s>>>(d_jobs, G, tcol, pv, pk, parts);
    }
    pick_lag<<<(njobs + 3) / 4, 128, 0, s>>>(d_jobs, njobs, pv, pk, parts);
    launch_counter() += 4;
}

void launch_refine_approx(const LagJob *d_job, int64_t n, int nchunks, cudaStream_t s) {
    const int parts = (int)((n + kB - 1) / kB);
    nominate_approx<<<parts, kThreads, 0, s>>>(d_job);
    pick_candidates<<<1, kThreads, 0, s>>>(d_job, parts);
    rescore_candidates<true><<<dim3((unsigned)nchunks, 1), kThreads, 0, s>>>(d_job, nchunks);
    pick_rescored<<<1, kThreads, 0, s>>>(d_job, 1, nchunks, parts);
    launch_counter() += 4;
}

void lag32_init_attributes() {
    const int one = kB * (int)sizeof(float2);
    cudaFuncSetAttribute(fwd_columns<float2, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, one);
    cudaFuncSetAttribute(fwd_columns<float2, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, one);
    cudaFuncSetAttribute(inv_columns_nominate, cudaFuncAttributeMaxDynamicSharedMemorySize, one);
    cudaFuncSetAttribute(small_lag32<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, one);
    cudaFuncSetAttribute(small_lag32<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, one);
    cudaFuncSetAttribute(middle_blocks<float2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)(2 * kPadB * sizeof(float2)));
}

size_t lag32_parts(int64_t n) { return n <= kB ? 1 : fused_lag_parts(n); }

int lag32_rescore_chunks(int64_t max_b_len) {
    return (int)std::max<int64_t>(1, (max_b_len + kRescoreChunk - 1) / kRescoreChunk);
}

void launch_lag32(const LagJob *d_jobs, int njobs, int64_t n, bool raw, const float2 *tcol, const float2 *tw_block,
                  const float2 *tst, int nchunks, int columns, cudaStream_t s) {
    if (njobs <= 0) return;
    const int parts = (int)lag32_parts(n);
    if (n <= kB) {
        const size_t smem = (size_t)n * sizeof(float2);
        if (raw)
            small_lag32<true><<<dim3(1, (unsigned)njobs), kThreads, smem, s>>>(d_jobs, tw_block);
        else
            small_lag32<false><<<dim3(1, (unsigned)njobs), kThreads, smem, s>>>(d_jobs, tw_block);
        launch_counter() += 1;
    } else {
        int G = 0;
        for (int64_t r = n / kB; r > 1; r >>= 1) ++G;
        const int64_t nblk = n / kB;
        const dim3 grid((unsigned)parts, (unsigned)njobs);
        const size_t one = (size_t)kB * sizeof(float2);
        const size_t reg_smem = G > 4 ? one : 0;
        const size_t stage_smem = (size_t)kB * sizeof(double2);
        // as launch_fused_lag: 1 register passes, 2 with staged forward samples
        const int Gr = fused_lag_register_columns(n) && columns != 0 ? G : 0;
        const bool staged = columns == 2;
        switch (Gr) {
#define VQB_COLS32(GG)                                                                                     \
    case GG:                                                                                               \
        if (staged && raw)                                                                                 \
            fwd_columns_staged<float2, GG, true><<<grid, kThreads, stage_smem, s>>>(d_jobs, tcol);         \
        else if (staged)                                                                                   \
            fwd_columns_staged<float2, GG, false><<<grid, kThreads, stage_smem, s>>>(d_jobs, tcol);        \
        else if (raw)                                                                                      \
            fwd_columns_reg<float2, GG, true><<<grid, kThreads, reg_smem, s>>>(d_jobs, tcol);              \
        else                                                                                               \
            fwd_columns_reg<float2, GG, false><<<grid, kThreads, reg_smem, s>>>(d_jobs, tcol);             \
        break;
            VQB_COLS32(4)
            VQB_COLS32(5)
            VQB_COLS32(6)
            VQB_COLS32(7)
            VQB_COLS32(8)
            VQB_COLS32(9)
            VQB_COLS32(10)
            VQB_COLS32(11)
#undef VQB_COLS32
        default:
            if (raw)
                fwd_columns<float2, true><<<grid, kThreads, one, s>>>(d_jobs, G, tcol);
            else
                fwd_columns<float2, false><<<grid, kThreads, one, s>>>(d_jobs, G, tcol);
        }
        middle_blocks<float2><<<dim3((unsigned)(nblk / 2 + 1), (unsigned)njobs), kMidThreads,
                                2 * kPadB * sizeof(float2), s>>>(d_jobs, tst);
        switch (Gr) {
#define VQB_COLS32(GG)                                                                                     \
    case GG:                                                                                               \
        inv_columns_reg_nominate<GG><<<grid, kThreads, reg_smem, s>>>(d_jobs, tcol, parts);               \
        break;
            VQB_COLS32(4)
            VQB_COLS32(5)
            VQB_COLS32(6)
            VQB_COLS32(7)
            VQB_COLS32(8)
            VQB_COLS32(9)
            VQB_COLS32(10)
            VQB_COLS32(11)
#undef VQB_COLS32
        default:
            inv_columns_nominate<<<grid, kThreads, one, s>>>(d_jobs, G, tcol, parts);
        }
        launch_counter() += 3;
    }
    pick_candidates<<<njobs, kThreads, 0, s>>>(d_jobs, parts);
    if (raw)
        rescore_candidates<true><<<dim3((unsigned)nchunks, (unsigned)njobs), kThreads, 0, s>>>(d_jobs, nchunks);
    else
        rescore_candidates<false><<<dim3((unsigned)nchunks, (unsigned)njobs), kThreads, 0, s>>>(d_jobs, nchunks);
    pick_rescored<<<njobs, kThreads, 0, s>>>(d_jobs, njobs, nchunks, parts);
    launch_counter() += 3;
}

}  // namespace vqb
