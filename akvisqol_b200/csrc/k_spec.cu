// Spectrogram preparation (reference src/spectrogram.zig:14-80): dB with an
// absolute -45 dB floor, a per-frame floor 45 dB under the frame's peak over
// both spectrograms, then the joint minimum subtracted.
//
// One CTA per spectrogram pair. A thread owns whole frames (columns), so
// the dB values and the per-frame floor need no exchange; max and min are
// exact in any order, so the block reductions match the CPU's loops.
//
// log10 follows fdlibm's e_log10.c (Sun Microsystems), the formula the
// CPU's glibc log10 evaluates: with x = 2^k * m, y = k (+1 below 1),
// log10(x) = (y*log10_2lo + ivln10*log(m)) + y*log10_2hi, evaluated in that
// order without FMA. The natural log is CUDA's; results agree with glibc
// to the last bit except where the two natural logs differ by an ulp.
#include <cfloat>

#include "device.cuh"
#include "kernels.h"

namespace vqb {

__device__ double vq_log10(double x) {
    // fdlibm e_log10.c constants.
    const double two54 = 1.80143985094819840000e+16;
    const double ivln10 = 4.34294481903251816668e-01;
    const double log10_2hi = 3.01029995663611771306e-01;
    const double log10_2lo = 3.69423907715893078616e-13;
    long long u = __double_as_longlong(x);
    int hx = (int)(u >> 32);
    const unsigned lx = (unsigned)u;
    int k = 0;
    if (hx < 0x00100000) {
        if (((hx & 0x7fffffff) | lx) == 0) return -INFINITY;
        if (hx < 0) return __longlong_as_double(0x7ff8000000000000LL);
        k -= 54;
        x *= two54;
        u = __double_as_longlong(x);
        hx = (int)(u >> 32);
    }
    if (hx >= 0x7ff00000) return x + x;
    k += (hx >> 20) - 1023;
    const int i = (int)(((unsigned)k & 0x80000000u) >> 31);
    hx = (hx & 0x000fffff) | ((0x3ff - i) << 20);
    const double y = (double)(k + i);
    x = __longlong_as_double(((long long)(unsigned)hx << 32) | (long long)(unsigned)u);
    const double z = y * log10_2lo + ivln10 * log(x);
    return z + y * log10_2hi;
}

namespace {

constexpr double kAbsFloor = -45.0;
constexpr double kRelFloor = 45.0;

// convertToDbAndRaiseFloor's per-value step (reference src/spectrogram.zig:14-20).
// Zig's @max is IEEE maxNum (a NaN operand yields the other), as fmax.
__device__ inline double to_db(double v) {
    const double sample = v == 0.0 ? DBL_EPSILON : fabs(v);
    const double db = 10.0 * vq_log10(sample);
    return fmax(db, kAbsFloor);
}

__device__ inline double dmax(double a, double b) { return fmax(a, b); }

__global__ void __launch_bounds__(256) prep_kernel(const PrepJob *__restrict__ jobs, int nb) {
    const PrepJob job = jobs[blockIdx.x];
    const int nfr = job.nfr, nfd = job.nfd;
    const int minf = nfr < nfd ? nfr : nfd;
    const int maxf = nfr > nfd ? nfr : nfd;
    double lo = INFINITY;
    for (int c = threadIdx.x; c < maxf; c += blockDim.x) {
        double col_max = -INFINITY;
        for (int b = 0; b < nb; ++b) {
            double r = 0, d = 0;
            if (c < nfr) job.ref[(int64_t)b * nfr + c] = r = to_db(job.ref_in[(int64_t)b * nfr + c]);
            if (c < nfd) job.deg[(int64_t)b * nfd + c] = d = to_db(job.deg_in[(int64_t)b * nfd + c]);
            if (c < minf) {
                const double m = dmax(r, d);
                if (m > col_max) col_max = m;
            }
        }
        if (c < minf) {
            const double floor_db = col_max - kRelFloor;
            for (int b = 0; b < nb; ++b) {
                double &rv = job.ref[(int64_t)b * nfr + c];
                if (rv < floor_db) rv = floor_db;
                double &dv = job.deg[(int64_t)b * nfd + c];
                if (dv < floor_db) dv = floor_db;
            }
        }
        for (int b = 0; b < nb; ++b) {
            if (c < nfr && job.ref[(int64_t)b * nfr + c] < lo) lo = job.ref[(int64_t)b * nfr + c];
            if (c < nfd && job.deg[(int64_t)b * nfd + c] < lo) lo = job.deg[(int64_t)b * nfd + c];
        }
    }
    // Joint minimum (reference src/spectrogram.zig:56-66).
    for (int off = 16; off > 0; off >>= 1) {
        const double o = __shfl_down_sync(0xffffffffu, lo, off);
        if (o < lo) lo = o;
    }
    __shared__ double wmin[8];
    if ((threadIdx.x & 31) == 0) wmin[threadIdx.x >> 5] = lo;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w)
            if (wmin[w] < lo) lo = wmin[w];
        wmin[0] = lo;
    }
    __syncthreads();
    lo = wmin[0];
    for (int64_t e = threadIdx.x; e < (int64_t)nb * nfr; e += blockDim.x) job.ref[e] -= lo;
    for (int64_t e = threadIdx.x; e < (int64_t)nb * nfd; e += blockDim.x) job.deg[e] -= lo;
}

__global__ void log10_kernel(const double *x, int64_t n, double *out) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = 10.0 * vq_log10(x[i]);
}

}  // namespace

void launch_prep(const PrepJob *d_jobs, int njobs, int nb, cudaStream_t s) {
    if (njobs <= 0) return;
    prep_kernel<<<njobs, 256, 0, s>>>(d_jobs, nb);
    launch_counter() += 1;
}

void launch_log10(const double *x, int64_t n, double *out, cudaStream_t s) {
    int64_t blocks = (n + 255) / 256;
    if (blocks > 4096) blocks = 4096;
    if (blocks < 1) blocks = 1;
    log10_kernel<<<(unsigned)blocks, 256, 0, s>>>(x, n, out);
    launch_counter() += 1;
}

}  // namespace vqb
