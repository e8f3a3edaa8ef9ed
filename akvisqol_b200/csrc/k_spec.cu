// Spectrogram preparation (reference src/spectrogram.zig:14-80): dB with an
// absolute -45 dB floor, a per-frame floor 45 dB under the frame's peak over
// both spectrograms, then the joint minimum subtracted.
//
// Two launches over all pairs: dB values and per-frame floors with one
// warp per band and 32 frames per CTA (plus a partial joint minimum per
// CTA), then the joint minimum subtracted. Max and min are exact in any
// order, so the reductions match the CPU's loops bit for bit.
//
// log10 follows fdlibm's e_log10.c (Sun Microsystems), the formula the
// CPU's glibc log10 evaluates: with x = 2^k * m, y = k (+1 below 1),
// log10(x) = (y*log10_2lo + ivln10*log(m)) + y*log10_2hi, evaluated in that
// order without FMA. The natural log is CUDA's; results agree with glibc
// to the last bit except where the two natural logs differ by an ulp.
#include <algorithm>
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

// Phase 1: one CTA per 32 frames of one spectrogram pair, one warp per
// band with its lanes along frames (coalesced rows). Each value's dB, the
// frame's floor (the maximum over both spectrograms' bands, a shared-memory
// reduction) and the floored values are formed in registers and written
// once; the CTA's minimum goes to part[job * nparts + blockIdx.x] (+inf
// when the CTA holds no frame of this pair). Max and min are exact in any
// order, so the results are the CPU loops' bit for bit.
constexpr int kPrepCols = 32;

__global__ void __launch_bounds__(1024) prep_db_kernel(const PrepJob *__restrict__ jobs, int nb,
                                                       double *__restrict__ part, int nparts) {
    __shared__ double colmax[32][kPrepCols + 1];
    __shared__ double floor_db[kPrepCols];
    __shared__ double wmin[32];
    const PrepJob job = jobs[blockIdx.y];
    const int b = threadIdx.x >> 5, j = threadIdx.x & 31;
    const int c = blockIdx.x * kPrepCols + j;
    const int nfr = job.nfr, nfd = job.nfd;
    const int minf = nfr < nfd ? nfr : nfd;
    double r = 0.0, d = 0.0;
    if (c < nfr) r = to_db(job.ref_in[(int64_t)b * nfr + c]);
    if (c < nfd) d = to_db(job.deg_in[(int64_t)b * nfd + c]);
    colmax[b][j] = c < minf ? dmax(r, d) : -INFINITY;
    __syncthreads();
    if (b == 0) {
        double m = -INFINITY;
        for (int k = 0; k < nb; ++k)
            if (colmax[k][j] > m) m = colmax[k][j];
        floor_db[j] = m - kRelFloor;
    }
    __syncthreads();
    double lo = INFINITY;
    if (c < minf) {
        const double f = floor_db[j];
        if (r < f) r = f;
        if (d < f) d = f;
    }
    if (c < nfr) {
        job.ref[(int64_t)b * nfr + c] = r;
        if (r < lo) lo = r;
    }
    if (c < nfd) {
        job.deg[(int64_t)b * nfd + c] = d;
        if (d < lo) lo = d;
    }
    for (int off = 16; off > 0; off >>= 1) {
        const double o = __shfl_down_sync(0xffffffffu, lo, off);
        if (o < lo) lo = o;
    }
    if (j == 0) wmin[b] = lo;
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = INFINITY;
        for (int k = 0; k < nb; ++k)
            if (wmin[k] < m) m = wmin[k];
        part[(int64_t)blockIdx.y * nparts + blockIdx.x] = m;
    }
}

// Phase 2: the joint minimum (reference src/spectrogram.zig:56-66) from the
// phase-1 parts, subtracted from every value of both spectrograms.
__global__ void __launch_bounds__(256) prep_sub_kernel(const PrepJob *__restrict__ jobs, int nb,
                                                       const double *__restrict__ part, int nparts) {
    __shared__ double lo_s;
    const PrepJob job = jobs[blockIdx.y];
    if (threadIdx.x < 32) {
        double lo = INFINITY;
        for (int k = threadIdx.x; k < nparts; k += 32) {
            const double v = part[(int64_t)blockIdx.y * nparts + k];
            if (v < lo) lo = v;
        }
        for (int off = 16; off > 0; off >>= 1) {
            const double o = __shfl_down_sync(0xffffffffu, lo, off);
            if (o < lo) lo = o;
        }
        if (threadIdx.x == 0) lo_s = lo;
    }
    __syncthreads();
    const double lo = lo_s;
    const int64_t nr = (int64_t)nb * job.nfr, nd = (int64_t)nb * job.nfd;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nr; e += stride) job.ref[e] -= lo;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nd; e += stride) job.deg[e] -= lo;
}

__global__ void log10_kernel(const double *x, int64_t n, double *out) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = 10.0 * vq_log10(x[i]);
}

}  // namespace

size_t prep_scratch_count(int njobs, int max_frames) {
    return (size_t)njobs * (size_t)((max_frames + kPrepCols - 1) / kPrepCols);
}

void launch_prep(const PrepJob *d_jobs, int njobs, int nb, int max_frames, double *d_scratch, cudaStream_t s) {
    if (njobs <= 0 || max_frames <= 0) return;
    const int nparts = (max_frames + kPrepCols - 1) / kPrepCols;
    prep_db_kernel<<<dim3((unsigned)nparts, (unsigned)njobs), 32 * nb, 0, s>>>(d_jobs, nb, d_scratch, nparts);
    // about four values per thread of the larger spectrogram
    const int sub_blocks = std::max(1, std::min(64, (nb * max_frames + 1023) / 1024));
    prep_sub_kernel<<<dim3((unsigned)sub_blocks, (unsigned)njobs), 256, 0, s>>>(d_jobs, nb, d_scratch, nparts);
    launch_counter() += 2;
}

void launch_log10(const double *x, int64_t n, double *out, cudaStream_t s) {
    int64_t blocks = (n + 255) / 256;
    if (blocks > 4096) blocks = 4096;
    if (blocks < 1) blocks = 1;
    log10_kernel<<<(unsigned)blocks, 256, 0, s>>>(x, n, out);
    launch_counter() += 1;
}

}  // namespace vqb
