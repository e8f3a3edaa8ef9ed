// FFT cross-correlation lag search in f64 (reference src/xcorr.zig:197-251,
// src/dsp/fft.zig:127-166).
//
// The lag is the argmax of |Re IFFT(cross spectrum)|. To give the CPU's lag
// on every input, the transform performs the very radix-2 butterflies of
// the reference's DIF forward / DIT inverse with the same twiddle values:
// any schedule of those butterflies gives identical bits, so only the
// schedule is ours. Large spans run as global passes of up to four fused
// stages (radix 16, one thread per 16-point group in registers); the last
// twelve stages of each 4096-point block run in shared memory. The cross
// spectrum is formed in bit-reversed order (no permutation pass), and the
// argmax keeps the reference's scan order: negative lags from the most
// negative, then 0, 1, ...; the first maximum wins.
#include "device.cuh"
#include "kernels.h"

namespace vqb {

namespace {

__device__ inline double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ inline double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
// cmul (reference src/dsp/fft.zig:181-183).
__device__ inline double2 cmul(double2 x, double2 w) {
    return make_double2(x.x * w.x - x.y * w.y, x.x * w.y + x.y * w.x);
}
// cmulConj (reference src/dsp/fft.zig:185-188).
__device__ inline double2 cmul_conj(double2 x, double2 w) {
    const double wi = -w.y;
    return make_double2(x.x * w.x - x.y * wi, x.x * wi + x.y * w.x);
}

// M fused stages on groups of R = 2^M points spaced q = S >> M apart; S is
// the largest span of the pass. DIF applies spans S, S/2, ...; DIT the
// reverse, ending at S. top[k] = W_n^k.
template <int M, bool DIT>
__global__ void __launch_bounds__(128) global_pass(double2 *__restrict__ z, int64_t n, int64_t S,
                                                   const double2 *__restrict__ top, int64_t job_stride) {
    constexpr int R = 1 << M;
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= (n >> M)) return;
    double2 *zz = z + (int64_t)blockIdx.y * job_stride;
    const int64_t q = S >> M;
    const int64_t blk = g / q, j = g - blk * q;
    const int64_t base = blk * S + j;
    double2 x[R];
#pragma unroll
    for (int t = 0; t < R; ++t) x[t] = zz[base + t * q];
    if (!DIT) {
#pragma unroll
        for (int l = 0; l < M; ++l) {
            const int h = R >> (l + 1);
            const int64_t stride = n / (S >> l);
#pragma unroll
            for (int t = 0; t < R; ++t) {
                if ((t % (2 * h)) < h) {
                    const double2 w = top[(j + (t % (2 * h)) * q) * stride];
                    const double2 a = x[t], b = x[t + h];
                    x[t] = cadd(a, b);
                    x[t + h] = cmul(csub(a, b), w);
                }
            }
        }
    } else {
#pragma unroll
        for (int li = 0; li < M; ++li) {
            const int l = M - 1 - li;
            const int h = R >> (l + 1);
            const int64_t stride = n / (S >> l);
#pragma unroll
            for (int t = 0; t < R; ++t) {
                if ((t % (2 * h)) < h) {
                    const double2 w = top[(j + (t % (2 * h)) * q) * stride];
                    const double2 a = x[t];
                    const double2 b = cmul_conj(x[t + h], w);
                    x[t] = cadd(a, b);
                    x[t + h] = csub(a, b);
                }
            }
        }
    }
#pragma unroll
    for (int t = 0; t < R; ++t) zz[base + t * q] = x[t];
}

// All stages with span <= B of each B-point block (B = min(n, 4096)) in
// shared memory, two stages per barrier (radix 4) with a radix-2 stage
// where the stage count is odd. tw[k] = W_B^k (k < B/2), so the span-s
// twiddle W_s^j is tw[j * B/s]: the same values as the full table.
__device__ inline void dif2(double2 *sm, int B, int s, const double2 *tw) {
    const int h = s >> 1, step = B / s;
    for (int bf = threadIdx.x; bf < (B >> 1); bf += blockDim.x) {
        const int blk = bf / h, j = bf - blk * h;
        const int i0 = blk * s + j;
        const double2 a = sm[i0], b = sm[i0 + h];
        sm[i0] = cadd(a, b);
        sm[i0 + h] = cmul(csub(a, b), tw[j * step]);
    }
}
__device__ inline void dit2(double2 *sm, int B, int s, const double2 *tw) {
    const int h = s >> 1, step = B / s;
    for (int bf = threadIdx.x; bf < (B >> 1); bf += blockDim.x) {
        const int blk = bf / h, j = bf - blk * h;
        const int i0 = blk * s + j;
        const double2 a = sm[i0];
        const double2 b = cmul_conj(sm[i0 + h], tw[j * step]);
        sm[i0] = cadd(a, b);
        sm[i0 + h] = csub(a, b);
    }
}
// Spans s then s/2 on 4-point groups spaced q = s/4 apart.
__device__ inline void dif4(double2 *sm, int B, int s, const double2 *tw) {
    const int q = s >> 2, st1 = B / s, st2 = 2 * st1;
    for (int g = threadIdx.x; g < (B >> 2); g += blockDim.x) {
        const int blk = g / q, j = g - blk * q;
        const int b0 = blk * s + j;
        double2 x0 = sm[b0], x1 = sm[b0 + q], x2 = sm[b0 + 2 * q], x3 = sm[b0 + 3 * q];
        double2 a = x0, b = x2;
        x0 = cadd(a, b);
        x2 = cmul(csub(a, b), tw[j * st1]);
        a = x1, b = x3;
        x1 = cadd(a, b);
        x3 = cmul(csub(a, b), tw[(j + q) * st1]);
        const double2 w = tw[j * st2];
        a = x0, b = x1;
        x0 = cadd(a, b);
        x1 = cmul(csub(a, b), w);
        a = x2, b = x3;
        x2 = cadd(a, b);
        x3 = cmul(csub(a, b), w);
        sm[b0] = x0, sm[b0 + q] = x1, sm[b0 + 2 * q] = x2, sm[b0 + 3 * q] = x3;
    }
}
// Spans s/2 then s.
__device__ inline void dit4(double2 *sm, int B, int s, const double2 *tw) {
    const int q = s >> 2, st1 = B / s, st2 = 2 * st1;
    for (int g = threadIdx.x; g < (B >> 2); g += blockDim.x) {
        const int blk = g / q, j = g - blk * q;
        const int b0 = blk * s + j;
        double2 x0 = sm[b0], x1 = sm[b0 + q], x2 = sm[b0 + 2 * q], x3 = sm[b0 + 3 * q];
        const double2 w = tw[j * st2];
        double2 a = x0, b = cmul_conj(x1, w);
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

template <bool DIT>
__global__ void __launch_bounds__(256) block_pass(double2 *__restrict__ z, int B, const double2 *__restrict__ tw,
                                                  int64_t job_stride) {
    extern __shared__ double2 sm[];
    double2 *zz = z + (int64_t)blockIdx.y * job_stride + (int64_t)blockIdx.x * B;
    for (int i = threadIdx.x; i < B; i += blockDim.x) sm[i] = zz[i];
    __syncthreads();
    int stages = 0;
    for (int r = B; r > 1; r >>= 1) ++stages;
    if (!DIT) {
        int s = B;
        for (; stages >= 2; stages -= 2, s >>= 2) {
            dif4(sm, B, s, tw);
            __syncthreads();
        }
        if (stages == 1) {
            dif2(sm, B, 2, tw);
            __syncthreads();
        }
    } else {
        int s = 2;
        if (stages & 1) {
            dit2(sm, B, 2, tw);
            __syncthreads();
            s = 8;
        } else {
            s = 4;
        }
        for (; s <= B; s <<= 2) {
            dit4(sm, B, s, tw);
            __syncthreads();
        }
    }
    for (int i = threadIdx.x; i < B; i += blockDim.x) zz[i] = sm[i];
}

// crossTerm (reference src/xcorr.zig:182-192).
__device__ inline double2 cross_term(double2 x, double2 zy) {
    const double2 y = make_double2(zy.x, -zy.y);
    const double2 sum = make_double2(x.x + y.x, x.y + y.y);
    const double2 dif_c = make_double2(x.x - y.x, -(x.y - y.y));
    const double2 idc = make_double2(-dif_c.y, dif_c.x);
    return make_double2(0.25 * (sum.x * idc.x - sum.y * idc.y), 0.25 * (sum.x * idc.y + sum.y * idc.x));
}

// In bit-reversed order Z[-k] pairs position a of block [h, 2h) with
// 3h-1-a; positions 0 and 1 pair with themselves (reference
// src/xcorr.zig:211-229). Thread i in [1, n/2) owns pair (i + p, 3h-1-a)
// with p = floor_pow2(i), h = 2p; thread 0 owns positions 0 and 1.
__global__ void __launch_bounds__(256) cross_kernel(double2 *__restrict__ z, int64_t n, int64_t job_stride) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (n >> 1) && !(i == 0 && n == 1)) return;
    double2 *zz = z + (int64_t)blockIdx.y * job_stride;
    if (i == 0) {
        zz[0] = cross_term(zz[0], zz[0]);
        if (n > 1) zz[1] = cross_term(zz[1], zz[1]);
        return;
    }
    const int64_t p = (int64_t)1 << (63 - __clzll(i));
    const int64_t h = 2 * p;
    const int64_t a = i + p, b = 3 * h - 1 - a;
    const double2 za = zz[a], zb = zz[b];
    zz[a] = cross_term(za, zb);
    zz[b] = cross_term(zb, za);
}

struct Best {
    double v;
    int64_t key;
};

__device__ inline Best better(Best a, Best b) {
    // Larger |corr|; on ties the earlier key (scan order). NaN never wins.
    if (b.v > a.v) return b;
    if (b.v == a.v && b.key < a.key) return b;
    return a;
}

// Keys k in [0, 2*max_lag] follow the CPU scan order; lag = k - max_lag.
// Position of key k: n - max_lag + k for k < max_lag, else k - max_lag.
__global__ void __launch_bounds__(256) argmax_partial(const double2 *__restrict__ z, const LagJob *__restrict__ jobs,
                                                      int64_t job_stride, double *pv, int64_t *pk, int parts) {
    const LagJob job = jobs[blockIdx.y];
    const double2 *zz = z + (int64_t)blockIdx.y * job_stride;
    const int64_t n = job.n, max_lag = job.biggest - 1;
    const int64_t nkeys = 2 * max_lag + 1;
    Best best{-INFINITY, INT64_MAX};
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nkeys; k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t pos = k < max_lag ? n - max_lag + k : k - max_lag;
        const double v = fabs(zz[pos].x);
        if (v > best.v) best = Best{v, k};
    }
    for (int off = 16; off > 0; off >>= 1) {
        Best o{__shfl_down_sync(0xffffffffu, best.v, off), __shfl_down_sync(0xffffffffu, best.key, off)};
        best = better(best, o);
    }
    __shared__ Best warp_best[8];
    if ((threadIdx.x & 31) == 0) warp_best[threadIdx.x >> 5] = best;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) best = better(best, warp_best[w]);
        pv[(int64_t)blockIdx.y * parts + blockIdx.x] = best.v;
        pk[(int64_t)blockIdx.y * parts + blockIdx.x] = best.key;
    }
}

__global__ void argmax_final(const LagJob *__restrict__ jobs, int njobs, const double *pv, const int64_t *pk,
                             int parts) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= njobs) return;
    Best best{-INFINITY, INT64_MAX};
    for (int p = 0; p < parts; ++p) best = better(best, Best{pv[(int64_t)j * parts + p], pk[(int64_t)j * parts + p]});
    const int64_t max_lag = jobs[j].biggest - 1;
    *jobs[j].lag_out = best.key == INT64_MAX ? 0 : best.key - max_lag;
}

void global_passes_dif(double2 *z, int64_t n, int64_t block, const double2 *top, int njobs, int64_t stride,
                       cudaStream_t s) {
    // DIF: spans n down to block*2, up to 4 stages per pass.
    int64_t size = n;
    while (size > block) {
        int stages = 0;
        for (int64_t r = size / block; r > 1; r >>= 1) ++stages;
        const int m = stages >= 4 ? 4 : stages;
        const int64_t groups = n >> m;
        dim3 grid((unsigned)((groups + 127) / 128), (unsigned)njobs);
        switch (m) {
            case 4: global_pass<4, false><<<grid, 128, 0, s>>>(z, n, size, top, stride); break;
            case 3: global_pass<3, false><<<grid, 128, 0, s>>>(z, n, size, top, stride); break;
            case 2: global_pass<2, false><<<grid, 128, 0, s>>>(z, n, size, top, stride); break;
            default: global_pass<1, false><<<grid, 128, 0, s>>>(z, n, size, top, stride); break;
        }
        launch_counter() += 1;
        size >>= m;
    }
}

void global_passes_dit(double2 *z, int64_t n, int64_t block, const double2 *top, int njobs, int64_t stride,
                       cudaStream_t s) {
    int64_t done = block;
    while (done < n) {
        int stages = 0;
        for (int64_t r = n / done; r > 1; r >>= 1) ++stages;
        const int m = stages >= 4 ? 4 : stages;
        done <<= m;
        const int64_t groups = n >> m;
        dim3 grid((unsigned)((groups + 127) / 128), (unsigned)njobs);
        switch (m) {
            case 4: global_pass<4, true><<<grid, 128, 0, s>>>(z, n, done, top, stride); break;
            case 3: global_pass<3, true><<<grid, 128, 0, s>>>(z, n, done, top, stride); break;
            case 2: global_pass<2, true><<<grid, 128, 0, s>>>(z, n, done, top, stride); break;
            default: global_pass<1, true><<<grid, 128, 0, s>>>(z, n, done, top, stride); break;
        }
        launch_counter() += 1;
    }
}

constexpr int kBlock = 4096;

void block_passes(double2 *z, int64_t n, bool dit, const double2 *tw_block, int njobs, int64_t stride,
                  cudaStream_t s) {
    const int B = (int)(n < kBlock ? n : kBlock);
    if (B < 2) return;
    const size_t smem = (size_t)B * sizeof(double2);
    dim3 grid((unsigned)(n / B), (unsigned)njobs);
    if (dit)
        block_pass<true><<<grid, 256, smem, s>>>(z, B, tw_block, stride);
    else
        block_pass<false><<<grid, 256, smem, s>>>(z, B, tw_block, stride);
    launch_counter() += 1;
}

}  // namespace

int fft_block_size(int64_t n) { return (int)(n < kBlock ? n : kBlock); }

void fft_init_attributes() {
    cudaFuncSetAttribute(block_pass<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kBlock * (int)sizeof(double2));
    cudaFuncSetAttribute(block_pass<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kBlock * (int)sizeof(double2));
}

void launch_fft(double2 *z, int64_t n, bool inverse, const double2 *top, const double2 *tw_block, int njobs,
                int64_t stride, cudaStream_t s) {
    const int64_t block = n < kBlock ? n : kBlock;
    if (!inverse) {
        global_passes_dif(z, n, block, top, njobs, stride, s);
        block_passes(z, n, false, tw_block, njobs, stride, s);
    } else {
        block_passes(z, n, true, tw_block, njobs, stride, s);
        global_passes_dit(z, n, block, top, njobs, stride, s);
    }
}

void launch_cross(double2 *z, int64_t n, int njobs, int64_t stride, cudaStream_t s) {
    const int64_t threads = n > 1 ? n / 2 : 1;
    dim3 grid((unsigned)((threads + 255) / 256), (unsigned)njobs);
    cross_kernel<<<grid, 256, 0, s>>>(z, n, stride);
    launch_counter() += 1;
}

int argmax_parts(int64_t n) {
    int64_t parts = (n + 65535) / 65536;
    if (parts < 1) parts = 1;
    if (parts > 256) parts = 256;
    return (int)parts;
}

void launch_argmax(const double2 *z, const LagJob *d_jobs, int njobs, int64_t n, int64_t stride, double *pv,
                   int64_t *pk, cudaStream_t s) {
    const int parts = argmax_parts(n);
    argmax_partial<<<dim3((unsigned)parts, (unsigned)njobs), 256, 0, s>>>(z, d_jobs, stride, pv, pk, parts);
    argmax_final<<<(njobs + 127) / 128, 128, 0, s>>>(d_jobs, njobs, pv, pk, parts);
    launch_counter() += 2;
}

}  // namespace vqb
