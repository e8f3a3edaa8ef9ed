// Patch-alignment DP and backtrack (reference src/dp.zig:216-352).
//
// One CTA per pair. Rows (reference patches) are serial. Within a row the
// CPU keeps a running maximum of the previous row over [prev_lo, slide)
// with `>=` (ties go to the later offset); that is an inclusive prefix scan
// under an associative operator, so the CTA forms it as a blocked scan
// (warp shuffles, then a carry across chunks), then evaluates every slide
// of the row in parallel. The backtrack is a short serial walk.
#include "device.cuh"
#include "kernels.h"

namespace vqb {

namespace {

constexpr int kDpThreads = 512;

struct RunMax {
    double v;
    int64_t i;  // -1: empty
};

// Sequential `if (val >= running_max) take` over A then B.
__device__ inline RunMax combine(RunMax a, RunMax b) {
    if (b.i < 0) return a;
    if (a.i < 0) return b;
    return b.v >= a.v ? b : a;
}

__global__ void __launch_bounds__(kDpThreads) dp_kernel(const DpJob *__restrict__ jobs) {
    const DpJob job = jobs[blockIdx.x];
    const int np = job.np;
    const int64_t cols = job.nf_deg;
    double *dp = job.dp;
    int64_t *bt = job.bt;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    __shared__ RunMax warp_tot[kDpThreads / 32];
    __shared__ RunMax carry_sm;

    // dp and bt start zeroed, as the CPU's memset (cells outside a row's
    // window are read as 0 by later rows and by the backtrack).
    for (int64_t e = tid; e < (int64_t)np * cols; e += blockDim.x) {
        dp[e] = 0.0;
        bt[e] = 0;
    }
    __syncthreads();

    for (int pi = 0; pi < np; ++pi) {
        const int64_t start = job.lo[pi], end = job.hi[pi];
        const double *sims = job.sims + (int64_t)pi * cols;
        double *row = dp + (int64_t)pi * cols;
        int64_t *brow = bt + (int64_t)pi * cols;
        if (pi == 0) {
            for (int64_t s = start + tid; s <= end; s += blockDim.x) {
                row[s] = sims[s];
                brow[s] = -1;
            }
            __syncthreads();
            continue;
        }
        const double *prev = dp + (int64_t)(pi - 1) * cols;
        const int64_t plo = job.lo[pi - 1];
        // Running max entering slide s is the scan over prev[plo .. s-1].
        // Chunks of blockDim elements covering prev[plo .. end-1], the slides
        // they feed evaluated in the same chunk.
        RunMax carry{0.0, -1};
        for (int64_t c0 = plo; c0 <= end; c0 += blockDim.x) {
            const int64_t e = c0 + tid;  // element index into prev; feeds slide e + 1
            RunMax x{0.0, -1};
            if (e < end) x = RunMax{prev[e], e};
            // inclusive warp scan
            for (int off = 1; off < 32; off <<= 1) {
                RunMax y{__shfl_up_sync(0xffffffffu, x.v, off), __shfl_up_sync(0xffffffffu, x.i, off)};
                if (lane >= off) x = combine(y, x);
            }
            if (lane == 31) warp_tot[wid] = x;
            __syncthreads();
            if (wid == 0) {
                RunMax t = lane < (int)(blockDim.x >> 5) ? warp_tot[lane] : RunMax{0.0, -1};
                for (int off = 1; off < 32; off <<= 1) {
                    RunMax y{__shfl_up_sync(0xffffffffu, t.v, off), __shfl_up_sync(0xffffffffu, t.i, off)};
                    if (lane >= off) t = combine(y, t);
                }
                if (lane < (int)(blockDim.x >> 5)) warp_tot[lane] = t;  // inclusive prefix of warp totals
            }
            __syncthreads();
            RunMax pre = wid > 0 ? warp_tot[wid - 1] : RunMax{0.0, -1};
            RunMax incl = combine(combine(carry, pre), x);
            // scan over prev[plo .. e] feeds slide s = e + 1; the first chunk's
            // slide plo (empty prefix) is handled by the thread with e = plo - 1,
            // i.e. separately below.
            const int64_t s = e + 1;
            if (s >= start && s <= end) {
                double sim = sims[s];
                int64_t past = -1;
                const double rm = incl.i >= 0 ? incl.v : -INFINITY;
                sim += rm;
                past = incl.i;
                const double no_move = prev[s];
                if (no_move > sim) {
                    sim = no_move;
                    past = s;
                }
                row[s] = sim;
                brow[s] = past;
            }
            // the chunk's total becomes the carry
            if (tid == blockDim.x - 1) carry_sm = incl;
            __syncthreads();
            carry = carry_sm;
            __syncthreads();
        }
        // Slide `start` when it equals plo: empty running max (-inf, -1).
        if (tid == 0 && start == plo) {
            double sim = sims[start] + -INFINITY;
            int64_t past = -1;
            const double no_move = prev[start];
            if (no_move > sim) {
                sim = no_move;
                past = start;
            }
            row[start] = sim;
            brow[start] = past;
        }
        __syncthreads();
    }

    // Backtrack from the first maximum of the last row (strict `>`).
    if (tid == 0) {
        const int last = np - 1;
        double best = -INFINITY;
        int64_t cur = 0;
        const double *row = dp + (int64_t)last * cols;
        for (int64_t off = job.lo[last]; off <= job.hi[last]; ++off)
            if (row[off] > best) best = row[off], cur = off;
        for (int p = 0; p < np; ++p) {
            job.offset[p] = -1;
            job.valid[p] = 1;
        }
        for (int p = last; p >= 0; --p) {
            job.offset[p] = cur;
            const int64_t back = bt[(int64_t)p * cols + cur];
            job.valid[p] = back == cur ? 0 : 1;
            if (back < 0) break;
            cur = back;
        }
    }
}

}  // namespace

void launch_dp(const DpJob *d_jobs, int njobs, cudaStream_t s) {
    if (njobs <= 0) return;
    dp_kernel<<<njobs, kDpThreads, 0, s>>>(d_jobs);
    launch_counter() += 1;
}

}  // namespace vqb
