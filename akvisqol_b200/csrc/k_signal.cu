// Signal-level kernels: serial reductions in the CPU's order, upper
// envelopes packed for the lag FFT, and the lag/SPL application.
//
// The reference sums signals left to right in f64 (envelope mean and
// Nyquist term, src/envelope.zig:28-41; SPL energy, src/audio.zig:132-136).
// A parallel tree would round differently, so each reduction is one warp per
// signal that reproduces the serial sum's every rounding: tiles of samples
// are staged in shared memory, the sums of x and x*x advance a whole tile at
// a time by an exact integer form of the serial additions (exact_prefix)
// and fall back to adding term by term where it does not apply; the
// alternating Nyquist sum is added term by term. Many signals run side by
// side.
#include "device.cuh"
#include "kernels.h"

namespace vqb {

namespace {

enum SumKind : int {
    kSumAndEnergy = 0,  // out[0] = sum x, out[2] = sum x*x
    kNyquist = 1,       // out[1] = sum (-1)^k (x - out[0]/len); reads out[0]
    kEnergy = 2,        // out[2] = sum x*x
};

// Tiles of 256 consecutive samples move into this warp's shared-memory
// stages by asynchronous copies (each lane 8 samples of coalesced 256-byte
// rows; zeros outside the stored window), kStages tiles in flight. In a
// stage, the 8 samples k = 8L .. 8L+7 of the tile sit at L * kPad + (k & 7):
// lane L reads its own run without bank conflicts, and all lanes read any
// one sample as a broadcast.
constexpr int kRows = 8;
constexpr int kTile = 32 * kRows;
constexpr int kPad = kRows + 1;
constexpr int kSlots = 32 * kPad;
constexpr int kStages = 8;
constexpr int kSerialWarps = 2;

__device__ inline int slot_of(int i) { return (i >> 3) * kPad + (i & 7); }

__device__ double g_copy_guard;  // source address of the zero-filling copies

// 8-byte asynchronous copy to shared memory; `in` false writes zeros.
__device__ inline void copy8(double *dst, const double *src, bool in) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(in ? src : &g_copy_guard),
                 "r"(in ? 8 : 0)
                 : "memory");
}

// Exact shortcut for a serial f64 sum (the CPU's `s += t`, left to right).
// While the running sum stays in one binade [2^e, 2^(e+1)), every value it
// takes is a multiple of u = 2^(e-52), and s + t rounds to the multiple of u
// nearest the exact value, s + u * rint(t / u), unless t / u is a
// half-integer (a tie, which round-half-even settles by the parity of s). A
// tile of terms is then added as integers: q = rint(t / u) per term, a
// prefix sum over the warp, and a check that every partial sum M (in units
// of u) stays a unit inside the binade, 2^52 + 1 <= M <= 2^53 - 2, so that
// the exact value of each addition, within half a unit of u * M, lies in the
// binade as well. The first term that breaks a condition ends the shortcut:
// the sum before it is exact, and the caller adds the rest one at a time.
// t: this lane's terms (tile index 8 * lane + j); left: the tile's terms.
// Returns how many leading terms were added into s (the same in all lanes).
__device__ inline int exact_prefix(double &s, const double (&t)[kRows], int left) {
    const int lane = threadIdx.x & 31;
    const long long bits = __double_as_longlong(s);
    const int e = (int)((bits >> 52) & 0x7ff);
    // zero, subnormal or below 2^-970 (the unit scales below must be
    // normal), infinite or NaN: no shortcut
    if (e < 53 || e == 0x7ff) return 0;
    const double to_units = __longlong_as_double((long long)(2098 - e) << 52);  // 1 / u
    const double from_units = __longlong_as_double((long long)(e - 52) << 52);  // u
    const bool neg = bits < 0;
    long long run[kRows];
    long long acc = 0;
    unsigned ok = 0;
#pragma unroll
    for (int j = 0; j < kRows; ++j) {
        // a power-of-two scale is exact (a result far below 1/2 may round,
        // but rounds to q = 0 either way)
        const double tau = neg ? -(t[j] * to_units) : t[j] * to_units;
        const double q = rint(tau);
        const bool good = fabs(q) <= 0x1p53 && fabs(tau - q) != 0.5;  // NaN and inf fail the first test
        acc += good ? (long long)q : 0;
        run[j] = acc;
        ok |= (unsigned)good << j;
    }
    long long incl = acc;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const long long v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
    }
    const long long base = ((bits & ((1LL << 52) - 1)) | (1LL << 52)) + (incl - acc);
    int first = kTile;
#pragma unroll
    for (int j = kRows - 1; j >= 0; --j) {
        const long long m = base + run[j];
        const bool bad = !((ok >> j) & 1u) || m < (1LL << 52) + 1 || m > (1LL << 53) - 2;
        if (bad && lane * kRows + j < left) first = lane * kRows + j;
    }
    int k = __reduce_min_sync(0xffffffffu, first);
    k = k < left ? k : left;
    if (k > 0) {
        const int last = k - 1, js = last & (kRows - 1);
        long long mine = 0;
#pragma unroll
        for (int j = 0; j < kRows; ++j)
            if (j == js) mine = base + run[j];
        const long long m = __shfl_sync(0xffffffffu, mine, last >> 3);
        const double v = (double)m * from_units;  // m < 2^53: exact
        s = neg ? -v : v;
    }
    return k;
}

// acc += stage terms from .. to - 1, in index order (every lane the same).
__device__ inline void serial_add(double &acc, const double *st, int from, int to) {
    if (from == 0 && to == kTile) {
#pragma unroll 8
        for (int g = 0; g < 32; ++g) {
            const double *p = st + g * kPad;
            double v[kRows];
#pragma unroll
            for (int j = 0; j < kRows; ++j) v[j] = p[j];
#pragma unroll
            for (int j = 0; j < kRows; ++j) acc += v[j];
        }
    } else {
#pragma unroll 8
        for (int i = from; i < to; ++i) acc += st[slot_of(i)];
    }
}

// Left-to-right sums, in index order, of KIND's per-sample terms over
// sample(start + k), k in [0, n): chain 0 (and chain 1 for kSumAndEnergy).
// Sums of x and x*x take the exact integer shortcut tile by tile; the
// alternating Nyquist sum, whose running value changes binade every few
// samples, is added one term at a time from the staged terms.
// stages: this warp's kStages * kSlots doubles. first_nz (kSumAndEnergy):
// the first k whose x*x is nonzero, n if none.
template <int KIND>
__device__ inline void warp_serial(const VSig &sig, int64_t start, int64_t n, double mean, double &acc0,
                                   double &acc1, double *stages, int64_t *first_nz = nullptr) {
    const int lane = threadIdx.x & 31;
    if (n <= 0) return;
    const int64_t ntiles = (n + kTile - 1) / kTile;
    auto issue = [&](int64_t t) {
        if (t < ntiles) {
            double *st = stages + (int)(t % kStages) * kSlots;
#pragma unroll
            for (int r = 0; r < kRows; ++r) {
                const int i = r * 32 + lane;
                const int64_t k = t * kTile + i;
                const int64_t j = start + k - sig.head;
                copy8(st + slot_of(i), sig.base + j, k < n && (uint64_t)j < (uint64_t)sig.avail);
            }
        }
        asm volatile("cp.async.commit_group;\n" ::: "memory");  // empty past the end: the count stays uniform
    };
#pragma unroll
    for (int t = 0; t < kStages - 1; ++t) issue(t);
    int64_t nz = n;
    for (int64_t t = 0; t < ntiles; ++t) {
        issue(t + kStages - 1);
        asm volatile("cp.async.wait_group %0;\n" ::"n"(kStages - 1) : "memory");
        __syncwarp();
        double *st = stages + (int)(t % kStages) * kSlots;
        const int left = (int)(n - t * kTile < kTile ? n - t * kTile : kTile);
        double own[kRows];
#pragma unroll
        for (int j = 0; j < kRows; ++j) own[j] = st[lane * kPad + j];
        if (KIND == kSumAndEnergy) {
            double sq[kRows];
#pragma unroll
            for (int j = 0; j < kRows; ++j) sq[j] = own[j] * own[j];
            if (nz == n) {
                int f = kTile;
#pragma unroll
                for (int j = kRows - 1; j >= 0; --j)
                    if (sq[j] != 0.0 && lane * kRows + j < left) f = lane * kRows + j;
                f = __reduce_min_sync(0xffffffffu, f);
                if (f < kTile) nz = t * kTile + f;
            }
            const int k0 = exact_prefix(acc0, own, left);
            const int k1 = exact_prefix(acc1, sq, left);
            for (int i = k0 < k1 ? k0 : k1; i < left; ++i) {
                const double x = st[slot_of(i)];
                if (i >= k0) acc0 += x;
                if (i >= k1) acc1 += x * x;
            }
        } else if (KIND == kEnergy) {
            double sq[kRows];
#pragma unroll
            for (int j = 0; j < kRows; ++j) sq[j] = own[j] * own[j];
            const int k0 = exact_prefix(acc0, sq, left);
            if (k0 < left) {
                __syncwarp();
#pragma unroll
                for (int j = 0; j < kRows; ++j) st[lane * kPad + j] = sq[j];
                __syncwarp();
                serial_add(acc0, st, k0, left);
            }
        } else {
            const int64_t k0 = start + t * kTile + lane * kRows;
            __syncwarp();
#pragma unroll
            for (int j = 0; j < kRows; ++j) {
                const double d = own[j] - mean;
                st[lane * kPad + j] = ((k0 + j) & 1) ? -d : d;
            }
            __syncwarp();
            serial_add(acc0, st, 0, left);
        }
        __syncwarp();
    }
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    if (KIND == kSumAndEnergy && first_nz) *first_nz = nz;
}

template <int KIND>
__global__ void __launch_bounds__(32 * kSerialWarps) serial_sum_kernel(const SumJob *__restrict__ jobs, int njobs) {
    __shared__ __align__(16) double tiles[kSerialWarps][kStages * kSlots];
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= njobs) return;
    const SumJob job = jobs[warp];
    const int64_t len = job.sig.len;
    const double mean = KIND == kNyquist ? job.out[0] / (double)len : 0.0;
    double acc0 = 0.0, acc1 = 0.0;
    int64_t first_nz = len;
    warp_serial<KIND>(job.sig, 0, len, mean, acc0, acc1, tiles[threadIdx.x >> 5], &first_nz);
    if (lane == 0) {
        if (KIND == kSumAndEnergy) {
            job.out[0] = acc0;
            job.out[2] = acc1;
            job.out[3] = (double)first_nz;  // first index with a nonzero energy term (len if none)
        } else if (KIND == kNyquist) {
            job.out[1] = acc0;
        } else {
            job.out[2] = acc0;
        }
    }
}

// Energy of the lag-aligned degraded signal (reference src/realign.zig:91-110
// then src/audio.zig:132-136): applyLag drops -lag leading samples, or
// prepends lag zeros (which add +0 to the sum), and leaves lags of 0 or
// beyond half the reference alone. The lag is read on the device.
struct AlignedEnergyArgs {
    VSig deg;
    int64_t ref_len;
    const int64_t *lag;
    double *out;  // [energy, aligned length]
    // the serial sums of the whole degraded signal ([sum, -, energy, first
    // index with a nonzero energy term]), or null
    const double *deg_stats;
};

__global__ void __launch_bounds__(32 * kSerialWarps) aligned_energy_kernel(const AlignedEnergyArgs *__restrict__ jobs,
                                                                            int njobs) {
    __shared__ __align__(16) double tiles[kSerialWarps][kStages * kSlots];
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= njobs) return;
    const AlignedEnergyArgs job = jobs[warp];
    const int64_t lag = *job.lag;
    const int64_t half_ref = job.ref_len / 2;
    const int64_t mag = lag < 0 ? -lag : lag;
    const int64_t L = job.deg.len;
    int64_t skip = 0, alen = L;
    if (lag != 0 && mag <= half_ref) {
        if (lag < 0) {
            skip = -lag < L ? -lag : L;
            alen = L - skip;
        } else {
            alen = L + lag;
        }
    }
    // The serial sum over samples skip.. equals the whole signal's when every
    // dropped term is zero: the whole-signal chain holds +0 through them (a
    // +0 term leaves +0 unchanged) and then adds the same terms in the same
    // order. Delays, whose dropped samples are the prepended silence, take
    // this path.
    if (job.deg_stats && (double)skip <= job.deg_stats[3]) {
        if (lane == 0) {
            job.out[0] = job.deg_stats[2];
            job.out[1] = (double)alen;
        }
        return;
    }
    double acc = 0.0, unused = 0.0;
    warp_serial<kEnergy>(job.deg, skip, L - skip, 0.0, acc, unused, tiles[threadIdx.x >> 5]);
    if (lane == 0) {
        job.out[0] = acc;
        job.out[1] = (double)alen;
    }
}

// ---- fast form: tree reductions -------------------------------------------
// The fast form does not reproduce the CPU's rounding, so its statistics are
// deterministic tree sums: kTreeParts CTAs per signal each reduce a
// contiguous range (strided, coalesced loads; warp shuffles; shared memory)
// into scratch, and one warp per signal adds the parts in order.
constexpr int kTreeThreads = 256;

__device__ inline double block_sum(double v, double *sm) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) sm[wid] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x < 32) {
        t = threadIdx.x < (blockDim.x >> 5) ? sm[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
    }
    return t;  // valid in thread 0
}

__device__ inline void part_range(int64_t n, int64_t &lo, int64_t &hi) {
    const int64_t per = (n + kTreeParts - 1) / kTreeParts;
    lo = per * blockIdx.x;
    hi = lo + per < n ? lo + per : n;
}

// Partial sums of x, (-1)^k x and x^2 over this CTA's range.
__global__ void __launch_bounds__(kTreeThreads) stats_tree_parts(const SumJob *__restrict__ jobs,
                                                                 double *__restrict__ scratch) {
    __shared__ double sm[kTreeThreads / 32];
    const SumJob job = jobs[blockIdx.y];
    int64_t lo, hi;
    part_range(job.sig.len, lo, hi);
    double s = 0.0, a = 0.0, e = 0.0;
#pragma unroll 4
    for (int64_t k = lo + threadIdx.x; k < hi; k += kTreeThreads) {
        const double x = vsig_at(job.sig, k);
        s += x;
        a += (k & 1) ? -x : x;
        e = __fma_rn(x, x, e);
    }
    s = block_sum(s, sm);
    a = block_sum(a, sm);
    e = block_sum(e, sm);
    if (threadIdx.x == 0) {
        double *p = scratch + ((int64_t)blockIdx.y * kTreeParts + blockIdx.x) * 3;
        p[0] = s;
        p[1] = a;
        p[2] = e;
    }
}

// out[0] = sum x, out[1] = sum (-1)^k (x - mean) = alt - mean * (len odd),
// out[2] = sum x^2.
__global__ void __launch_bounds__(32) stats_tree_finish(const SumJob *__restrict__ jobs,
                                                        const double *__restrict__ scratch) {
    const SumJob job = jobs[blockIdx.x];
    const double *p = scratch + (int64_t)blockIdx.x * kTreeParts * 3;
    const int lane = threadIdx.x;
    double s = p[lane * 3], a = p[lane * 3 + 1], e = p[lane * 3 + 2];
    for (int o = 16; o > 0; o >>= 1) {
        s += __shfl_down_sync(0xffffffffu, s, o);
        a += __shfl_down_sync(0xffffffffu, a, o);
        e += __shfl_down_sync(0xffffffffu, e, o);
    }
    if (lane == 0) {
        const int64_t len = job.sig.len;
        const double mean = len > 0 ? s / (double)len : 0.0;
        job.out[0] = s;
        job.out[1] = (len & 1) ? a - mean : a;
        job.out[2] = e;
    }
}

// Aligned energy (as aligned_energy_kernel) as a tree sum.
__device__ inline void aligned_range(const AlignedEnergyArgs &job, int64_t &skip, int64_t &alen) {
    const int64_t lag = *job.lag;
    const int64_t half_ref = job.ref_len / 2;
    const int64_t mag = lag < 0 ? -lag : lag;
    const int64_t L = job.deg.len;
    skip = 0;
    alen = L;
    if (lag != 0 && mag <= half_ref) {
        if (lag < 0) {
            skip = -lag < L ? -lag : L;
            alen = L - skip;
        } else {
            alen = L + lag;
        }
    }
}

__global__ void __launch_bounds__(kTreeThreads) aligned_tree_parts(const AlignedEnergyArgs *__restrict__ jobs,
                                                                   double *__restrict__ scratch) {
    __shared__ double sm[kTreeThreads / 32];
    const AlignedEnergyArgs job = jobs[blockIdx.y];
    int64_t skip, alen;
    aligned_range(job, skip, alen);
    int64_t lo, hi;
    part_range(job.deg.len - skip, lo, hi);
    double e = 0.0;
#pragma unroll 4
    for (int64_t k = lo + threadIdx.x; k < hi; k += kTreeThreads) {
        const double x = vsig_at(job.deg, skip + k);
        e = __fma_rn(x, x, e);
    }
    e = block_sum(e, sm);
    if (threadIdx.x == 0) scratch[((int64_t)blockIdx.y * kTreeParts + blockIdx.x) * 3] = e;
}

__global__ void __launch_bounds__(32) aligned_tree_finish(const AlignedEnergyArgs *__restrict__ jobs,
                                                          const double *__restrict__ scratch) {
    const AlignedEnergyArgs job = jobs[blockIdx.x];
    double e = scratch[((int64_t)blockIdx.x * kTreeParts + threadIdx.x) * 3];
    for (int o = 16; o > 0; o >>= 1) e += __shfl_down_sync(0xffffffffu, e, o);
    if (threadIdx.x == 0) {
        int64_t skip, alen;
        aligned_range(job, skip, alen);
        job.out[0] = e;
        job.out[1] = (double)alen;
    }
}

__host__ __device__ inline int64_t next_pow_two(int64_t x) {
    int64_t n = 1;
    while (n < x) n <<= 1;
    return n;
}

// upperEnvelope's closed form (reference src/envelope.zig:23-53) for both
// signals of a lag job, packed as z = env_a + i env_b zero-padded to n
// (reference src/xcorr.zig:204-208). raw: the signals themselves.
template <bool RAW>
__global__ void __launch_bounds__(256) pack_kernel(const LagJob *__restrict__ jobs, int njobs) {
    const LagJob job = jobs[blockIdx.y];
    const int64_t n = job.n;
    double mean_a = 0, q_a = 0, mean_b = 0, q_b = 0;
    if (!RAW) {
        const int64_t la = job.a.len, lb = job.b.len;
        if (la > 0) {
            mean_a = job.stats_a[0] / (double)la;
            const int64_t Na = next_pow_two(la) > 32 ? next_pow_two(la) : 32;
            q_a = job.stats_a[1] / (double)Na;
        }
        if (lb > 0) {
            mean_b = job.stats_b[0] / (double)lb;
            const int64_t Nb = next_pow_two(lb) > 32 ? next_pow_two(lb) : 32;
            q_b = job.stats_b[1] / (double)Nb;
        }
    }
    const double eps = 0.000001;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double re = 0.0, im = 0.0;
        if (i < job.a.len) {
            const double x = vsig_at(job.a, i);
            if (RAW) {
                re = x;
            } else {
                const double pc = x - mean_a;
                const double nt = (i & 1) ? -q_a : q_a;
                re = fabs(2.0 * (pc - nt) - eps) + mean_a;
            }
        }
        if (i < job.b.len) {
            const double x = vsig_at(job.b, i);
            if (RAW) {
                im = x;
            } else {
                const double pc = x - mean_b;
                const double nt = (i & 1) ? -q_b : q_b;
                im = fabs(2.0 * (pc - nt) - eps) + mean_b;
            }
        }
        job.z[i] = make_double2(re, im);
    }
}

// out[i] = aligned(i) * factor: scaleToMatchSpl on the lag-aligned signal
// (reference src/audio.zig:152-158; x * 1.0 == x when unscaled).
struct ScaleArgs {
    VSig src;
    double factor;
    double *out;
};

__global__ void __launch_bounds__(256) scale_kernel(const ScaleArgs *__restrict__ jobs, int njobs) {
    const ScaleArgs job = jobs[blockIdx.y];
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < job.src.len;
         i += (int64_t)gridDim.x * blockDim.x)
        job.out[i] = vsig_at(job.src, i) * job.factor;
}

}  // namespace

uint64_t &launch_counter() {
    static thread_local uint64_t count = 0;
    return count;
}

void launch_envelope_stats(const SumJob *d_jobs, int njobs, cudaStream_t s) {
    if (njobs <= 0) return;
    const int per_block = kSerialWarps;
    const int grid = (njobs + per_block - 1) / per_block;
    serial_sum_kernel<kSumAndEnergy><<<grid, 32 * per_block, 0, s>>>(d_jobs, njobs);
    serial_sum_kernel<kNyquist><<<grid, 32 * per_block, 0, s>>>(d_jobs, njobs);
    launch_counter() += 2;
}

void launch_energy(const SumJob *d_jobs, int njobs, cudaStream_t s) {
    if (njobs <= 0) return;
    const int per_block = kSerialWarps;
    serial_sum_kernel<kEnergy><<<(njobs + per_block - 1) / per_block, 32 * per_block, 0, s>>>(d_jobs, njobs);
    launch_counter() += 1;
}

void launch_aligned_energy(const void *d_args, int njobs, cudaStream_t s) {
    if (njobs <= 0) return;
    const int per_block = kSerialWarps;
    aligned_energy_kernel<<<(njobs + per_block - 1) / per_block, 32 * per_block, 0, s>>>(
        static_cast<const AlignedEnergyArgs *>(d_args), njobs);
    launch_counter() += 1;
}

void launch_envelope_stats_tree(const SumJob *d_jobs, int njobs, double *d_scratch, cudaStream_t s) {
    if (njobs <= 0) return;
    static_assert(kTreeParts == 32, "the finishing warp adds one part per lane");
    stats_tree_parts<<<dim3(kTreeParts, (unsigned)njobs), kTreeThreads, 0, s>>>(d_jobs, d_scratch);
    stats_tree_finish<<<njobs, 32, 0, s>>>(d_jobs, d_scratch);
    launch_counter() += 2;
}

void launch_aligned_energy_tree(const void *d_args, int njobs, double *d_scratch, cudaStream_t s) {
    if (njobs <= 0) return;
    const auto *a = static_cast<const AlignedEnergyArgs *>(d_args);
    aligned_tree_parts<<<dim3(kTreeParts, (unsigned)njobs), kTreeThreads, 0, s>>>(a, d_scratch);
    aligned_tree_finish<<<njobs, 32, 0, s>>>(a, d_scratch);
    launch_counter() += 2;
}

size_t aligned_energy_args_size() { return sizeof(AlignedEnergyArgs); }

void fill_aligned_energy_args(void *dst, const VSig &deg, int64_t ref_len, const int64_t *d_lag, double *d_out,
                              const double *d_deg_stats) {
    AlignedEnergyArgs a{deg, ref_len, d_lag, d_out, d_deg_stats};
    *static_cast<AlignedEnergyArgs *>(dst) = a;
}

void launch_pack(const LagJob *d_jobs, int njobs, int64_t max_n, bool raw, cudaStream_t s) {
    if (njobs <= 0) return;
    const int threads = 256;
    int64_t blocks = (max_n + threads - 1) / threads;
    if (blocks > 4096) blocks = 4096;
    dim3 grid((unsigned)blocks, (unsigned)njobs);
    if (raw)
        pack_kernel<true><<<grid, threads, 0, s>>>(d_jobs, njobs);
    else
        pack_kernel<false><<<grid, threads, 0, s>>>(d_jobs, njobs);
    launch_counter() += 1;
}

size_t scale_args_size() { return sizeof(ScaleArgs); }
void fill_scale_args(void *dst, const VSig &src, double factor, double *out) {
    *static_cast<ScaleArgs *>(dst) = ScaleArgs{src, factor, out};
}
void launch_scale(const void *d_args, int njobs, int64_t max_len, cudaStream_t s) {
    if (njobs <= 0) return;
    const int threads = 256;
    int64_t blocks = (max_len + threads - 1) / threads;
    if (blocks > 2048) blocks = 2048;
    if (blocks < 1) blocks = 1;
    scale_kernel<<<dim3((unsigned)blocks, (unsigned)njobs), threads, 0, s>>>(static_cast<const ScaleArgs *>(d_args),
                                                                            njobs);
    launch_counter() += 1;
}

}  // namespace vqb
