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

// Tiles of 1024 consecutive samples move into this warp's shared-memory
// stages by asynchronous copies (coalesced 256-byte rows; zeros outside the
// stored window), kStages tiles in flight. In a stage, the 32 samples
// k = 32L .. 32L+31 of the tile sit at L * kPad + (k & 31): lane L reads its
// own run without bank conflicts, and all lanes read any one sample as a
// broadcast.
constexpr int kRows = 32;
constexpr int kTile = 32 * kRows;
constexpr int kPad = kRows + 1;
constexpr int kSlots = 32 * kPad;
constexpr int kStages = 4;
constexpr int kSerialWarps = 1;

__device__ inline int slot_of(int i) { return (i >> 5) * kPad + (i & 31); }

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
// half-integer (a tie, which round-half-even settles by the parity of s).
// A tile of terms then adds as integers in units of u: q = rint(t / u) per
// term, a prefix sum over the warp, and a check that every partial sum M
// stays a unit inside the binade, 2^52 + 1 <= M <= 2^53 - 2, so that the
// exact value of each addition, within half a unit of u * M, lies in the
// binade as well. The integers are held in f64. Every lane runs a sum of
// its own q and the warp scans the lane totals; the checks find the first
// lane holding a failing position exactly: before it, every partial sum
// (a difference of two valid M) is an integer below 2^52 in magnitude; in
// it, each of its sums up to the failing position adds one |q| <= 2^52 to
// such a sum, which stays below 2^53; and its starting offset comes from the
// exclusive scan of the lanes before it alone. The lanes before it are
// added at once, that lane's run one term at a time, and the rest of the
// tile is tried again from the new sum.
constexpr double kLo = 0x1p52 + 1.0, kHi = 0x1p53 - 2.0;
constexpr int kMinRetry = 96;  // fewer terms left in a tile than this are added one at a time
constexpr int kMaxRetries = 3;  // shortcut attempts after the first in one tile

struct Chain {
    double to, from, m0;  // +-1/u, +-u (the sum's sign folded in), |s| / u
    bool ok;              // s is normal and above 2^-970 (the unit scales are normal)
    double run, lo, hi;   // this lane's running sum of q, and its extremes over its positions
    bool good;            // no tie or oversized term among this lane's positions
    __device__ inline void begin(double s) {
        const long long bits = __double_as_longlong(s);
        const int e = (int)((bits >> 52) & 0x7ff);
        ok = e >= 53 && e != 0x7ff;
        const double inv = __longlong_as_double((long long)((unsigned long long)(2098 - e) << 52));
        const double u = __longlong_as_double((long long)((unsigned long long)(e - 52) << 52));
        to = bits < 0 ? -inv : inv;
        from = bits < 0 ? -u : u;
        m0 = (double)((bits & ((1LL << 52) - 1)) | (1LL << 52));
        run = 0.0;
        lo = INFINITY;
        hi = -INFINITY;
        good = true;
    }
    // the term t of this lane's next position (a zero-filled position past
    // the end adds q = 0)
    __device__ inline void add(double t) {
        const double tau = t * to;  // a power-of-two scale: exact (or far below 1/2)
        const double q = rint(tau);
        // |q| <= 2^52 keeps every partial sum up to the first failing position
        // below 2^53 (exact); NaN and inf fail the first test
        const bool b = fabs(q) <= 0x1p52 && fabs(tau - q) != 0.5;
        good = good && b;
        run += b ? q : 0.0;
        lo = run < lo ? run : lo;
        hi = run > hi ? run : hi;
    }
    // After the lanes' passes: adds to s every lane before the first lane
    // holding a failing position, or the whole tile; returns that lane (32
    // if none). The same in all lanes.
    __device__ inline int settle(double &s) const {
        const int lane = threadIdx.x & 31;
        double incl = run;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const double v = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += v;
        }
        const double excl = __shfl_up_sync(0xffffffffu, incl, 1);
        const double base = m0 + (lane == 0 ? 0.0 : excl);
        const unsigned failing = __ballot_sync(0xffffffffu, !(good && base + lo >= kLo && base + hi <= kHi));
        const int fail = failing ? __ffs(failing) - 1 : 32;
        // every lane before the first failing one holds only valid partial
        // sums, so the sum at the start of that lane's run is exact
        s = (fail < 32 ? __shfl_sync(0xffffffffu, base, fail & 31) : m0 + __shfl_sync(0xffffffffu, incl, 31)) * from;
        return fail;
    }
};

// True when every term of the tile from position k on is zero: a sum at +0
// stays +0 through them.
__device__ inline bool zeros_from(const double *own, int k) {
    const int lane = threadIdx.x & 31;
    bool z = true;
#pragma unroll 8
    for (int j = 0; j < kRows; ++j) z = z && (lane * kRows + j < k || own[j] == 0.0);
    return __all_sync(0xffffffffu, z);
}

// s += the tile's terms of one chain at positions from .. to - 1 (all in one
// lane's run of 32), one at a time in index order. Positions outside the
// range add +0.0, which leaves any sum that started at +0.0 unchanged (such
// a sum is never -0.0).
template <bool SQUARE>
__device__ inline void serial_run(double &s, const double *st, int run_start, int from, int to) {
    const double *p = st + (run_start >> 5) * kPad;
    double v[kRows];
#pragma unroll
    for (int j = 0; j < kRows; ++j) {
        const int i = run_start + j;
        const double x = p[j];
        v[j] = i >= from && i < to ? (SQUARE ? x * x : x) : 0.0;
    }
#pragma unroll
    for (int j = 0; j < kRows; ++j) s += v[j];
}

// The rest of a tile from position k, where the shortcut stopped: the run
// holding k one term at a time, then the shortcut again over what follows
// (at most kMaxRetries times), else term by term to the end.
template <bool SQUARE>
__device__ __noinline__ void add_rest(double &s, const double *st, const double *own, int k, int left) {
    const int lane = threadIdx.x & 31;
    for (int tries = 0;; ++tries) {
        const int end = (k | (kRows - 1)) + 1 < left ? (k | (kRows - 1)) + 1 : left;
        serial_run<SQUARE>(s, st, k & ~(kRows - 1), k, end);
        k = end;
        if (k >= left) return;
        if (left - k < kMinRetry || tries == kMaxRetries) break;
        if (s == 0.0 && zeros_from(own, k)) return;
        Chain c;
        c.begin(s);
        if (!c.ok) continue;
#pragma unroll 8
        for (int j = 0; j < kRows; ++j) c.add(lane * kRows + j >= k ? (SQUARE ? own[j] * own[j] : own[j]) : 0.0);
        // Lanes wholly before k add only zeros: settle leaves s as it was if
        // one of them is reported (its check sees s itself, which may sit
        // on the binade's edge), and k does not move back.
        const int fail = c.settle(s);
        if (fail == 32) return;
        k = fail * kRows > k ? fail * kRows : k;
    }
    for (; k < left; k = (k & ~(kRows - 1)) + kRows) serial_run<SQUARE>(s, st, k & ~(kRows - 1), k, left);
}

// One chain's tile after its pass: the shortcut where the checks pass, the
// rest through add_rest.
template <bool SQUARE>
__device__ inline void finish_tile(double &s, const Chain &c, const double *st, const double *own, int left) {
    if (s == 0.0 && zeros_from(own, 0)) return;
    int k = 0;
    if (c.ok) {
        const int fail = c.settle(s);
        if (fail == 32) return;
        k = fail * kRows;
    }
    add_rest<SQUARE>(s, st, own, k, left);
}

// Left-to-right sums, in index order, of KIND's per-sample terms over
// sample(start + k), k in [0, n): chain 0 (and chain 1 for kSumAndEnergy).
// Sums of x and x*x take the exact integer shortcut tile by tile and add
// term by term where it does not apply; the alternating Nyquist sum, whose
// running value changes binade every few samples, is added term by term
// from staged terms. stages: this warp's kStages * kSlots doubles.
// first_nz (kSumAndEnergy): the first k whose x*x is nonzero, n if none.
template <int KIND>
__device__ inline void warp_serial(const VSig &sig, int64_t start, int64_t n, double mean, double &acc0,
                                   double &acc1, double *stages, int64_t *first_nz = nullptr) {
    const int lane = threadIdx.x & 31;
    if (n <= 0) return;
    const int64_t ntiles = (n + kTile - 1) / kTile;
    auto issue_row = [&](int64_t t, int r) {  // row r of tile t (32 samples), if the tile exists
        if (t < ntiles) {
            const int64_t k = t * kTile + r * 32 + lane;
            const int64_t j = start + k - sig.head;
            copy8(stages + (int)(t % kStages) * kSlots + r * kPad + lane, sig.base + j,
                  k < n && (uint64_t)j < (uint64_t)sig.avail);
        }
    };
    auto commit = [] { asm volatile("cp.async.commit_group;\n" ::: "memory"); };  // one group a tile, even empty
    auto issue = [&](int64_t t) {
#pragma unroll 8
        for (int r = 0; r < kRows; ++r) issue_row(t, r);
        commit();
    };
#pragma unroll
    for (int t = 0; t < kStages - 1; ++t) issue(t);
    int64_t nz = n;
    for (int64_t t = 0; t < ntiles; ++t) {
        issue(t + kStages - 1);
        asm volatile("cp.async.wait_group %0;\n" ::"n"(kStages - 1) : "memory");
        __syncwarp();
        double *st = stages + (int)(t % kStages) * kSlots;
        double *own = st + lane * kPad;
        const int left = (int)(n - t * kTile < kTile ? n - t * kTile : kTile);
        if (KIND == kSumAndEnergy) {
            Chain c0, c1;
            c0.begin(acc0);
            c1.begin(acc1);
#pragma unroll 8
            for (int j = 0; j < kRows; ++j) {
                const double x = own[j];
                c0.add(x);
                c1.add(x * x);
            }
            if (nz == n) {
                int f = kTile;
                for (int j = kRows - 1; j >= 0; --j)
                    if (own[j] * own[j] != 0.0) f = lane * kRows + j;
                f = __reduce_min_sync(0xffffffffu, f);
                if (f < left) nz = t * kTile + f;
            }
            finish_tile<false>(acc0, c0, st, own, left);
            finish_tile<true>(acc1, c1, st, own, left);
        } else if (KIND == kEnergy) {
            Chain c0;
            c0.begin(acc0);
#pragma unroll 8
            for (int j = 0; j < kRows; ++j) c0.add(own[j] * own[j]);
            finish_tile<true>(acc0, c0, st, own, left);
        } else {
            const int64_t k0 = start + t * kTile + lane * kRows;
#pragma unroll 8
            for (int j = 0; j < kRows; ++j) {
                const double d = own[j] - mean;
                own[j] = ((k0 + j) & 1) ? -d : d;
            }
            __syncwarp();
            if (left == kTile) {
#pragma unroll 2
                for (int g = 0; g < 32; ++g) {
                    const double *p = st + g * kPad;
                    double v[kRows];
#pragma unroll
                    for (int j = 0; j < kRows; ++j) v[j] = p[j];
#pragma unroll
                    for (int j = 0; j < kRows; ++j) acc0 += v[j];
                }
            } else {
                for (int i = 0; i < left; ++i) acc0 += st[slot_of(i)];
            }
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
#pragma unroll 4
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
    // eight or more samples a thread: a CTA per 2048 samples, at most 256 a
    // signal (one sample a thread made block scheduling the cost)
    const int threads = 256;
    int64_t blocks = (max_len + 8 * threads - 1) / (8 * threads);
    if (blocks > 256) blocks = 256;
    if (blocks < 1) blocks = 1;
    scale_kernel<<<dim3((unsigned)blocks, (unsigned)njobs), threads, 0, s>>>(static_cast<const ScaleArgs *>(d_args),
                                                                            njobs);
    launch_counter() += 1;
}

}  // namespace vqb
