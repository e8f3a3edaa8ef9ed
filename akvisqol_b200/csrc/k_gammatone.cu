// Gammatone filterbank spectrogram, exact form (reference
// src/gammatone.zig:268-306 and 432-467).
//
// Every (frame, band) RMS is an independent 4-biquad recurrence over one
// Hann-windowed frame from zero state, so one thread owns one (frame, band)
// and keeps the eight state values in registers. A CTA takes F consecutive
// frames of one job with all NB bands (F = 256 / NB: 8 frames for 32 bands,
// 12 for 21); in a warp the lanes read the same or neighbouring samples,
// which L1 serves as a broadcast, and the Hann value is uniform across the
// CTA. The work is FP64-pipe bound: 31 dependent-chain f64 operations per
// sample (no FMA, as the CPU), 1 load of signal and 1 of window.
#include "device.cuh"
#include "kernels.h"

namespace vqb {

namespace {

struct Tile {
    int32_t job;
    int32_t frame0;
};

__global__ void __launch_bounds__(256) gammatone_kernel(const SpecJob *__restrict__ jobs, const Tile *__restrict__ tiles,
                                                        const BandCoeffs *__restrict__ coeffs, int nb,
                                                        const double *__restrict__ hann, int window, int hop) {
    const Tile tile = tiles[blockIdx.x];
    const int frames_per_cta = blockDim.x / nb;
    const int fl = threadIdx.x / nb;
    const int band = threadIdx.x - fl * nb;
    if (fl >= frames_per_cta) return;
    const SpecJob job = jobs[tile.job];
    const int64_t f = (int64_t)tile.frame0 + fl;
    if (f >= job.nf) return;
    const BandCoeffs k = coeffs[band];
    double s1c0 = 0, s1c1 = 0, s2c0 = 0, s2c1 = 0, s3c0 = 0, s3c1 = 0, s4c0 = 0, s4c1 = 0;
    double sum_sq = 0;
    const int64_t k0 = f * hop;
    const VSig sig = job.sig;
    auto step = [&](double s) {
        const double f1 = k.s1n0 * s + s1c0;
        s1c0 = k.s1n1 * s + s1c1 - k.d1 * f1;
        s1c1 = -(k.d2 * f1);
        const double f2 = k.ca0 * f1 + s2c0;
        s2c0 = k.s2n1 * f1 + s2c1 - k.d1 * f2;
        s2c1 = -(k.d2 * f2);
        const double f3 = k.ca0 * f2 + s3c0;
        s3c0 = k.s3n1 * f2 + s3c1 - k.d1 * f3;
        s3c1 = -(k.d2 * f3);
        const double f4 = k.ca0 * f3 + s4c0;
        s4c0 = k.s4n1 * f3 + s4c1 - k.d1 * f4;
        s4c1 = -(k.d2 * f4);
        sum_sq += f4 * f4;
    };
    if (nb == 32) {
        // A warp is one frame's 32 bands: lane j forms windowed sample
        // i0 + j once (coalesced loads, one multiply per 32 samples) and the
        // warp reads it by shuffle, taking the product off the FP64 pipe.
        const int lane = threadIdx.x & 31;
        int i0 = 0;
        for (; i0 + 32 <= window; i0 += 32) {
            const double x = vsig_at(sig, k0 + i0 + lane) * __ldg(hann + i0 + lane);
#pragma unroll 8
            for (int j = 0; j < 32; ++j) step(__shfl_sync(0xffffffffu, x, j));
        }
        const int rest = window - i0;
        const double x = lane < rest ? vsig_at(sig, k0 + i0 + lane) * __ldg(hann + i0 + lane) : 0.0;
        for (int j = 0; j < rest; ++j) step(__shfl_sync(0xffffffffu, x, j));
    } else {
#pragma unroll 4
        for (int i = 0; i < window; ++i) step(vsig_at(sig, k0 + i) * __ldg(hann + i));
    }
    const double inv_n = 1.0 / (double)window;
    job.out[(int64_t)band * job.nf + f] = sqrt(sum_sq * inv_n);
}

// Grid-aligned frames copied from a full-signal spectrogram (reference
// src/realign.zig:262-281): dst[b*ncols + c] = src[b*stride + col + c].
__global__ void __launch_bounds__(256) copy_frames_kernel(const CopyJob *__restrict__ jobs, int nb) {
    const CopyJob job = jobs[blockIdx.y];
    const int total = nb * job.ncols;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += gridDim.x * blockDim.x) {
        const int b = e / job.ncols, c = e - b * job.ncols;
        job.dst[e] = job.src[(int64_t)b * job.src_stride + job.src_col + c];
    }
}

}  // namespace

int gammatone_frames_per_cta(int nb) { return 256 / nb; }

std::vector<int> gammatone_frames_candidates(int nb) {
    const int f = 256 / nb;
    std::vector<int> c{f};
    if (f / 2 >= 1) c.push_back(f / 2);
    if (f / 4 >= 1) c.push_back(f / 4);
    return c;
}
size_t gammatone_tile_size() { return sizeof(Tile); }
void fill_gammatone_tile(void *dst, int job, int frame0) { *static_cast<Tile *>(dst) = Tile{job, frame0}; }

void launch_gammatone(const SpecJob *d_jobs, const void *d_tiles, int ntiles, const BandCoeffs *d_coeffs, int nb,
                      const double *d_hann, int window, int hop, int frames_per_cta, cudaStream_t s) {
    if (ntiles <= 0) return;
    const int threads = frames_per_cta * nb;
    gammatone_kernel<<<ntiles, threads, 0, s>>>(d_jobs, static_cast<const Tile *>(d_tiles), d_coeffs, nb, d_hann,
                                               window, hop);
    launch_counter() += 1;
}

void launch_copy_frames(const CopyJob *d_jobs, int njobs, int nb, int max_cols, cudaStream_t s) {
    if (njobs <= 0) return;
    const int total = nb * max_cols;
    const int blocks = (total + 255) / 256;
    copy_frames_kernel<<<dim3((unsigned)(blocks < 1 ? 1 : blocks), (unsigned)njobs), 256, 0, s>>>(d_jobs, nb);
    launch_counter() += 1;
}

}  // namespace vqb
