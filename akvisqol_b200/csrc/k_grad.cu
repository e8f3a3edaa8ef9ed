// Reverse of the gammatone RMS spectrogram (reference src/gpu/pipeline.zig:842-1143,
// its gammatone_bwd kernel): from d loss / d RMS cell to d loss / d sample.
//
// One (frame, band) is RMS = post sqrt(sum_i y_i^2 / W) with y the unit
// cascade of four biquads (direct form I, numerators 1 + beta z^-1, the
// FP64-FMA form's arithmetic) over the Hann-windowed frame x_i. So
//
//   d loss / d x = H^T (g post^2 / (W RMS) y),
//
// H the cascade as a lower-triangular Toeplitz map over the frame (zero
// state at its start). H^T is H run backwards in time (zero state at the
// frame's end): reverse the sequence, filter with the same four stages,
// reverse again. The sequence it filters is y in reverse order, so y is
// recomputed block by block, last block first, from states the forward
// pass saves every kBlock samples (in global scratch), into this thread's
// shared-memory column. A warp is one frame's bands (lane = band): each
// reversed step's d loss / d sample is summed over the warp's lanes by
// shuffles and added to the sample's gradient by one atomic (four frames
// overlap a sample).
#include "device.cuh"
#include "kernels.h"

namespace vqb {

namespace {

constexpr int kBlock = 64;     // samples between saved states
constexpr int kWarps = 4;      // frames per CTA
constexpr int kState = 9;      // doubles of the cascade's state

struct Cascade {
    double xp = 0.0, y1a = 0.0, y2a = 0.0, y1b = 0.0, y2b = 0.0, y1c = 0.0, y2c = 0.0, y1d = 0.0, y2d = 0.0;
    __device__ inline double step(double x, const double (&b)[4], double nd1, double nd2) {
        const double ya = __fma_rn(nd1, y1a, __fma_rn(nd2, y2a, __fma_rn(b[0], xp, x)));
        const double yb = __fma_rn(nd1, y1b, __fma_rn(nd2, y2b, __fma_rn(b[1], y1a, ya)));
        const double yc = __fma_rn(nd1, y1c, __fma_rn(nd2, y2c, __fma_rn(b[2], y1b, yb)));
        const double yd = __fma_rn(nd1, y1d, __fma_rn(nd2, y2d, __fma_rn(b[3], y1c, yc)));
        xp = x;
        y2a = y1a, y1a = ya;
        y2b = y1b, y1b = yb;
        y2c = y1c, y1c = yc;
        y2d = y1d, y1d = yd;
        return yd;
    }
    __device__ inline void save(double *p) const {
        p[0] = xp, p[1] = y1a, p[2] = y2a, p[3] = y1b, p[4] = y2b, p[5] = y1c, p[6] = y2c, p[7] = y1d, p[8] = y2d;
    }
    __device__ inline void load(const double *p) {
        xp = p[0], y1a = p[1], y2a = p[2], y1b = p[3], y2b = p[4], y1c = p[5], y2c = p[6], y1d = p[7], y2d = p[8];
    }
};

struct GradTile {
    int32_t job, frame0;
};

// grid: tiles of kWarps frames; block: kWarps x 32 threads; dynamic shared
// memory kBlock x blockDim doubles. scratch: per thread nblk x kState.
__global__ void __launch_bounds__(kWarps * 32) gammatone_bwd_kernel(const GradSpecJob *__restrict__ jobs,
                                                                    const GradTile *__restrict__ tiles,
                                                                    const FastBandCoeffs *__restrict__ coeffs, int nb,
                                                                    const double *__restrict__ hann, int window,
                                                                    int hop, double *__restrict__ scratch) {
    extern __shared__ double ybuf[];  // [i][thread]
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const GradTile tile = tiles[blockIdx.x];
    const GradSpecJob job = jobs[tile.job];
    const int64_t f = (int64_t)tile.frame0 + warp;
    const int band = lane < nb ? lane : nb - 1;
    const double g = (lane < nb && f < job.nf) ? job.g_rms[(int64_t)band * job.nf + f] : 0.0;
    if (!__any_sync(0xffffffffu, g != 0.0)) return;  // warp-uniform: no gradient in this frame
    const FastBandCoeffs k = coeffs[band];
    const double b[4] = {k.beta64[0], k.beta64[1], k.beta64[2], k.beta64[3]};
    const double nd1 = -k.d1, nd2 = -k.d2;
    const int nblk = (window + kBlock - 1) / kBlock;
    double *ck = scratch + ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) * nblk * kState;
    const int64_t k0 = f * hop;
    auto x_at = [&](int i) { return vsig_at(job.sig, k0 + i) * __ldg(hann + i); };

    // forward: y and its sum of squares, the state at each block's start
    Cascade c;
    double ss = 0.0;
    for (int blk = 0; blk < nblk; ++blk) {
        c.save(ck + blk * kState);
        const int end = min(window, (blk + 1) * kBlock);
        for (int i = blk * kBlock; i < end; ++i) {
            const double y = c.step(x_at(i), b, nd1, nd2);
            ss = __fma_rn(y, y, ss);
        }
    }
    const double rms = sqrt(ss / (double)window) * k.post64;
    // d loss / d y_i = scale y_i
    const double scale = rms > 0.0 ? g * k.post64 * k.post64 / ((double)window * rms) : 0.0;

    // reverse: blocks last to first; y of the block recomputed into this
    // thread's column, then fed backwards through the same cascade
    Cascade a;
    double *col = ybuf + threadIdx.x;
    for (int blk = nblk - 1; blk >= 0; --blk) {
        c.load(ck + blk * kState);
        const int i0 = blk * kBlock, end = min(window, i0 + kBlock);
        for (int i = i0; i < end; ++i) col[(i - i0) * blockDim.x] = c.step(x_at(i), b, nd1, nd2);
        for (int i = end - 1; i >= i0; --i) {
            const double gx = a.step(scale * col[(i - i0) * blockDim.x], b, nd1, nd2) * __ldg(hann + i);
            double sum = lane < nb ? gx : 0.0;
            for (int off = 16; off > 0; off >>= 1) sum += __shfl_down_sync(0xffffffffu, sum, off);
            if (lane == 0) {
                const int64_t j = k0 + i - job.sig.head;
                if ((uint64_t)j < (uint64_t)job.sig.avail) atomicAdd(job.grad + j, sum);
            }
        }
    }
}

}  // namespace

int gammatone_bwd_frames_per_cta() { return kWarps; }

size_t gammatone_bwd_scratch_count(int ntiles, int window) {
    return (size_t)ntiles * kWarps * 32 * (size_t)((window + kBlock - 1) / kBlock) * kState;
}

void launch_gammatone_bwd(const GradSpecJob *d_jobs, const void *d_tiles, int ntiles, const FastBandCoeffs *d_coeffs,
                          int nb, const double *d_hann, int window, int hop, double *d_scratch, cudaStream_t s) {
    if (ntiles <= 0) return;
    const size_t smem = (size_t)kBlock * kWarps * 32 * sizeof(double);
    cudaFuncSetAttribute(gammatone_bwd_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    gammatone_bwd_kernel<<<ntiles, kWarps * 32, smem, s>>>(d_jobs, static_cast<const GradTile *>(d_tiles), d_coeffs,
                                                           nb, d_hann, window, hop, d_scratch);
    launch_counter() += 1;
}

}  // namespace vqb
