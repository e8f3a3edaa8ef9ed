// Kernel launchers and the job records they read (device memory).
#pragma once

#include <cstddef>
#include <cstdint>
#include <vector>
#include <cuda_runtime.h>

#include "device.cuh"

namespace vqb {

// Degraded plane of one pair (reference src/nsim.zig:224-263).
struct PlaneJob {
    const double *spec;  // prepared degraded spectrogram, nb x nf
    int32_t nf, width;
    double *pad, *mu, *dms, *sds;  // nb x width each
    int32_t roots;  // fast forms: sds holds the signed square root of the variance
};

// Reference-patch terms: spec columns [col, col+P) of a prepared
// spectrogram with nf frames; out is 4 x nb x P.
struct RefTermsJob {
    const double *spec;
    int32_t nf, col;
    double *out;
    int32_t roots;  // fast forms: the variance term holds its signed square root
};

// NSIM table block: offsets [off0, min(off0+127, hi)] of one patch.
struct TableTask {
    const double *ref_terms;  // 4 x nb x P
    const double *pad, *mu, *dms, *sds;
    int32_t width;
    int32_t off0, hi;
    double *out;  // row of the table: out[off]
};

// DP of one pair over its sims table (np x nf_deg).
struct DpJob {
    const double *sims;
    const int64_t *lo, *hi;
    int32_t np;
    int64_t nf_deg;
    double *dp;
    int64_t *bt;
    int64_t *offset;  // np: matched offset, -1 when not reached
    uint8_t *valid;   // np
};

// Per-band coefficients of the fast gammatone forms (k_gammatone_fast.cu).
// Every stage is a biquad with the band's pole pair and a numerator
// normalised to 1 + beta z^-1; the numerator gains are one factor, post64.
struct FastBandCoeffs {
    double d1, d2;             // poles, all four stages
    double beta64[4];          // f64 numerators of stages 1-4
    double post64;             // |s1n0 a0^3|, applied to the RMS
    float beta[2];             // f32 form: numerators of stages 3-4
    float p1h, p1l, p2h, p2l;  // f32 form: poles d1, d2 as hi + lo f32 pairs
    int32_t arith;             // f32 form, per band group: kArith* below
};

// Arithmetic of a band group in the f32 form's gammatone kernel.
constexpr int32_t kArithF32Df2t = 0;  // stages 3-4 f32, transposed direct form II
constexpr int32_t kArithF32Df1 = 1;   // stages 3-4 f32, direct form I
constexpr int32_t kArithF64 = 2;      // all four stages f64 (poles nearest the unit circle)

// Arithmetic forms of the batch pipeline.
enum Form : int32_t {
    kFormExact = 0,  // f64, no FMA, the CPU's operation order (bit-identical stages)
    kFormF32 = 1,    // gammatone stages 3-4 in f32 but in the lowest band group, tree-summed statistics
    kFormF64 = 2,    // gammatone in f64 with FMA (direct form I), tree-summed statistics
};

// Kernels launched by this thread so far (each launcher counts its own).
uint64_t &launch_counter();

// k_signal.cu
void launch_envelope_stats(const SumJob *d_jobs, int njobs, cudaStream_t s);
void launch_energy(const SumJob *d_jobs, int njobs, cudaStream_t s);
size_t aligned_energy_args_size();
// d_deg_stats: the exact form's serial sums of the whole degraded signal
// (launch_envelope_stats), from which the aligned energy is taken when the
// lag drops only zero terms; or null.
void fill_aligned_energy_args(void *dst, const VSig &deg, int64_t ref_len, const int64_t *d_lag, double *d_out,
                              const double *d_deg_stats = nullptr);
void launch_aligned_energy(const void *d_args, int njobs, cudaStream_t s);
void launch_pack(const LagJob *d_jobs, int njobs, int64_t max_n, bool raw, cudaStream_t s);
size_t scale_args_size();
void fill_scale_args(void *dst, const VSig &src, double factor, double *out);
void launch_scale(const void *d_args, int njobs, int64_t max_len, cudaStream_t s);

// Fast form: the same statistics as deterministic tree reductions.
// scratch: kTreeParts * 3 doubles per job.
constexpr int kTreeParts = 32;
void launch_envelope_stats_tree(const SumJob *d_jobs, int njobs, double *d_scratch, cudaStream_t s);
void launch_aligned_energy_tree(const void *d_args, int njobs, double *d_scratch, cudaStream_t s);

// k_fft.cu
void fft_init_attributes();
// Block size of the shared-memory passes, min(n, 4096); tw_block[k] =
// W_B^k = top[k * n/B] for k < B/2.
int fft_block_size(int64_t n);
void launch_fft(double2 *z, int64_t n, bool inverse, const double2 *top, const double2 *tw_block, int njobs,
                int64_t stride, cudaStream_t s);
void launch_cross(double2 *z, int64_t n, int njobs, int64_t stride, cudaStream_t s);
int argmax_parts(int64_t n);
void launch_argmax(const double2 *z, const LagJob *d_jobs, int njobs, int64_t n, int64_t stride, double *pv,
                   int64_t *pk, cudaStream_t s);

// k_lag.cu: the fused three-pass lag search (n <= 2^24).
void lag_init_attributes();
bool fused_lag_supported(int64_t n);
size_t fused_lag_parts(int64_t n);  // argmax candidates per job
// Stage-major column twiddles of the global stages (host-side, from the
// full table top[k] = W_n^k): column_twiddle_count(n) entries.
size_t column_twiddle_count(int64_t n);
void fill_column_twiddles(const double2 *top, int64_t n, double2 *out);
// Stage-major twiddles of the 4096-point block stages, from the block table
// (block[k] = W_4096^k): block_stage_twiddle_count() entries.
size_t block_stage_twiddle_count();
void fill_block_stage_twiddles(const double2 *block, double2 *out);
// columns: 0 = the shared-memory column passes (any n), 1 = the register
// ones, 2 = the register ones with the forward pass's samples staged in
// shared memory (1 and 2 only where fused_lag_register_columns(n); else as
// 0). Same results.
bool fused_lag_register_columns(int64_t n);
void launch_fused_lag(const LagJob *d_jobs, int njobs, int64_t n, bool raw, const double2 *tcol,
                      const double2 *tw_block, const double2 *tst, double *pv, int64_t *pk, int columns,
                      cudaStream_t s);

// k_lag.cu: the f32-nominated search (fused_lag_supported(n)): the same three
// passes in f32, candidates within the f32 error bound of the maximum, f64
// rescoring. Per job: z32 (n points), energy (lag32_parts(n)), cands
// (lag32_parts(n)), status, ncand, cand_key (kLagCandCap), rescore
// (kLagCandCap x nchunks, nchunks = lag32_rescore_chunks(the jobs' largest
// b.len)). A job whose status is 1 afterwards has no lag: the caller reruns
// it with launch_fused_lag. Twiddles: the f64 tables rounded to f32.
void lag32_init_attributes();
size_t lag32_parts(int64_t n);
int lag32_rescore_chunks(int64_t max_b_len);
void launch_lag32(const LagJob *d_jobs, int njobs, int64_t n, bool raw, const float2 *tcol, const float2 *tw_block,
                  const float2 *tst, int nchunks, int columns, cudaStream_t s);  // columns as launch_fused_lag's
// The nomination, pick and rescoring kernels on one job's caller-supplied
// approximate correlation (corr_out, n values) with slack_fixed as the slack,
// raw signals; the job's cands array holds ceil(n / 4096) records.
void launch_refine_approx(const LagJob *d_job, int64_t n, int nchunks, cudaStream_t s);

// k_gammatone.cu
int gammatone_frames_per_cta(int nb);
// CTA shapes the autotuner may choose among for the exact and FP64 FMA
// kernels (frames per CTA; the first is the default).
std::vector<int> gammatone_frames_candidates(int nb);
size_t gammatone_tile_size();
void fill_gammatone_tile(void *dst, int job, int frame0);
void launch_gammatone(const SpecJob *d_jobs, const void *d_tiles, int ntiles, const BandCoeffs *d_coeffs, int nb,
                      const double *d_hann, int window, int hop, int frames_per_cta, cudaStream_t s);
void launch_copy_frames(const CopyJob *d_jobs, int njobs, int nb, int max_cols, cudaStream_t s);

// k_gammatone_fast.cu (tiles as fill_gammatone_tile writes them)
int gammatone_fast_frames_per_cta();
void fill_fast_band_coeffs(const BandCoeffs *run, const double *cf, int nb, FastBandCoeffs *out);
// shape: one of gammatone_fast_shape_candidates(): CTAs per SM (register
// budget), plus 100 for the persistent form, which takes its tiles from a
// work queue: d_queue, one int that is zero when the launch starts.
std::vector<int> gammatone_fast_shape_candidates();  // measured by the autotuner
std::vector<int> gammatone_fast_shapes();            // all valid shapes
void launch_gammatone_fast(const SpecJob *d_jobs, const void *d_tiles, int ntiles, const FastBandCoeffs *d_coeffs,
                           int nb, const double *d_hann, int window, int hop, int shape, int *d_queue,
                           cudaStream_t s);
// f64 FMA form: two frames per thread; tiles of frames_per_cta frames, one
// of gammatone_f64fma_frames_candidates(nb) (the first is the default).
std::vector<int> gammatone_f64fma_frames_candidates(int nb);
void launch_gammatone_f64fma(const SpecJob *d_jobs, const void *d_tiles, int ntiles, const FastBandCoeffs *d_coeffs,
                             int nb, const double *d_hann, int window, int hop, int frames_per_cta, cudaStream_t s);
// The f64 FMA form on the FP32 kernel's staged tiles (tiles of
// gammatone_fast_frames_per_cta() frames): the same bits as
// launch_gammatone_f64fma. Candidates of the autotuner: 1 = this one (the
// default), 0 = that kernel.
std::vector<int> gammatone_f64_staged_candidates();
void launch_gammatone_f64_staged(const SpecJob *d_jobs, const void *d_tiles, int ntiles,
                                 const FastBandCoeffs *d_coeffs, int nb, const double *d_hann, int window, int hop,
                                 cudaStream_t s);

// k_grad.cu: the gammatone spectrogram's reverse (FP64-FMA arithmetic).
// Tiles as fill_gammatone_tile writes them, of gammatone_bwd_frames_per_cta()
// frames; d_scratch holds gammatone_bwd_scratch_count(ntiles, window) doubles.
int gammatone_bwd_frames_per_cta();
size_t gammatone_bwd_scratch_count(int ntiles, int window);
void launch_gammatone_bwd(const GradSpecJob *d_jobs, const void *d_tiles, int ntiles, const FastBandCoeffs *d_coeffs,
                          int nb, const double *d_hann, int window, int hop, double *d_scratch, cudaStream_t s);

// k_spec.cu
// Spectrogram preparation of njobs pairs (max_frames = the largest nfr or
// nfd); d_scratch holds prep_scratch_count(njobs, max_frames) doubles.
size_t prep_scratch_count(int njobs, int max_frames);
void launch_prep(const PrepJob *d_jobs, int njobs, int nb, int max_frames, double *d_scratch, cudaStream_t s);
void launch_log10(const double *x, int64_t n, double *out, cudaStream_t s);

// k_nsim.cu
void nsim_init_attributes();
void launch_plane(const PlaneJob *d_jobs, int njobs, int nb, int max_width, cudaStream_t s);
void launch_ref_terms(const RefTermsJob *d_jobs, int njobs, int nb, int P, cudaStream_t s);
int table_offsets_per_cta();
// fast: the fast forms' cell arithmetic (FMA, one division per cell);
// width: offsets per CTA, one of table_width_candidates(P) (the first is the
// default); tasks must be built with the same width.
std::vector<int> table_width_candidates(int P);
void launch_table(const TableTask *d_tasks, int ntasks, int nb, int P, bool fast, int width, cudaStream_t s);
void launch_stats(const StatsJob *d_jobs, int njobs, int nb, cudaStream_t s);
// The fast forms' NSIM quotient n / d (d > 0, normal) elementwise, for its
// direct test.
void launch_fast_quotient(const double *num, const double *den, double *out, size_t count, cudaStream_t s);

// k_dp.cu
void launch_dp(const DpJob *d_jobs, int njobs, cudaStream_t s);

}  // namespace vqb
