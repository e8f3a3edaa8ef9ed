/* CPU oracle for the ViSQOL hot path: a plain C++ restatement of the
 * reference CPU model (jdek/akvisqol src/visqol.zig and the L2 stages it
 * calls), op for op in f64 with no FMA contraction.
 *
 * TEST INFRASTRUCTURE ONLY. This library is the checker that the CUDA path
 * is compared against, and the timed CPU baseline. The product library
 * (akvisqol_b200/libvisqol.so) never links, loads or calls it.
 *
 * Every function cites the reference file:line it follows.
 */
#ifndef VISQOL_ORACLE_H
#define VISQOL_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Same layout as visqol_options / visqol_patch / visqol_result
 * (reference src/include/visqol.h:45-82). */
typedef struct {
    uint32_t mode;
    int32_t search_window_radius;
    uint8_t use_unscaled_speech_mos_mapping;
    uint8_t disable_global_alignment;
    uint8_t disable_realignment;
    uint8_t use_lattice_model;
    const char *model_path;
    uint32_t backend;
    uint32_t precision;
} vqo_options;

typedef struct {
    double similarity;
    double ref_patch_start_time;
    double ref_patch_end_time;
    double deg_patch_start_time;
    double deg_patch_end_time;
    const double *freq_band_means;
    const double *freq_band_stddevs;
    const double *freq_band_deg_energy;
} vqo_patch;

typedef struct {
    double moslqo;
    double vnsim;
    double alignment_lag_s;
    size_t num_bands;
    const double *fvnsim;
    const double *fvnsim10;
    const double *fstdnsim;
    const double *fvdegenergy;
    const double *center_freq_bands;
    size_t num_patches;
    const vqo_patch *patch_sims;
} vqo_result;

/* Discrete decisions and work counters of one measurement, for parity
 * checks (lags, frames, matches) and roofline accounting. */
typedef struct {
    int64_t global_lag;          /* samples, before applyLag's half-ref rule */
    double spl_factor;           /* scaleToMatchSpl factor, 1 when unscaled */
    uint64_t deg_len;            /* aligned degraded length */
    uint64_t nf_ref, nf_deg;
    uint64_t num_patches;
    const int64_t *ref_index;    /* per patch: reference start frame */
    const int64_t *deg_offset;   /* per patch: DP-matched degraded frame */
    const uint8_t *valid;        /* per patch: DP match valid */
    const int64_t *realign_lag;  /* per patch: envelope lag of the slices (0 if not run) */
    const int64_t *realign_frames; /* per patch: frames of the trimmed slices, -1 if not run */
    const uint8_t *realign_reused; /* per patch: bit0 ref frames copied, bit1 deg frames copied */
    const uint8_t *realign_accepted;
    uint64_t n_rms;              /* (frame, band) RMS evaluations computed */
    uint64_t n_rms_window;       /* samples per RMS evaluation (W) */
    uint64_t n_cells;            /* NSIM cells evaluated (table + stats) */
    double fft_nlogn;            /* sum of n*log2(n) over complex FFTs (2 per lag) */
} vqo_trace;

/* ---- full model ---------------------------------------------------- */

void vqo_options_default(vqo_options *o);
/* Returns 0 or a visqol.h error code (-1 invalid, -4 model, -5 signal). */
int vqo_measure(const vqo_options *o, const double *ref, size_t ref_len,
                const double *deg, size_t deg_len, uint32_t sample_rate,
                vqo_result **out, vqo_trace **trace);
void vqo_result_free(vqo_result *r);
void vqo_trace_free(vqo_trace *t);
/* Pair-parallel batch over num_threads std::threads (0: hardware
 * concurrency), each with its own model, as reference
 * src/backend.zig:182-221. status[i] holds each pair's code. */
int vqo_measure_batch(const vqo_options *o, size_t n,
                      const double *const *refs, const size_t *ref_lens,
                      const double *const *degs, const size_t *deg_lens,
                      uint32_t sample_rate, uint32_t num_threads,
                      vqo_result **out, int32_t *status);
const char *vqo_last_error(void);

/* ---- stages (known-answer tests and kernel parity) ------------------ */

/* Centre frequencies descending (src/dsp/erb.zig:30-52). */
void vqo_uniform_center_freqs(size_t n, double low, double high, double *out);
/* Filters.init: coeffs[b*8 + {a0,a11,a12,a13,a14,b1,b2,gain}] ascending,
 * cf ascending (src/gammatone.zig:41-70). */
void vqo_filters(size_t nb, uint32_t sample_rate, double low, double high,
                 double *coeffs, double *cf);
void vqo_hann(size_t size, double *out);
/* filterBand from zero state over `n` samples (src/gammatone.zig:216-265). */
void vqo_filter_band(const double *coeffs8, const double *x, size_t n, double *out);
double vqo_filter_band_rms_fresh(const double *coeffs8, const double *x, size_t n);
/* buildSpectrogramBands; returns frames written (src/gammatone.zig:432-467). */
size_t vqo_spectrogram(size_t nb, const double *coeffs, const double *hann,
                       size_t window, size_t hop, const double *x, size_t n, double *out);
void vqo_upper_envelope(const double *x, size_t n, double *out);
size_t vqo_fft_size_for(size_t biggest);
/* Unscaled DIF forward, bit-reversed out (src/dsp/fft.zig:127-145); and
 * DIT inverse (src/dsp/fft.zig:148-166). buf is interleaved re,im. */
void vqo_fft_dif(double *buf, size_t n);
void vqo_fft_dit(double *buf, size_t n);
/* Twiddles W_n^k, k < n/2, interleaved (src/dsp/fft.zig:55-61). */
void vqo_fft_twiddles(size_t n, double *out);
int64_t vqo_best_lag(const double *a, size_t la, const double *b, size_t lb);
/* bestLag of the upper envelopes (src/accel.zig:100-107). */
int64_t vqo_envelope_lag(const double *a, size_t la, const double *b, size_t lb);
void vqo_convert_to_db(double *x, size_t n, double floor_db);
void vqo_raise_floor_per_frame(double *ref, double *deg, size_t nb, size_t nfr, size_t nfd, double rel);
void vqo_subtract_joint_minimum(double *ref, size_t rn, double *deg, size_t dn);
void vqo_prepare_for_comparison(double *ref, double *deg, size_t nb, size_t nfr, size_t nfd);
void vqo_conv2d3x3(const double *in, double *out, size_t nrows, size_t ncols);
/* measurePatchSimilarity; returns mean_freq_band_means (src/nsim.zig:427-510). */
double vqo_patch_similarity(const double *ref, const double *deg, size_t nrows, size_t ncols,
                            double *means, double *stddevs, double *deg_energy);
/* measureSimilarityScalar (src/nsim.zig:332-360). */
double vqo_similarity_scalar(const double *ref, const double *deg, size_t nrows, size_t ncols);
/* accel.Cpu.patchSimilarities for one pair (src/accel.zig:126-146):
 * out[p*nf_deg + off] for off in [lo[p], hi[p]]. */
void vqo_nsim_table(const double *ref_spec, size_t nf_ref, const double *deg_spec, size_t nf_deg,
                    size_t nb, size_t patch, size_t np, const int64_t *ref_idx,
                    const int64_t *lo, const int64_t *hi, double *out);
/* DP + backtrack over a sims table (src/dp.zig:205-288, 313-352):
 * matched deg offset and validity per patch; returns patches reached. */
size_t vqo_dp_backtrack(const double *sims, size_t np, size_t nf_deg,
                        const int64_t *lo, const int64_t *hi,
                        int64_t *offset, uint8_t *valid);
/* Reference patch start frames; -5 on ReferenceSpectrogramTooSmall. */
int vqo_ref_patch_indices(size_t nf, size_t patch, int64_t *out, size_t *count);
int vqo_vad_patch_indices(const double *ref, size_t n, size_t nf, size_t patch,
                          size_t window, double overlap, int64_t *out, size_t *count);
size_t vqo_calc_max_num_patches(const int64_t *idx, size_t n, size_t nf_deg, size_t patch);
void vqo_slice_layout(size_t len, uint32_t sr, double t0, double t1, int64_t *pad, int64_t *base, int64_t *n);
void vqo_trim_geometry(size_t ref_len, size_t deg_len, int64_t lag, uint32_t sr,
                       int64_t *len, int64_t *ref_off, int64_t *deg_off, double *lag_seconds);
/* truncateAligned (src/realign.zig:147-210): writes ref_out/deg_out
 * (each at least ref_len long); returns the shared length. */
size_t vqo_truncate_aligned(const double *ref, size_t ref_len, const double *deg, size_t deg_len,
                            int64_t lag, uint32_t sr, double *ref_out, double *deg_out);
double vqo_spl(const double *x, size_t n);
double vqo_pow(double x, double y);
/* The SVR model text path (NULL: the bundled default) and prediction. */
int vqo_svr_predict(const char *model_path, const double *x, size_t n, double *y);
int vqo_svr_predict_text(const char *text, size_t len, const double *x, size_t n, double *y);

#ifdef __cplusplus
}
#endif
#endif
