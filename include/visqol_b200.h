/* akvisqol_b200 extensions to the ViSQOL C ABI (include/visqol.h).
 *
 * Entry points the reference has no C declaration for but that a host
 * binding this backend needs: batches with device-resident inputs and the
 * discrete decisions of each pair (the reference's backend.Engine
 * measureBatch, src/backend.zig:78-82, and its GPU pipeline's lag/match
 * read-backs, src/gpu/pipeline.zig:223-283), per-stage device timing, and
 * single-stage entry points that run one kernel family on host buffers (the
 * reference's accel.Cpu stage jobs, src/accel.zig:21-146). Plain pointers
 * and sizes only. All functions return VISQOL_OK or a negative visqol.h
 * error code and set visqol_last_error().
 */
#ifndef VISQOL_B200_H
#define VISQOL_B200_H

#include "visqol.h"

#ifdef __cplusplus
extern "C" {
#endif

/* visqol_b200_measure_batch flags. */
enum {
    /* refs/degs are device pointers (cudaMalloc'd on the context's GPU). */
    VISQOL_B200_DEVICE_INPUTS = 1u << 0,
};

/* Discrete decisions and work counts of one measured pair. */
typedef struct {
    int64_t global_lag;            /* envelope xcorr lag in samples (0 if not run) */
    double spl_factor;             /* degraded SPL scale factor, 1 when unscaled */
    uint64_t deg_len;              /* aligned degraded length */
    uint64_t nf_ref, nf_deg;       /* spectrogram frames */
    uint64_t num_patches;
    const int64_t *ref_index;      /* per patch: reference start frame */
    const int64_t *deg_offset;     /* per patch: DP-matched degraded frame */
    const uint8_t *valid;          /* per patch: DP match valid */
    const int64_t *realign_lag;    /* per patch: slice envelope lag (0 if not run) */
    const int64_t *realign_frames; /* per patch: trimmed frames, -1 if not run */
    const uint8_t *realign_reused; /* per patch: bit0 ref / bit1 deg frames copied */
    const uint8_t *realign_accepted;
    uint64_t n_rms;                /* gammatone (frame, band) evaluations */
    uint64_t n_rms_window;         /* samples per evaluation */
    uint64_t n_cells;              /* NSIM cells evaluated */
    double fft_nlogn;              /* sum of n*log2(n) over complex FFTs */
} visqol_b200_trace;

/* Device time of the last batch on a context, by stage (CUDA events on the
 * context's stream), plus the counts behind the roofline figures. */
typedef struct {
    double total_ms;               /* first launch to last result copy */
    double lag_ms;                 /* envelopes, FFT xcorr, argmax (global) */
    double spectrogram_ms;         /* gammatone of full signals */
    double prep_ms;                /* dB, floors, joint minimum */
    double nsim_ms;                /* planes, NSIM table, DP, match stats */
    double realign_ms;             /* slice lags, realigned spectrograms, stats */
    double gammatone_kernel_ms;    /* sum of gammatone kernel durations */
    uint64_t gammatone_launches;
    uint64_t gammatone_rms;        /* (frame, band) RMS evaluations launched */
    uint64_t gammatone_window;     /* samples per evaluation */
    uint64_t kernel_launches;      /* all kernels of the batch */
    uint64_t h2d_bytes, d2h_bytes;
    uint64_t host_syncs;
    double lag_kernel_ms;          /* the global lag search's kernels, first to last */
    uint64_t lag_bytes;            /* their algorithmic DRAM bytes (signals, transform passes) */
    uint64_t lag_reruns;           /* FP32 form: lag searches the f32 pass left undecided */
} visqol_b200_timing;

/* Score n pairs as visqol_measure_batch does; with traces non-NULL,
 * traces[i] receives pair i's decisions (free with visqol_b200_trace_free).
 * flags: VISQOL_B200_DEVICE_INPUTS. */
int visqol_b200_measure_batch(visqol_ctx *ctx, size_t n,
                              const double *const *refs, const size_t *ref_lens,
                              const double *const *degs, const size_t *deg_lens,
                              uint32_t sample_rate, uint32_t flags,
                              visqol_result **out, int32_t *status,
                              visqol_b200_trace **traces);
void visqol_b200_trace_free(visqol_b200_trace *trace);

/* Scores n pairs as visqol_b200_measure_batch does and also d moslqo / d
 * degraded signal of each (reference backend.Engine.measureBatchGrad,
 * src/backend.zig:101-109): grads[i], a host buffer of deg_lens[i]
 * doubles (NULL: pair i's gradient is skipped), receives the gradient with
 * respect to each degraded sample. The forward pass's discrete choices are
 * held fixed: the global and per-patch lags, the patch matches and the
 * realignment decisions, and which cells the spectrogram floors and the
 * joint minimum select. Where the MOS mapping is clamped the gradient is
 * zero. The speech lattice mapper's own gradient is by central
 * differences over its features, as the reference's. */
int visqol_b200_measure_batch_grad(visqol_ctx *ctx, size_t n,
                                   const double *const *refs, const size_t *ref_lens,
                                   const double *const *degs, const size_t *deg_lens,
                                   uint32_t sample_rate, uint32_t flags,
                                   visqol_result **out, int32_t *status, double *const *grads);
int visqol_b200_last_timing(visqol_ctx *ctx, visqol_b200_timing *out);

/* ---- prepared references ---------------------------------------------------
 * The reference-side work (samples, envelope statistics and spectrogram on
 * the device; patch indices, VAD in speech mode) done once for references
 * that are scored against many degraded signals (the reference's
 * backend.Engine.prepare / measurePrepared, src/backend.zig:84-97,
 * src/visqol.zig:194-244). Prepared with one context; usable by any context
 * of the same device, mode and precision. Results equal those of
 * visqol_measure_batch on the same pairs. */
typedef struct visqol_b200_prepared visqol_b200_prepared;

/* flags: VISQOL_B200_DEVICE_INPUTS (refs are device pointers). A reference
 * that cannot be scored (too short, no patches) makes every pair scored
 * against it fail with its code. */
int visqol_b200_prepare(visqol_ctx *ctx, size_t n, const double *const *refs, const size_t *ref_lens,
                        uint32_t sample_rate, uint32_t flags, visqol_b200_prepared **out);
/* degs[i] against prepared reference ref_index[i] (ref_index NULL: i), as
 * visqol_measure_batch: out[i] NULL and status[i] set on failure, the first
 * error returned. flags: VISQOL_B200_DEVICE_INPUTS (degs on the device). */
int visqol_b200_measure_prepared(visqol_ctx *ctx, const visqol_b200_prepared *prepared, size_t n,
                                 const size_t *ref_index, const double *const *degs, const size_t *deg_lens,
                                 uint32_t flags, visqol_result **out, int32_t *status);
void visqol_b200_prepared_free(visqol_b200_prepared *prepared);

/* ---- request server: continuous batching on one GPU ---------------------
 * No counterpart in the reference (its batch call is synchronous). Requests
 * are submitted one at a time from any thread and complete asynchronously.
 * A pool of lanes (engines with their own streams) runs on the GPU at once;
 * a lane that finishes a batch immediately takes the requests queued
 * meanwhile (oldest first, one mode and sample rate per batch) up to
 * max_batch pairs and its share of the HBM budget, estimated per pair from
 * the signal lengths. So requests that arrive while others are on the GPU
 * are admitted as lanes and memory free up, and their work overlaps the
 * other lanes' work on the device. Results do not depend on which requests
 * share a batch. */
typedef struct visqol_b200_server visqol_b200_server;

typedef struct {
    uint64_t hbm_budget_bytes; /* device memory for in-flight pairs; 0: half of the free memory */
    uint32_t lanes;            /* concurrent batches; 0: 4 */
    uint32_t max_batch;        /* pairs per batch; 0: 64 */
} visqol_b200_serve_config;

typedef struct {
    uint64_t submitted, completed, failed, queued, in_flight;
    uint64_t batches;               /* batches run */
    uint64_t hbm_budget_bytes;      /* admission budget (all lanes) */
    uint64_t hbm_in_flight_bytes;   /* estimated footprint of the pairs on the GPU now */
    uint64_t hbm_reserved_bytes;    /* device memory the lanes hold */
    double latency_p50_ms, latency_p99_ms, latency_mean_ms; /* submit -> result, completed since reset */
    double queue_p50_ms, queue_p99_ms;                     /* submit -> admitted */
    double mean_batch;              /* pairs per batch */
} visqol_b200_serve_stats;

/* Server for the options' precision, radius and flags; `mode` of opts is
 * ignored (each request names its own). Speech requests are mapped with the
 * TF-Lattice model when use_lattice_model is set, else the exponential fit;
 * model_path applies to the lattice model when it is set, else to the SVR. */
int visqol_b200_server_create(const visqol_options *opts, const visqol_b200_serve_config *cfg,
                              visqol_b200_server **out);
/* Stops taking requests, finishes those admitted, frees everything (results
 * not yet collected are freed too). */
void visqol_b200_server_destroy(visqol_b200_server *s);
/* Queue one pair (mode VISQOL_MODE_AUDIO or _SPEECH). Host signals are
 * copied before the call returns; with VISQOL_B200_DEVICE_INPUTS the device
 * pointers must stay valid until the request completes. A pair whose
 * estimated footprint exceeds one lane's share of the budget fails with
 * VISQOL_E_OUT_OF_MEMORY. */
int visqol_b200_server_submit(visqol_b200_server *s, uint32_t mode, const double *ref, size_t ref_len,
                              const double *deg, size_t deg_len, uint32_t sample_rate, uint32_t flags,
                              uint64_t *ticket);
/* Next completed request in completion order, waiting up to timeout_ms
 * (< 0: no limit). Returns VISQOL_OK with *ticket, *status (the pair's
 * code) and *out (NULL on failure; free with visqol_result_free), or
 * VISQOL_B200_PENDING when nothing completed in time. */
#define VISQOL_B200_PENDING 1
int visqol_b200_server_next(visqol_b200_server *s, int32_t timeout_ms, uint64_t *ticket, int32_t *status,
                            visqol_result **out);
/* Device memory one pair of these lengths may take in a batch (an upper
 * bound of its arena use): the unit of the server's HBM admission. */
int visqol_b200_pair_footprint(size_t ref_len, size_t deg_len, uint32_t sample_rate, uint32_t mode,
                               uint64_t *bytes);

/* Counters and latency percentiles; reset != 0 clears the latency samples
 * and the batch counters after reading. The server keeps two doubles per
 * completed request (latency, queueing) until a reset, so a long-running
 * caller resets periodically. */
int visqol_b200_server_stats(visqol_b200_server *s, visqol_b200_serve_stats *out, int reset);

/* The speech-mode TF-Lattice MOS mapping alone, on the host (reference
 * src/lattice.zig:14-71): nb values per feature; model_path NULL or "" for
 * the bundled model. No GPU needed. */
int visqol_b200_lattice_predict(const char *model_path, size_t nb, const double *fvnsim,
                                const double *fvnsim10, const double *fstdnsim,
                                const double *fvdegenergy, double *mos);

/* Launch shapes the autotuner has chosen in this process: *n_rows rows of
 * {device, kernel (0 gammatone frames per CTA, 1 NSIM-table offsets per
 * CTA, 2 lag-search column passes: 0 shared-memory tiles, 1 registers, 3
 * FP32-form gammatone: CTAs per SM (its register budget), + 100 for the
 * persistent form that takes its tiles from a device-side work queue, 4
 * FP64-FMA-form gammatone: 0 its own kernel, 1 on the FP32 kernel's staged
 * tiles), variant a (form / cell arithmetic / log2 transform size), variant b
 * (bands / raw signals), choice},
 * written to rows up to max_rows. Each kernel class is measured on its
 * first batch per device (candidate shapes write identical results);
 * VISQOL_AUTOTUNE=0 keeps the default shapes. */
int visqol_b200_autotune_choices(int32_t *rows, size_t max_rows, size_t *n_rows);

/* Device name, SM count and compute capability of the context's GPU. */
int visqol_b200_device_info(int device, char *name, size_t name_len,
                            int *sm_count, int *cc_major, int *cc_minor);

/* Measured arithmetic peak of the current GPU in TFLOP/s, the denominator
 * of the roofline fractions: kind 0 = f64 multiply and add as separate
 * instructions (the exact form's arithmetic), 1 = f64 FMA, 2 = f32 FMA. */
int visqol_b200_peak(int kind, double *tflops);

/* ---- single-stage entry points (host buffers in and out, exact f64) ----
 * Each runs the same kernels the batch pipeline uses. */

/* Gammatone spectrogram, row-major [nb][nf] (reference
 * src/gammatone.zig:432-467). coeffs: nb x {a0,a11,a12,a13,a14,b1,b2,gain}
 * ascending. Returns the frame count in *nf. */
int visqol_b200_spectrogram(size_t nb, const double *coeffs, const double *hann,
                            size_t window, size_t hop, const double *x, size_t len,
                            double *out, size_t *nf);

/* Upper-envelope FFT cross-correlation lag (reference src/accel.zig:100-107,
 * src/xcorr.zig:197-251). */
int visqol_b200_envelope_lag(const double *a, size_t la, const double *b, size_t lb,
                             int64_t *lag);

/* A signal's serial statistics, each in the CPU's left-to-right f64
 * summation order, bit for bit: out[0] = sum x, out[1] = sum (-1)^k
 * (x - out[0] / len) (upperEnvelope's Nyquist bin, reference
 * src/envelope.zig:28-41), out[2] = sum x*x (reference src/audio.zig:132-136),
 * out[3] = the first k with x[k]*x[k] != 0 (len if none), out[4] = sum x*x
 * over x[skip..] (the energy of a lag-aligned signal, src/realign.zig:91-110).
 * skip <= len. */
int visqol_b200_signal_sums(const double *x, size_t len, size_t skip, double *out);

/* Raw-signal FFT cross-correlation lag (reference src/xcorr.zig:197-251). */
int visqol_b200_best_lag(const double *a, size_t la, const double *b, size_t lb,
                         int64_t *lag);

/* The lag search of one pair in an arithmetic form: form 0 the exact f64
 * search (as visqol_b200_envelope_lag / visqol_b200_best_lag), form 1 the
 * search every form's batches run: the correlation in f32, every lag within twice its error
 * bound of the maximum rescored by f64 dot products, first maximum in
 * ascending lag (reference refineLag / rescore, src/xcorr.zig:270-340, and
 * the GPU flow src/gpu/engine.zig:445-540). raw: 1 for the signals
 * themselves, 0 for their upper envelopes. *undecided (optional) is 1 when
 * the f32 pass found more than 64 candidates or a near-tie and the exact
 * search decided.
 * corr (optional, form 1): receives the f32 correlation's real part
 * (n x the circular cross-correlation, n = fftSizeFor(max(la, lb)) =
 * corr_len values). */
int visqol_b200_lag_search(const double *a, size_t la, const double *b, size_t lb, int raw, int form,
                           int64_t *lag, int32_t *undecided, float *corr, size_t corr_len);

/* refineLag (reference src/xcorr.zig:278-300) on the device: approx[i]
 * (n values) approximates scale * sum_t s1[t + i] s2[t] (circular index i)
 * within tol * (|s1|^2 + |s2|^2) * scale; the lags within twice that of
 * the largest |approx| are rescored by f64 dot products. *decided is 0
 * (and *lag untouched) when more than 64 qualify, the reference's null. */
int visqol_b200_refine_lag(const double *s1, size_t l1, const double *s2, size_t l2, const float *approx,
                           size_t n, double scale, double tol, int64_t *lag, int32_t *decided);

/* out[i] = num[i] / den[i] by the FP32 and FP64-FMA forms' NSIM quotient: a
 * reciprocal estimate refined by Markstein's Newton-Raphson steps, then one
 * correction of the quotient. For den[i] > 0 in [2^-1000, 2^1000] the
 * result is within one ulp of the IEEE quotient. */
int visqol_b200_nsim_quotient(const double *num, const double *den, size_t n, double *out);

/* Reverse of measurePatchSimilarity (reference src/nsim.zig:427-510), on the
 * host: for nrows x ncols prepared ref and deg cells and the gradients with
 * respect to the patch's band means, standard deviations and deg energies
 * (each nrows values, or NULL for zero), accumulates the gradients with
 * respect to the cells into dref and ddeg. */
int visqol_b200_patch_similarity_grad(const double *ref, const double *deg, size_t nrows, size_t ncols,
                                      const double *dmeans, const double *dstddevs, const double *denergy,
                                      double *dref, double *ddeg);

/* Reverse of prepareForComparison (reference src/spectrogram.zig:69-80), on
 * the host: from the raw spectrograms (nb x nfr, nb x nfd) and the
 * gradients with respect to the prepared cells, accumulates the gradient
 * with respect to the raw degraded cells into g_deg_raw. The cells the
 * floors and the joint minimum select are those of the forward pass. */
int visqol_b200_prepare_grad(const double *ref_raw, const double *deg_raw, size_t nb, size_t nfr, size_t nfd,
                             const double *g_ref, const double *g_deg, double *g_deg_raw);

/* Unscaled radix-2 DIF forward (natural in, bit-reversed out) and DIT
 * inverse, in place on n interleaved complex values (reference
 * src/dsp/fft.zig:127-166). */
int visqol_b200_fft(double *buf, size_t n, int inverse);

/* dB, per-frame floor, joint minimum in place (reference
 * src/spectrogram.zig:69-80); nb from 1 to 32 bands. */
int visqol_b200_prepare_for_comparison(double *ref, double *deg, size_t nb,
                                       size_t nf_ref, size_t nf_deg);

/* 10*log10 as the dB conversion computes it on the device. */
int visqol_b200_log10(const double *x, size_t n, double *out);

/* NSIM of each reference patch at each degraded offset in [lo, hi]:
 * out[p*nf_deg + off] (reference src/accel.zig:126-146). */
int visqol_b200_nsim_table(const double *ref_spec, size_t nf_ref,
                           const double *deg_spec, size_t nf_deg, size_t nb,
                           size_t patch, size_t np, const int64_t *ref_idx,
                           const int64_t *lo, const int64_t *hi, double *out);

/* DP and backtrack over a similarity table (reference src/dp.zig:216-352):
 * matched offset and validity per patch; *reached counts patches visited. */
int visqol_b200_dp(const double *sims, size_t np, size_t nf_deg,
                   const int64_t *lo, const int64_t *hi,
                   int64_t *offset, uint8_t *valid, size_t *reached);

/* visqol_b200_dp without device allocation. No counterpart in the
 * reference: it exists for callers that cannot allocate device memory at
 * call time (a process whose caching allocator already holds the free HBM,
 * or one that cannot let cudaFree wait for the whole device). Its device
 * buffers come from one ~6 MiB array reserved in the library image.
 * Limits: np <= 2048 and np * nf_deg <= 262144, else
 * VISQOL_E_INVALID_ARGUMENT. The first call on a device resolves the array
 * (make it before any stream capture); calls that overlap in time on one
 * device share the array and race, so serialise them. Same arguments and
 * results as visqol_b200_dp. */
int visqol_b200_dp_static(const double *sims, size_t np, size_t nf_deg,
                          const int64_t *lo, const int64_t *hi,
                          int64_t *offset, uint8_t *valid, size_t *reached);

/* Per-band NSIM statistics of one patch pair (reference
 * src/nsim.zig:427-510); *mean gets the mean of the band means. */
int visqol_b200_patch_similarity(const double *ref, const double *deg,
                                 size_t nrows, size_t ncols, double *means,
                                 double *stddevs, double *deg_energy, double *mean);

#ifdef __cplusplus
}
#endif

#endif /* VISQOL_B200_H */
