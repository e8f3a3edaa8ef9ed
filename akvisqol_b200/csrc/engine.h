// Batched ViSQOL pipeline on one GPU.
#pragma once

#include <cstddef>
#include <cstdint>
#include <functional>
#include <tuple>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "device.cuh"
#include "host_model.h"
#include "kernels.h"

namespace vqb {

namespace detail {
struct PairState;  // one pair's state through measure_batch (engine.cu)
}

struct Options {
    bool speech = false;
    int32_t radius = 60;
    bool unscaled_speech = false;
    bool disable_global_alignment = false;
    bool disable_realignment = false;
    // Arithmetic form (kFormExact, kFormF32, kFormF64).
    int32_t form = kFormExact;
    // Lag searches by the f64 transform throughout. Otherwise (every form)
    // the f32 transform nominates the near-maxima, f64 dot products rescore
    // them, and the searches that leaves undecided (near-ties, more than
    // kLagCandCap candidates) rerun with the f64 transform: the same lags.
    bool exact_lag_search = false;
};

struct PairTrace {
    int64_t global_lag = 0;
    double spl_factor = 1.0;
    uint64_t deg_len = 0, nf_ref = 0, nf_deg = 0;
    std::vector<int64_t> ref_index, deg_offset, realign_lag, realign_frames;
    std::vector<uint8_t> valid, realign_reused, realign_accepted;
    uint64_t n_rms = 0, n_rms_window = 0, n_cells = 0;
    double fft_nlogn = 0;
};

struct PairOutcome {
    int code = 0;
    std::string message;
    host::Scores scores;
    PairTrace trace;
    std::vector<double> grad;  // d moslqo / d degraded sample (deg_len), when requested
};

// Algorithmic DRAM bytes of one lag search (f32: the f32-nominated search).
uint64_t lag_search_bytes(const LagJob &j, bool f32);

struct Timing {
    double total_ms = 0, lag_ms = 0, spectrogram_ms = 0, prep_ms = 0, nsim_ms = 0, realign_ms = 0;
    double gammatone_kernel_ms = 0;
    uint64_t gammatone_launches = 0, gammatone_rms = 0, gammatone_window = 0;
    uint64_t kernel_launches = 0, h2d_bytes = 0, d2h_bytes = 0, host_syncs = 0;
    uint64_t lag_reruns = 0;  // f32 lag searches left undecided and rerun exactly
    double lag_kernel_ms = 0;  // the global lag search's kernels (events around them)
    uint64_t lag_bytes = 0;    // their algorithmic DRAM bytes
};

// Device memory that grows by whole chunks and is recycled per batch.
class Arena {
public:
    ~Arena();
    void reset();
    // Frees every chunk (the device must be done with them).
    void release();
    void *alloc(size_t bytes);
    template <class T>
    T *alloc_n(size_t n) {
        return static_cast<T *>(alloc(n * sizeof(T)));
    }
    size_t reserved() const;

private:
    struct Chunk {
        char *base;
        size_t size, used;
    };
    std::vector<Chunk> chunks_;
    size_t current_ = 0;
};

// Page-locked host memory with the same policy.
class PinnedArena {
public:
    ~PinnedArena();
    void reset();
    void *alloc(size_t bytes);
    template <class T>
    T *alloc_n(size_t n) {
        return static_cast<T *>(alloc(n * sizeof(T)));
    }

private:
    struct Chunk {
        char *base;
        size_t size, used;
    };
    std::vector<Chunk> chunks_;
    size_t current_ = 0;
};

// A reference scored against many degraded signals: the work that depends
// only on it, done once (reference src/visqol.zig:194-244, the prepared
// references of src/gpu/pipeline.zig:336-472): its samples, envelope
// statistics and raw spectrogram on the device, its patch indices (VAD in
// speech mode) on the host. Computed by Engine::prepare in the engine's
// form; device buffers are owned here.
struct PreparedRef {
    int code = 0;  // non-zero: the reference itself cannot be scored
    std::string message;
    int device = 0;
    size_t len = 0, nf = 0;
    double *d_sig = nullptr, *d_stats = nullptr, *d_spec = nullptr;
    double stats[4] = {};  // host copy of d_stats: sum, nyquist term, energy, -
    std::vector<int64_t> idx;
    ~PreparedRef();
};

class Engine {
public:
    Engine(int device, const Options &opt, std::shared_ptr<const host::Svr> svr,
           std::shared_ptr<const host::LatticeMapper> lattice = nullptr);
    ~Engine();
    Engine(const Engine &) = delete;
    Engine &operator=(const Engine &) = delete;

    // Score n pairs at one sample rate. Pointers are host memory unless
    // device_inputs. Per-pair failures land in out[i].code.
    // With prepared non-NULL, pair i whose prepared[i] is set takes its
    // reference from there (refs[i] and ref_lens[i] are ignored).
    // host_refs (device inputs only, may be NULL): host copies of the
    // references, read by the speech-mode VAD instead of a read-back.
    // grads: also d moslqo / d degraded signal of each pair scored
    // (PairOutcome::grad), the forward's discrete decisions fixed.
    void measure_batch(size_t n, const double *const *refs, const size_t *ref_lens, const double *const *degs,
                       const size_t *deg_lens, uint32_t sample_rate, bool device_inputs,
                       std::vector<PairOutcome> &out, const PreparedRef *const *prepared = nullptr,
                       const double *const *host_refs = nullptr, bool grads = false);
    // Host inputs scored in consecutive chunks of growing size: chunk k+1's
    // signals are copied to the device on a copy stream (from a helper
    // thread, so pageable sources do not block scoring) while chunk k is
    // scored, so the host-to-device transfer overlaps the GPU work instead of
    // preceding it. Results are identical to measure_batch with host inputs
    // (every pair's result depends only on its own signals). Small batches
    // take the direct path.
    void measure_batch_streamed(size_t n, const double *const *refs, const size_t *ref_lens,
                                const double *const *degs, const size_t *deg_lens, uint32_t sample_rate,
                                std::vector<PairOutcome> &out, const PreparedRef *const *prepared = nullptr);
    // Reference-side work of n references in this engine's form and mode.
    void prepare(size_t n, const double *const *refs, const size_t *ref_lens, uint32_t sample_rate,
                 bool device_inputs, std::vector<std::unique_ptr<PreparedRef>> &out);
    const Options &options() const { return opt_; }

    const Timing &last_timing() const { return timing_; }
    // Upper bound on the device memory one pair of these lengths takes in
    // measure_batch (host inputs included), for admission by footprint.
    static size_t pair_footprint(size_t ref_len, size_t deg_len, uint32_t sample_rate, bool speech);
    // Device memory the engine holds now (arena chunks, upload slots).
    size_t reserved_bytes() const { return arena_.reserved() + slot_bytes_[0] + slot_bytes_[1]; }
    // Waits for this engine's work, then frees its arena and upload slots;
    // the next batch allocates them again.
    void release_device_memory();
    int device() const { return device_; }
    cudaStream_t stream() const { return stream_; }

    // Single-stage entry points (device buffers, exact form).
    void spectrogram(const host::Filterbank &fb, const double *d_hann, size_t window, size_t hop, const double *d_x,
                     size_t len, double *d_out, size_t nf);
    // status_out (optional, njobs): FP32 form, 1 where the f32 search left
    // the job to the exact one.
    void lags(size_t njobs, const VSig *a, const VSig *b, bool raw, int64_t *h_lags, int32_t *status_out = nullptr,
              float *d_corr = nullptr);
    // The f32 search's nomination and f64 rescoring on a caller-supplied
    // approximate correlation of raw signals a and b (n values, device),
    // with the given slack; energy = |a|^2 + |b|^2. Returns false when it
    // leaves the lag undecided.
    bool refine_approx(const VSig &a, const VSig &b, const float *d_approx, int64_t n, double slack, double energy,
                       int64_t *lag);
    // FFT twiddles of size n on the device: the full table and the block
    // passes' compact one (cached per size).
    struct Twiddles {
        const double2 *top, *block, *cols, *stages;
        const float2 *block32, *cols32, *stages32;  // the same tables rounded to f32 (the f32 search)
    };
    Twiddles twiddles(size_t n);

private:
    struct RateCache {
        host::Filterbank fb;
        host::Geometry geo;
        BandCoeffs *d_coeffs = nullptr;
        FastBandCoeffs *d_fast_coeffs = nullptr;
        double *d_hann = nullptr;
    };
    // Envelope statistics of sum jobs: serial (exact) or tree (fast).
    void launch_sums(const std::vector<SumJob> &sums);
    // The launch shape for a kernel class among candidates: measured on the
    // caller's jobs at first use per device (launch(c) launches them with
    // shape c on st), then reused; candidates[0] when autotuning is off.
    enum TuneKernel {
        kTuneGammatone = 0,
        kTuneTable = 1,
        kTuneLagColumns = 2,
        kTuneGammatoneFastCtas = 3,
        kTuneGammatoneF64Staged = 4
    };
    // VISQOL_TUNE_<kernel> may fix the shape to one of `allowed` (default:
    // the candidates).
    int tuned(int kernel, int a, int b, const std::vector<int> &candidates, const std::function<void(int)> &launch,
              cudaStream_t st, const std::vector<int> *allowed = nullptr);
    // Gammatone spectrograms of the jobs in this engine's form on stream st;
    // returns the RMS count.
    uint64_t launch_spectrograms(const std::vector<SpecJob> &jobs, const RateCache &rc, cudaStream_t st,
                                 cudaEvent_t begin = nullptr, cudaEvent_t end = nullptr);
    const RateCache &rate_cache(uint32_t sample_rate);
    // d moslqo / d degraded signal of the pairs measure_batch just scored
    // (grad_ok), into out[i].grad: the host reverses of the MOS mapping,
    // NSIM statistics and spectrogram preparation, the gammatone reverse on
    // the device, then the SPL scaling's and the lag's reverses on the host.
    void gradients(detail::PairState *ps, size_t n, const size_t *deg_lens, const RateCache &rc,
                   std::vector<PairOutcome> &out);

    // Envelope (or raw) lag search for jobs whose a/b/stat pointers are set;
    // lags land in the jobs' lag_out (device). Launches only. The FP32 form
    // (unless `exact`) runs the f32 search and returns a device array of one
    // status word per job, in job order: 1 where the f32 search left the job
    // undecided (its lag_out is untouched); the caller reads it back with the
    // lags and passes it to rerun_undecided. Else returns null.
    int32_t *launch_lag_jobs(std::vector<LagJob> &jobs, bool raw, bool exact = false);
    // The jobs whose status (host copy) is 1, rerun with the exact search;
    // returns their indices (launches only; nothing when none).
    std::vector<size_t> rerun_undecided(const std::vector<LagJob> &jobs, const int32_t *h_status, bool raw);
    template <class T>
    T *upload(const std::vector<T> &v);
    void *upload_bytes(const void *src, size_t bytes);
    void d2h(void *dst, const void *src, size_t bytes);
    void sync();
    void record(cudaEvent_t e);
    float elapsed(cudaEvent_t a, cudaEvent_t b);

    int device_;
    Options opt_;
    std::shared_ptr<const host::Svr> svr_;
    std::shared_ptr<const host::LatticeMapper> lattice_;
    size_t nb_, patch_;
    double max_freq_;
    cudaStream_t stream_ = nullptr;
    Arena arena_;
    PinnedArena pinned_;
    std::map<uint32_t, RateCache> rates_;
    std::map<size_t, Twiddles> twiddles_;
    std::vector<cudaEvent_t> events_;
    cudaStream_t side_ = nullptr;    // reference spectrograms, concurrent with the lag phase
    cudaEvent_t ev_inputs_ = nullptr, ev_ref_done_ = nullptr;
    cudaEvent_t gt_events_[6] = {};  // begin/end of up to three gammatone launches
    cudaEvent_t lag_events_[2] = {};  // begin/end of the global lag search
    Timing timing_;
    // measure_batch_streamed: copy stream, two upload slots (grow-only
    // device buffers) and the events that mark each slot's upload done.
    cudaStream_t copy_ = nullptr;
    cudaEvent_t ev_up_[2] = {};
    cudaEvent_t ev_piece_ = nullptr;  // the upload copy in flight
    double *slot_[2] = {};
    size_t slot_bytes_[2] = {};
};

// The autotuner's choices so far: (device, kernel, variant a, variant b,
// chosen shape).
std::vector<std::tuple<int, int, int, int, int>> autotune_choices();

// CUDA call check: throws Error(kBackend) with the call and message.
void cuda_check(cudaError_t e, const char *what);

// The calling thread's visqol_last_error() text.
void set_last_error(const std::string &message);
#define VQB_CUDA(call) ::vqb::cuda_check((call), #call)

}  // namespace vqb
