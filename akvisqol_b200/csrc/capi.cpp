// C ABI of libvisqol (include/visqol.h, include/visqol_b200.h).
//
// Mirrors the reference's src/capi.zig:119-456: options with defaults,
// thread-local last-error text, heap-boxed results that own their arrays,
// per-pair status in batches (the first error is the return value), and
// files grouped by sample rate. The engine behind it is the GPU pipeline;
// there is no CPU fallback.
#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <map>
#include <memory>
#include <mutex>
#include <set>
#include <string>
#include <thread>
#include <tuple>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/visqol.h"
#include "../../include/visqol_b200.h"
#include "capi_internal.h"
#include "engine.h"
#include "host_model.h"

using vqb::Error;

// A context owns one or more lanes: engines with their own streams and
// memory on the same GPU (VISQOL_GPU_LANES, default 6; the reference's GPU
// engine runs two, src/gpu/engine.zig:551-591). A batch is split across the
// lanes and the lanes run concurrently from host threads, so one lane's
// serial phases, host planning and uploads overlap another's kernels. On one
// B200 the device-resident rate of a 128-pair batch of 10 s 48 kHz pairs is
// the same for 2, 4 and 6 lanes; with host inputs, 6 lanes score it ~5%
// faster than 4 (the uploads hide behind more concurrent chunks).
// References prepared once for many degraded signals (visqol_b200_prepare).
struct visqol_b200_prepared {
    int device = 0;
    vqb::Options opt;
    uint32_t sample_rate = 0;
    std::vector<std::unique_ptr<vqb::PreparedRef>> refs;
};

// Device staging for host-input batches scored through the shared chunk
// queue (run_lanes_queued): a grow-only buffer for a whole batch's signals,
// a copy stream and one event per chunk (created on first use).
struct HostStaging {
    int device = 0;
    double *buf = nullptr;
    size_t bytes = 0;
    cudaStream_t copy = nullptr;
    cudaEvent_t piece = nullptr;
    std::vector<cudaEvent_t> chunk_done;
    ~HostStaging() {
        cudaSetDevice(device);
        if (copy) cudaStreamSynchronize(copy);
        for (auto e : chunk_done) cudaEventDestroy(e);
        if (piece) cudaEventDestroy(piece);
        if (copy) cudaStreamDestroy(copy);
        cudaFree(buf);
    }
};

struct visqol_ctx {
    vqb::Options opt;
    std::shared_ptr<const vqb::host::Svr> svr;
    std::vector<std::unique_ptr<vqb::Engine>> lanes;
    vqb::Timing timing;
    std::unique_ptr<HostStaging> staging;
};

namespace {

// The calling thread's last error, 512 bytes as the reference's
// (src/capi.zig:85-91).
thread_local char g_error[512] = {0};

void set_error(const std::string &m) { std::snprintf(g_error, sizeof g_error, "%s", m.c_str()); }

int fail(int code, const std::string &m) {
    set_error(m);
    return code;
}

}  // namespace

// A result and the storage its pointers view (reference src/capi.zig:66-70).
struct Box {
    visqol_result c{};
    vqb::host::Scores s;
    std::vector<double> band_data;
    std::vector<visqol_patch> patches;
};

visqol_result *vqb::box_result(vqb::host::Scores &&s) {
    auto *b = new Box();
    b->s = std::move(s);
    const size_t nb = b->s.fvnsim.size(), np = b->s.patches.size();
    b->band_data.resize(np * nb * 3);
    b->patches.resize(np);
    for (size_t i = 0; i < np; ++i) {
        const auto &m = b->s.patches[i];
        double *dst = b->band_data.data() + i * nb * 3;
        std::copy(m.means.begin(), m.means.end(), dst);
        std::copy(m.stddevs.begin(), m.stddevs.end(), dst + nb);
        std::copy(m.energy.begin(), m.energy.end(), dst + 2 * nb);
        b->patches[i] = visqol_patch{m.similarity, m.ref_start, m.ref_end, m.deg_start, m.deg_end,
                                     dst, dst + nb, dst + 2 * nb};
    }
    b->c.moslqo = b->s.moslqo;
    b->c.vnsim = b->s.vnsim;
    b->c.alignment_lag_s = b->s.lag_s;
    b->c.num_bands = nb;
    b->c.fvnsim = b->s.fvnsim.data();
    b->c.fvnsim10 = b->s.fvnsim10.data();
    b->c.fstdnsim = b->s.fstdnsim.data();
    b->c.fvdegenergy = b->s.fvdegenergy.data();
    b->c.center_freq_bands = b->s.cf.data();
    b->c.num_patches = np;
    b->c.patch_sims = b->patches.data();
    return &b->c;
}

namespace {

struct TraceBox {
    visqol_b200_trace c{};
    vqb::PairTrace t;
};

visqol_b200_trace *box_trace(vqb::PairTrace &&t) {
    auto *b = new TraceBox();
    b->t = std::move(t);
    visqol_b200_trace &c = b->c;
    c.global_lag = b->t.global_lag;
    c.spl_factor = b->t.spl_factor;
    c.deg_len = b->t.deg_len;
    c.nf_ref = b->t.nf_ref;
    c.nf_deg = b->t.nf_deg;
    c.num_patches = b->t.ref_index.size();
    c.ref_index = b->t.ref_index.data();
    c.deg_offset = b->t.deg_offset.data();
    c.valid = b->t.valid.data();
    c.realign_lag = b->t.realign_lag.data();
    c.realign_frames = b->t.realign_frames.data();
    c.realign_reused = b->t.realign_reused.data();
    c.realign_accepted = b->t.realign_accepted.data();
    c.n_rms = b->t.n_rms;
    c.n_rms_window = b->t.n_rms_window;
    c.n_cells = b->t.n_cells;
    c.fft_nlogn = b->t.fft_nlogn;
    return &b->c;
}

int device_count() {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

// Whether a batch of this kind (device, form, mode, sample rate) has run in
// this process. The first one scores its first share on one lane alone, so
// that the autotuner's measurements (made on that first batch's jobs) are
// not timed beside other lanes' kernels; the rest then runs concurrently.
bool first_of_its_kind(const visqol_ctx *c, uint32_t sample_rate) {
    static std::mutex mu;
    static std::set<std::tuple<int, int, bool, uint32_t>> seen;
    const auto key = std::make_tuple(c->lanes[0]->device(), (int)c->opt.form, c->opt.speech, sample_rate);
    std::lock_guard<std::mutex> lock(mu);
    return seen.insert(key).second;
}

// One lane's successive batches (chunks): spans and counts add up.
void add_batch_timing(vqb::Timing &a, const vqb::Timing &x) {
    a.total_ms += x.total_ms;
    a.lag_ms += x.lag_ms;
    a.spectrogram_ms += x.spectrogram_ms;
    a.prep_ms += x.prep_ms;
    a.nsim_ms += x.nsim_ms;
    a.realign_ms += x.realign_ms;
    a.gammatone_kernel_ms += x.gammatone_kernel_ms;
    a.gammatone_launches += x.gammatone_launches;
    a.gammatone_rms += x.gammatone_rms;
    a.gammatone_window = std::max(a.gammatone_window, x.gammatone_window);
    a.kernel_launches += x.kernel_launches;
    a.h2d_bytes += x.h2d_bytes;
    a.d2h_bytes += x.d2h_bytes;
    a.host_syncs += x.host_syncs;
    a.lag_kernel_ms += x.lag_kernel_ms;
    a.lag_bytes += x.lag_bytes;
    a.lag_reruns += x.lag_reruns;
}

// Lanes side by side: spans are the longest lane's, work counts add up.
void merge_lane_timing(vqb::Timing &t, const vqb::Timing &x) {
    t.total_ms = std::max(t.total_ms, x.total_ms);
    t.lag_ms = std::max(t.lag_ms, x.lag_ms);
    t.spectrogram_ms = std::max(t.spectrogram_ms, x.spectrogram_ms);
    t.prep_ms = std::max(t.prep_ms, x.prep_ms);
    t.nsim_ms = std::max(t.nsim_ms, x.nsim_ms);
    t.realign_ms = std::max(t.realign_ms, x.realign_ms);
    t.gammatone_kernel_ms += x.gammatone_kernel_ms;
    t.gammatone_launches += x.gammatone_launches;
    t.gammatone_rms += x.gammatone_rms;
    t.gammatone_window = std::max(t.gammatone_window, x.gammatone_window);
    t.kernel_launches += x.kernel_launches;
    t.h2d_bytes += x.h2d_bytes;
    t.d2h_bytes += x.d2h_bytes;
    t.host_syncs += x.host_syncs;
    t.lag_kernel_ms = std::max(t.lag_kernel_ms, x.lag_kernel_ms);
    t.lag_bytes += x.lag_bytes;
    t.lag_reruns += x.lag_reruns;
}

// Joins the threads it holds when it goes out of scope, so that an exception
// while starting them (a thread that cannot be created) never destroys a
// joinable std::thread; the threads' work ends by itself.
struct JoinAll {
    std::vector<std::thread> threads;
    ~JoinAll() {
        for (auto &t : threads)
            if (t.joinable()) t.join();
    }
};

// Host-input batches through all lanes at once: the signals go up in chunks
// of consecutive pairs, in order, on a copy stream of their own (one copy in
// flight, so the lanes' own small uploads never queue behind a whole chunk),
// and the lanes take chunks from a shared queue as they free up, each
// waiting on its chunk's upload. The GPU starts scoring when the first chunk
// has landed, the transfer of the rest overlaps the scoring, and every chunk
// is scored as one batch of a reasonable size. Returns false (nothing done)
// when the batch is too small to split or too large for one staging buffer;
// the caller then takes the per-lane path.
bool run_lanes_queued(visqol_ctx *c, size_t n, const double *const *refs, const size_t *ref_lens,
                      const double *const *degs, const size_t *deg_lens, uint32_t sample_rate,
                      std::vector<vqb::PairOutcome> &res, const vqb::PreparedRef *const *prepared) {
    const size_t L = c->lanes.size();
    auto up = [](size_t len) { return (len * sizeof(double) + 255) & ~size_t(255); };
    std::vector<size_t> ref_off(n, SIZE_MAX), deg_off(n, SIZE_MAX);
    size_t total = 0;
    for (size_t i = 0; i < n; ++i) {
        if (!(prepared && prepared[i]) && refs[i]) ref_off[i] = total, total += up(ref_lens[i]);
        if (degs[i]) deg_off[i] = total, total += up(deg_lens[i]);
    }
    // chunks per lane (VISQOL_STREAMED_CHUNKS overrides): more, smaller chunks
    // start every lane sooner and shorten the tail, but smaller lane batches
    // cost more (measured on one B200: 2 a lane scores a 128-pair batch of
    // 10 s pairs fastest, 3, 4 and 6 a lane 4-12% slower)
    size_t per_lane = 2;
    if (const char *env = std::getenv("VISQOL_STREAMED_CHUNKS"))
        per_lane = std::max<size_t>(1, std::min<size_t>(16, (size_t)std::strtoull(env, nullptr, 10)));
    const size_t K = std::min(n, per_lane * L);
    size_t min_bytes = size_t(64) << 20;  // VISQOL_STREAMED_MIN_BYTES overrides, as for the per-lane path
    if (const char *env = std::getenv("VISQOL_STREAMED_MIN_BYTES")) min_bytes = (size_t)std::strtoull(env, nullptr, 10);
    if (L < 2 || K < 2 || total < min_bytes || total > (size_t(16) << 30)) return false;
    const int device = c->lanes[0]->device();
    VQB_CUDA(cudaSetDevice(device));
    if (!c->staging) {
        c->staging = std::make_unique<HostStaging>();
        c->staging->device = device;
        VQB_CUDA(cudaStreamCreateWithFlags(&c->staging->copy, cudaStreamNonBlocking));
        VQB_CUDA(cudaEventCreateWithFlags(&c->staging->piece, cudaEventDisableTiming));
    }
    HostStaging &st = *c->staging;
    if (st.bytes < total) {
        VQB_CUDA(cudaStreamSynchronize(st.copy));
        if (st.buf) VQB_CUDA(cudaFree(st.buf));
        st.buf = nullptr;
        st.bytes = 0;
        VQB_CUDA(cudaMalloc(&st.buf, total));
        st.bytes = total;
    }
    while (st.chunk_done.size() < K) {
        cudaEvent_t e;
        VQB_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        st.chunk_done.push_back(e);
    }
    // chunks of consecutive pairs: the first L (one a lane) at front/100 of
    // the average size, so that every lane starts scoring soon after the
    // first uploads, and the rest of equal bytes (VISQOL_STREAMED_FRONT,
    // default 30; 0 gives equal chunks throughout). Measured on one B200
    // with 128 pairs of 10 s: 25-33% upload-and-score ~6% faster than equal
    // chunks, 20% and 50% in between.
    size_t front = 30;
    if (const char *env = std::getenv("VISQOL_STREAMED_FRONT")) front = (size_t)std::strtoull(env, nullptr, 10);
    std::vector<size_t> sizes(n);
    for (size_t i = 0; i < n; ++i)
        sizes[i] = (ref_off[i] != SIZE_MAX ? up(ref_lens[i]) : 0) + (deg_off[i] != SIZE_MAX ? up(deg_lens[i]) : 0);
    const std::vector<size_t> bounds = vqb::host::chunk_bounds(sizes, K, L, front);
    const size_t nk = bounds.size() - 1;
    char *base = reinterpret_cast<char *>(st.buf);
    std::vector<const double *> d_ref(n, nullptr), d_deg(n, nullptr);
    for (size_t i = 0; i < n; ++i) {
        if (ref_off[i] != SIZE_MAX) d_ref[i] = reinterpret_cast<const double *>(base + ref_off[i]);
        if (deg_off[i] != SIZE_MAX) d_deg[i] = reinterpret_cast<const double *>(base + deg_off[i]);
    }
    // uploader: chunk k's copies, then its event; `recorded` tells the lanes
    // (host side) that the event they will wait on has been recorded
    std::mutex mu;
    std::condition_variable cv;
    size_t recorded = 0;
    bool failed = false;
    std::exception_ptr upload_error;
    JoinAll uploader;
    uploader.threads.emplace_back([&] {
        try {
            VQB_CUDA(cudaSetDevice(device));
            size_t copies = 0;
            auto copy = [&](const double *dst, const double *src, size_t len) {
                if (!len) return;
                if (copies++) VQB_CUDA(cudaEventSynchronize(st.piece));
                VQB_CUDA(cudaMemcpyAsync(const_cast<double *>(dst), src, len * sizeof(double), cudaMemcpyHostToDevice,
                                         st.copy));
                VQB_CUDA(cudaEventRecord(st.piece, st.copy));
            };
            for (size_t k = 0; k < nk; ++k) {
                for (size_t i = bounds[k]; i < bounds[k + 1]; ++i) {
                    if (d_ref[i]) copy(d_ref[i], refs[i], ref_lens[i]);
                    if (d_deg[i]) copy(d_deg[i], degs[i], deg_lens[i]);
                }
                VQB_CUDA(cudaEventRecord(st.chunk_done[k], st.copy));
                std::lock_guard<std::mutex> lock(mu);
                recorded = k + 1;
                cv.notify_all();
            }
        } catch (...) {
            upload_error = std::current_exception();
            std::lock_guard<std::mutex> lock(mu);
            failed = true;
            cv.notify_all();
        }
    });
    std::atomic<size_t> next{0};
    std::vector<std::exception_ptr> errs(L);
    std::vector<vqb::Timing> lane_t(L);
    const bool alone_first = first_of_its_kind(c, sample_rate);
    // Lane l scores chunk k; false when the upload failed (reported below).
    auto score_chunk = [&](size_t l, size_t k) -> bool {
        try {
            vqb::Engine &e = *c->lanes[l];
            std::vector<vqb::PairOutcome> part;
            {
                std::unique_lock<std::mutex> lock(mu);
                cv.wait(lock, [&] { return recorded > k || failed; });
                if (recorded <= k) return false;
            }
            VQB_CUDA(cudaStreamWaitEvent(e.stream(), st.chunk_done[k], 0));
            const size_t b0 = bounds[k], m = bounds[k + 1] - b0;
            e.measure_batch(m, d_ref.data() + b0, ref_lens + b0, d_deg.data() + b0, deg_lens + b0, sample_rate,
                            true, part, prepared ? prepared + b0 : nullptr, refs + b0);
            for (size_t j = 0; j < m; ++j) res[b0 + j] = std::move(part[j]);
            add_batch_timing(lane_t[l], e.last_timing());
        } catch (...) {
            if (!errs[l]) errs[l] = std::current_exception();
            return false;
        }
        return true;
    };
    auto work = [&](size_t l) {
        for (size_t k = next++; k < nk; k = next++)
            if (!score_chunk(l, k)) return;
    };
    JoinAll lanes;
    if (alone_first) {
        // lane 0 scores chunk 0 alone (the autotuner measures there), then
        // all lanes share the remaining chunks
        next = 1;
        score_chunk(0, 0);
    }
    for (size_t l = 1; l < L; ++l) lanes.threads.emplace_back(work, l);
    work(0);
    for (auto &t : lanes.threads) t.join();
    uploader.threads[0].join();
    if (upload_error) std::rethrow_exception(upload_error);
    for (auto &e : errs)
        if (e) std::rethrow_exception(e);
    vqb::Timing t{};
    for (const vqb::Timing &x : lane_t) merge_lane_timing(t, x);
    for (size_t i = 0; i < n; ++i)
        t.h2d_bytes += (d_ref[i] ? ref_lens[i] : 0) * sizeof(double) + (d_deg[i] ? deg_lens[i] : 0) * sizeof(double);
    c->timing = t;
    return true;
}

// The batch across the context's lanes: pairs dealt longest-first to the
// least-loaded lane, lanes run concurrently, outcomes gathered back in order.
void run_lanes(visqol_ctx *c, size_t n, const double *const *refs, const size_t *ref_lens, const double *const *degs,
               const size_t *deg_lens, uint32_t sample_rate, bool device_inputs, std::vector<vqb::PairOutcome> &res,
               const vqb::PreparedRef *const *prepared = nullptr, bool grads = false) {
    const size_t L = std::min(c->lanes.size(), std::max<size_t>(1, n));
    res.assign(n, vqb::PairOutcome{});
    // Host inputs: uploads overlap scoring, through the shared chunk queue
    // when the batch splits, else lane by lane (gradients: signals uploaded
    // whole, the gradient pass reads them after scoring).
    const bool streamed = !device_inputs && !grads && vqb::env_streamed_uploads();
    if (streamed && run_lanes_queued(c, n, refs, ref_lens, degs, deg_lens, sample_rate, res, prepared)) return;
    auto measure = [&](vqb::Engine &e, size_t m, const double *const *r, const size_t *rl, const double *const *d,
                       const size_t *dl, std::vector<vqb::PairOutcome> &o, const vqb::PreparedRef *const *pr) {
        if (streamed)
            e.measure_batch_streamed(m, r, rl, d, dl, sample_rate, o, pr);
        else
            e.measure_batch(m, r, rl, d, dl, sample_rate, device_inputs, o, pr, nullptr, grads);
    };
    if (L <= 1) {
        measure(*c->lanes[0], n, refs, ref_lens, degs, deg_lens, res, prepared);
        c->timing = c->lanes[0]->last_timing();
        return;
    }
    // Device inputs through a chunk queue: lanes take chunks of consecutive
    // pairs as they free up, each lane's first chunk at 30% of the average,
    // so that the lanes fall out of step and their light phases (host
    // planning, small kernels) overlap other lanes' heavy ones instead of
    // coinciding. Measured on one B200 (128 pairs of 10 s): three chunks a
    // lane score the FP32 and FP64-FMA forms ~1% faster than one share a
    // lane; the exact form, whose lanes wait on serial sums, 6-17% slower
    // with chunks, so it keeps one share a lane. VISQOL_DEVICE_CHUNKS
    // overrides (chunks a lane, 0: one share a lane).
    size_t dev_chunks = c->opt.form == vqb::kFormExact ? 0 : 3;
    if (const char *env = std::getenv("VISQOL_DEVICE_CHUNKS"))
        dev_chunks = std::min<size_t>(16, (size_t)std::strtoull(env, nullptr, 10));
    if (device_inputs && !grads && dev_chunks > 0 && n >= dev_chunks * L) {
        std::vector<size_t> sizes(n);
        for (size_t i = 0; i < n; ++i) sizes[i] = ref_lens[i] + deg_lens[i];
        const std::vector<size_t> bounds = vqb::host::chunk_bounds(sizes, dev_chunks * L, L, 30);
        const size_t nk = bounds.size() - 1;
        std::atomic<size_t> next{0};
        std::vector<std::exception_ptr> errs(L);
        std::vector<vqb::Timing> lane_t(L);
        auto run_chunk = [&](size_t l, size_t k) {
            const size_t b0 = bounds[k], m = bounds[k + 1] - b0;
            std::vector<vqb::PairOutcome> part;
            c->lanes[l]->measure_batch(m, refs + b0, ref_lens + b0, degs + b0, deg_lens + b0, sample_rate, true, part,
                                       prepared ? prepared + b0 : nullptr);
            for (size_t j = 0; j < m; ++j) res[b0 + j] = std::move(part[j]);
            add_batch_timing(lane_t[l], c->lanes[l]->last_timing());
        };
        auto work = [&](size_t l) {
            try {
                for (size_t k = next++; k < nk; k = next++) run_chunk(l, k);
            } catch (...) {
                errs[l] = std::current_exception();
            }
        };
        JoinAll lanes;
        if (first_of_its_kind(c, sample_rate)) {
            next = 1;
            try {
                run_chunk(0, 0);
            } catch (...) {
                errs[0] = std::current_exception();
            }
        }
        for (size_t l = 1; l < L; ++l) lanes.threads.emplace_back(work, l);
        work(0);
        for (auto &th : lanes.threads) th.join();
        for (auto &e : errs)
            if (e) std::rethrow_exception(e);
        vqb::Timing t{};
        for (const vqb::Timing &x : lane_t) merge_lane_timing(t, x);
        c->timing = t;
        return;
    }
    std::vector<size_t> order(n);
    for (size_t i = 0; i < n; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) {
        return ref_lens[a] + deg_lens[a] > ref_lens[b] + deg_lens[b];
    });
    std::vector<std::vector<size_t>> part(L);
    std::vector<size_t> load(L, 0);
    for (size_t i : order) {
        const size_t l = (size_t)(std::min_element(load.begin(), load.end()) - load.begin());
        part[l].push_back(i);
        load[l] += ref_lens[i] + deg_lens[i];
    }
    std::vector<std::vector<vqb::PairOutcome>> lane_out(L);
    std::vector<std::exception_ptr> errs(L);
    const bool alone_first = first_of_its_kind(c, sample_rate);
    auto work = [&](size_t l) {
        try {
            const auto &ix = part[l];
            std::vector<const double *> r(ix.size()), d(ix.size());
            std::vector<size_t> rl(ix.size()), dl(ix.size());
            std::vector<const vqb::PreparedRef *> pr(prepared ? ix.size() : 0);
            for (size_t k = 0; k < ix.size(); ++k) {
                r[k] = refs[ix[k]], d[k] = degs[ix[k]], rl[k] = ref_lens[ix[k]], dl[k] = deg_lens[ix[k]];
                if (prepared) pr[k] = prepared[ix[k]];
            }
            measure(*c->lanes[l], ix.size(), r.data(), rl.data(), d.data(), dl.data(), lane_out[l],
                    prepared ? pr.data() : nullptr);
        } catch (...) {
            errs[l] = std::current_exception();
        }
    };
    JoinAll lanes;
    // the first batch of its kind: lane 0's share alone (the autotuner
    // measures there), then the other lanes
    if (alone_first) work(0);
    for (size_t l = 1; l < L; ++l) lanes.threads.emplace_back(work, l);
    if (!alone_first) work(0);
    for (auto &t : lanes.threads) t.join();
    for (auto &e : errs)
        if (e) std::rethrow_exception(e);
    vqb::Timing t{};
    for (size_t l = 0; l < L; ++l) {
        for (size_t k = 0; k < part[l].size(); ++k) res[part[l][k]] = std::move(lane_out[l][k]);
        merge_lane_timing(t, c->lanes[l]->last_timing());
    }
    c->timing = t;
}

// One batch through the engine with per-pair results and status.
int run_batch(visqol_ctx *c, size_t n, const double *const *refs, const size_t *ref_lens, const double *const *degs,
              const size_t *deg_lens, uint32_t sample_rate, bool device_inputs, visqol_result **out, int32_t *status,
              visqol_b200_trace **traces, const vqb::PreparedRef *const *prepared = nullptr,
              double *const *grads = nullptr) {
    std::vector<vqb::PairOutcome> res;
    try {
        run_lanes(c, n, refs, ref_lens, degs, deg_lens, sample_rate, device_inputs, res, prepared, grads != nullptr);
    } catch (const Error &e) {
        for (size_t i = 0; i < n; ++i) {
            out[i] = nullptr;
            if (status) status[i] = e.code;
            if (traces) traces[i] = nullptr;
        }
        return fail(e.code, e.what());
    } catch (const std::bad_alloc &) {
        return fail(VISQOL_E_OUT_OF_MEMORY, "OutOfMemory");
    } catch (const std::exception &e) {
        return fail(VISQOL_E_INTERNAL, e.what());
    }
    int first = VISQOL_OK;
    for (size_t i = 0; i < n; ++i) {
        out[i] = nullptr;
        if (traces) traces[i] = nullptr;
        int rc = res[i].code;
        if (rc == VISQOL_OK) {
            if (grads && grads[i] && res[i].grad.size() == deg_lens[i])
                std::copy(res[i].grad.begin(), res[i].grad.end(), grads[i]);
            out[i] = vqb::box_result(std::move(res[i].scores));
            if (traces) traces[i] = box_trace(std::move(res[i].trace));
        } else {
            set_error(res[i].message);
        }
        if (status) status[i] = rc;
        if (rc != VISQOL_OK && first == VISQOL_OK) first = rc;
    }
    if (first != VISQOL_OK) {
        for (size_t i = 0; i < n; ++i)
            if (res[i].code == first) {
                set_error(res[i].message);
                break;
            }
    }
    return first;
}

}  // namespace

void vqb::set_last_error(const std::string &message) { set_error(message); }

int vqb::engine_options(const visqol_options &o, Options *opt, std::shared_ptr<const host::Svr> *svr,
                        std::shared_ptr<const host::LatticeMapper> *lattice, std::string *message) {
    // EXACT (and AUTO, which resolves to exact on a device with native f64)
    // reproduce the CPU path; FAST runs the gammatone's later stages in f32;
    // BALANCED keeps f64 throughout but with FMA and reassociated sums.
    opt->form = o.precision == VISQOL_PRECISION_FAST       ? kFormF32
                : o.precision == VISQOL_PRECISION_BALANCED ? kFormF64
                                                           : kFormExact;
    opt->speech = o.mode == VISQOL_MODE_SPEECH;
    opt->radius = o.search_window_radius > 0 ? o.search_window_radius : 60;
    opt->unscaled_speech = o.use_unscaled_speech_mos_mapping != 0;
    opt->disable_global_alignment = o.disable_global_alignment != 0;
    opt->disable_realignment = o.disable_realignment != 0;
    (void)message;
    if (opt->speech && o.use_lattice_model) {
        // model_path names the lattice model in speech mode (reference src/capi.zig:189-203)
        const std::string bytes =
            (o.model_path && o.model_path[0]) ? host::read_file(o.model_path) : host::default_lattice_bytes();
        *lattice = std::make_shared<host::LatticeMapper>(bytes, 21);
    }
    if (!opt->speech) {
        const std::string text =
            (o.model_path && o.model_path[0]) ? host::read_file(o.model_path) : host::default_svr_text();
        *svr = std::make_shared<host::Svr>(host::parse_svr(text));
    }
    return VISQOL_OK;
}

int vqb::context_device(int *device, std::string *message) {
    const int ndev = device_count();
    if (ndev == 0) {
        *message = "BackendUnavailable: no CUDA device";
        return VISQOL_E_BACKEND;
    }
    // VISQOL_CUDA_DEVICE picks the GPU (one process per GPU); else device 0.
    int dev = 0;
    if (const char *env = std::getenv("VISQOL_CUDA_DEVICE")) dev = std::atoi(env);
    if (dev < 0 || dev >= ndev) {
        *message = "VISQOL_CUDA_DEVICE out of range";
        return VISQOL_E_INVALID_ARGUMENT;
    }
    *device = dev;
    return VISQOL_OK;
}

bool vqb::env_streamed_uploads() {
    const char *env = std::getenv("VISQOL_STREAMED_UPLOADS");
    return !(env && env[0] == '0');
}

int vqb::env_lanes(int fallback) {
    int lanes = fallback;
    if (const char *env = std::getenv("VISQOL_GPU_LANES")) lanes = std::atoi(env);
    return std::max(1, std::min(lanes, 8));
}

extern "C" {

uint32_t visqol_abi_version(void) { return VISQOL_ABI_VERSION; }

const char *visqol_version(void) { return "0.1.0-b200"; }

const char *visqol_last_error(void) { return g_error; }

uint32_t visqol_available_backends(void) { return device_count() > 0 ? (1u << VISQOL_BACKEND_CUDA) : 0u; }

void visqol_options_default(visqol_options *o) {
    if (!o) return;
    o->mode = VISQOL_MODE_AUDIO;
    o->search_window_radius = 60;
    o->use_unscaled_speech_mos_mapping = 0;
    o->disable_global_alignment = 0;
    o->disable_realignment = 0;
    o->use_lattice_model = 1;
    o->model_path = nullptr;
    o->backend = VISQOL_BACKEND_CUDA;
    o->precision = VISQOL_PRECISION_AUTO;
}

int visqol_create(const visqol_options *in, visqol_ctx **out) {
    if (!out) return fail(VISQOL_E_INVALID_ARGUMENT, "out is NULL");
    *out = nullptr;
    visqol_options o;
    visqol_options_default(&o);
    if (in) o = *in;
    if (o.mode > 1) return fail(VISQOL_E_INVALID_ARGUMENT, "invalid mode " + std::to_string(o.mode));
    if (o.backend > VISQOL_BACKEND_VULKAN) return fail(VISQOL_E_INVALID_ARGUMENT, "invalid backend " + std::to_string(o.backend));
    if (o.precision > VISQOL_PRECISION_AUTO)
        return fail(VISQOL_E_INVALID_ARGUMENT, "invalid precision " + std::to_string(o.precision));
    if (o.backend != VISQOL_BACKEND_CUDA)
        return fail(VISQOL_E_BACKEND, "BackendUnavailable: this libvisqol serves backend cuda (2) only");
    auto c = std::make_unique<visqol_ctx>();
    try {
        std::string msg;
        std::shared_ptr<const vqb::host::LatticeMapper> lattice;
        if (int rc = vqb::engine_options(o, &c->opt, &c->svr, &lattice, &msg)) return fail(rc, msg);
        int dev = 0;
        if (int rc = vqb::context_device(&dev, &msg)) return fail(rc, msg);
        const int lanes = vqb::env_lanes(6);
        for (int l = 0; l < lanes; ++l)
            c->lanes.push_back(std::make_unique<vqb::Engine>(dev, c->opt, c->svr, lattice));
    } catch (const Error &e) {
        return fail(e.code, e.what());
    } catch (const std::bad_alloc &) {
        return fail(VISQOL_E_OUT_OF_MEMORY, "OutOfMemory");
    } catch (const std::exception &e) {
        return fail(VISQOL_E_INTERNAL, e.what());
    }
    *out = c.release();
    return VISQOL_OK;
}

void visqol_destroy(visqol_ctx *c) { delete c; }

int visqol_measure(visqol_ctx *c, const double *ref, size_t ref_len, const double *deg, size_t deg_len,
                   uint32_t sample_rate, visqol_result **out) {
    if (!c) return fail(VISQOL_E_INVALID_ARGUMENT, "ctx is NULL");
    if (!out) return fail(VISQOL_E_INVALID_ARGUMENT, "out is NULL");
    *out = nullptr;
    if ((!ref && ref_len) || (!deg && deg_len)) return fail(VISQOL_E_INVALID_ARGUMENT, "signal pointer is NULL");
    int32_t st = 0;
    return run_batch(c, 1, &ref, &ref_len, &deg, &deg_len, sample_rate, false, out, &st, nullptr);
}

int visqol_measure_batch(visqol_ctx *c, size_t n, const double *const *refs, const size_t *ref_lens,
                         const double *const *degs, const size_t *deg_lens, uint32_t sample_rate, uint32_t num_threads,
                         visqol_result **out, int32_t *status) {
    (void)num_threads;
    if (!c) return fail(VISQOL_E_INVALID_ARGUMENT, "ctx is NULL");
    if (n == 0) return VISQOL_OK;
    if (!out) return fail(VISQOL_E_INVALID_ARGUMENT, "out is NULL");
    if (!refs) return fail(VISQOL_E_INVALID_ARGUMENT, "refs is NULL");
    if (!ref_lens) return fail(VISQOL_E_INVALID_ARGUMENT, "ref_lens is NULL");
    if (!degs) return fail(VISQOL_E_INVALID_ARGUMENT, "degs is NULL");
    if (!deg_lens) return fail(VISQOL_E_INVALID_ARGUMENT, "deg_lens is NULL");
    return run_batch(c, n, refs, ref_lens, degs, deg_lens, sample_rate, false, out, status, nullptr);
}

int visqol_measure_files(visqol_ctx *c, const char *ref_path, const char *deg_path, visqol_result **out) {
    if (!c) return fail(VISQOL_E_INVALID_ARGUMENT, "ctx is NULL");
    if (!out) return fail(VISQOL_E_INVALID_ARGUMENT, "out is NULL");
    *out = nullptr;
    if (!ref_path) return fail(VISQOL_E_INVALID_ARGUMENT, "ref_path is NULL");
    if (!deg_path) return fail(VISQOL_E_INVALID_ARGUMENT, "deg_path is NULL");
    uint32_t rr = 0, dr = 0;
    std::vector<double> r, d;
    try {
        r = vqb::host::decode_wav(vqb::host::read_file(ref_path), &rr);
    } catch (const Error &e) {
        return fail(e.code, std::string(ref_path) + ": " + e.what());
    }
    try {
        d = vqb::host::decode_wav(vqb::host::read_file(deg_path), &dr);
    } catch (const Error &e) {
        return fail(e.code, std::string(deg_path) + ": " + e.what());
    }
    if (rr != dr)
        return fail(VISQOL_E_SIGNAL, "Input audio signals have different sample rates! Reference audio sample rate: " +
                                         std::to_string(rr) + ". Degraded audio sample rate: " + std::to_string(dr));
    const double *rp = r.data(), *dp = d.data();
    const size_t rl = r.size(), dl = d.size();
    int32_t st = 0;
    return run_batch(c, 1, &rp, &rl, &dp, &dl, rr, false, out, &st, nullptr);
}

int visqol_measure_files_batch(visqol_ctx *c, size_t n, const char *const *ref_paths, const char *const *deg_paths,
                               uint32_t num_threads, visqol_result **out, int32_t *status) {
    (void)num_threads;
    if (!c) return fail(VISQOL_E_INVALID_ARGUMENT, "ctx is NULL");
    if (n == 0) return VISQOL_OK;
    if (!out) return fail(VISQOL_E_INVALID_ARGUMENT, "out is NULL");
    if (!ref_paths) return fail(VISQOL_E_INVALID_ARGUMENT, "ref_paths is NULL");
    if (!deg_paths) return fail(VISQOL_E_INVALID_ARGUMENT, "deg_paths is NULL");
    std::vector<std::vector<double>> r(n), d(n);
    std::vector<uint32_t> rate(n, 0);
    std::vector<int32_t> codes(n, VISQOL_OK);
    for (size_t i = 0; i < n; ++i) {
        out[i] = nullptr;
        uint32_t rr = 0, dr = 0;
        try {
            r[i] = vqb::host::decode_wav(vqb::host::read_file(ref_paths[i]), &rr);
        } catch (const Error &e) {
            codes[i] = fail(e.code, std::string(ref_paths[i]) + ": " + e.what());
            continue;
        }
        try {
            d[i] = vqb::host::decode_wav(vqb::host::read_file(deg_paths[i]), &dr);
        } catch (const Error &e) {
            codes[i] = fail(e.code, std::string(deg_paths[i]) + ": " + e.what());
            continue;
        }
        rate[i] = rr;
        if (rr != dr) {
            codes[i] = fail(VISQOL_E_SIGNAL, "pair " + std::to_string(i) + ": reference and degraded sample rates differ (" +
                                                 std::to_string(rr) + " vs " + std::to_string(dr) + ")");
        }
    }
    std::map<uint32_t, std::vector<size_t>> groups;
    for (size_t i = 0; i < n; ++i)
        if (codes[i] == VISQOL_OK) groups[rate[i]].push_back(i);
    for (auto &g : groups) {
        const size_t m = g.second.size();
        std::vector<const double *> rp(m), dp(m);
        std::vector<size_t> rl(m), dl(m);
        for (size_t k = 0; k < m; ++k) {
            const size_t i = g.second[k];
            rp[k] = r[i].data(), dp[k] = d[i].data(), rl[k] = r[i].size(), dl[k] = d[i].size();
        }
        std::vector<visqol_result *> res(m, nullptr);
        std::vector<int32_t> st(m, 0);
        run_batch(c, m, rp.data(), rl.data(), dp.data(), dl.data(), g.first, false, res.data(), st.data(), nullptr);
        for (size_t k = 0; k < m; ++k) {
            out[g.second[k]] = res[k];
            codes[g.second[k]] = st[k];
        }
    }
    int first = VISQOL_OK;
    for (size_t i = 0; i < n; ++i) {
        if (status) status[i] = codes[i];
        if (codes[i] != VISQOL_OK && first == VISQOL_OK) first = codes[i];
    }
    return first;
}

void visqol_result_free(visqol_result *r) {
    if (!r) return;
    delete reinterpret_cast<Box *>(r);
}

int visqol_b200_measure_batch_grad(visqol_ctx *c, size_t n, const double *const *refs, const size_t *ref_lens,
                                   const double *const *degs, const size_t *deg_lens, uint32_t sample_rate,
                                   uint32_t flags, visqol_result **out, int32_t *status, double *const *grads) {
    if (!c) return fail(VISQOL_E_INVALID_ARGUMENT, "ctx is NULL");
    if (n == 0) return VISQOL_OK;
    if (!out || !grads) return fail(VISQOL_E_INVALID_ARGUMENT, "out or grads is NULL");
    if (!refs || !degs || !ref_lens || !deg_lens) return fail(VISQOL_E_INVALID_ARGUMENT, "NULL signal table");
    return run_batch(c, n, refs, ref_lens, degs, deg_lens, sample_rate, (flags & VISQOL_B200_DEVICE_INPUTS) != 0, out,
                     status, nullptr, nullptr, grads);
}

int visqol_b200_measure_batch(visqol_ctx *c, size_t n, const double *const *refs, const size_t *ref_lens,
                              const double *const *degs, const size_t *deg_lens, uint32_t sample_rate, uint32_t flags,
                              visqol_result **out, int32_t *status, visqol_b200_trace **traces) {
    if (!c) return fail(VISQOL_E_INVALID_ARGUMENT, "ctx is NULL");
    if (n == 0) return VISQOL_OK;
    if (!out || !refs || !ref_lens || !degs || !deg_lens) return fail(VISQOL_E_INVALID_ARGUMENT, "NULL argument");
    return run_batch(c, n, refs, ref_lens, degs, deg_lens, sample_rate, (flags & VISQOL_B200_DEVICE_INPUTS) != 0, out,
                     status, traces);
}

int visqol_b200_prepare(visqol_ctx *c, size_t n, const double *const *refs, const size_t *ref_lens,
                        uint32_t sample_rate, uint32_t flags, visqol_b200_prepared **out) {
    if (!c || !out) return fail(VISQOL_E_INVALID_ARGUMENT, "NULL argument");
    *out = nullptr;
    if (n && (!refs || !ref_lens)) return fail(VISQOL_E_INVALID_ARGUMENT, "NULL argument");
    if (sample_rate == 0) return fail(VISQOL_E_INVALID_ARGUMENT, "sample_rate is 0");
    try {
        auto p = std::make_unique<visqol_b200_prepared>();
        p->device = c->lanes[0]->device();
        p->opt = c->opt;
        p->sample_rate = sample_rate;
        c->lanes[0]->prepare(n, refs, ref_lens, sample_rate, (flags & VISQOL_B200_DEVICE_INPUTS) != 0, p->refs);
        *out = p.release();
        return VISQOL_OK;
    } catch (const Error &e) {
        return fail(e.code, e.what());
    } catch (const std::bad_alloc &) {
        return fail(VISQOL_E_OUT_OF_MEMORY, "OutOfMemory");
    } catch (const std::exception &e) {
        return fail(VISQOL_E_INTERNAL, e.what());
    }
}

void visqol_b200_prepared_free(visqol_b200_prepared *p) { delete p; }

int visqol_b200_measure_prepared(visqol_ctx *c, const visqol_b200_prepared *p, size_t n, const size_t *ref_index,
                                 const double *const *degs, const size_t *deg_lens, uint32_t flags,
                                 visqol_result **out, int32_t *status) {
    if (!c || !p) return fail(VISQOL_E_INVALID_ARGUMENT, "NULL argument");
    if (n == 0) return VISQOL_OK;
    if (!out || !degs || !deg_lens) return fail(VISQOL_E_INVALID_ARGUMENT, "NULL argument");
    if (p->device != c->lanes[0]->device() || p->opt.form != c->opt.form || p->opt.speech != c->opt.speech)
        return fail(VISQOL_E_INVALID_ARGUMENT, "prepared references come from a context of another device, "
                                               "mode or precision");
    std::vector<const vqb::PreparedRef *> prep(n);
    std::vector<const double *> rp(n, nullptr);
    std::vector<size_t> rl(n);
    for (size_t i = 0; i < n; ++i) {
        const size_t k = ref_index ? ref_index[i] : i;
        if (k >= p->refs.size()) return fail(VISQOL_E_INVALID_ARGUMENT, "ref_index out of range");
        prep[i] = p->refs[k].get();
        rl[i] = prep[i]->len;
    }
    return run_batch(c, n, rp.data(), rl.data(), degs, deg_lens, p->sample_rate,
                     (flags & VISQOL_B200_DEVICE_INPUTS) != 0, out, status, nullptr, prep.data());
}

int visqol_b200_lattice_predict(const char *model_path, size_t nb, const double *fvnsim, const double *fvnsim10,
                                const double *fstdnsim, const double *fvdegenergy, double *mos) {
    if (!fvnsim || !fvnsim10 || !fstdnsim || !fvdegenergy || !mos || nb == 0)
        return fail(VISQOL_E_INVALID_ARGUMENT, "NULL argument");
    try {
        static std::mutex mu;
        static std::map<std::pair<std::string, size_t>, std::shared_ptr<const vqb::host::LatticeMapper>> cache;
        const std::string path = model_path ? model_path : "";
        std::shared_ptr<const vqb::host::LatticeMapper> m;
        {
            std::lock_guard<std::mutex> lock(mu);
            auto &slot = cache[{path, nb}];
            if (!slot)
                slot = std::make_shared<vqb::host::LatticeMapper>(
                    path.empty() ? vqb::host::default_lattice_bytes() : vqb::host::read_file(path), nb);
            m = slot;
        }
        *mos = m->predict(fvnsim, fvnsim10, fstdnsim, fvdegenergy);
        return VISQOL_OK;
    } catch (const Error &e) {
        return fail(e.code, e.what());
    } catch (const std::exception &e) {
        return fail(VISQOL_E_INTERNAL, e.what());
    }
}

int visqol_b200_autotune_choices(int32_t *rows, size_t max_rows, size_t *n_rows) {
    if (!n_rows) return fail(VISQOL_E_INVALID_ARGUMENT, "NULL argument");
    const auto all = vqb::autotune_choices();
    *n_rows = all.size();
    for (size_t i = 0; i < all.size() && i < max_rows && rows; ++i) {
        int32_t *r = rows + 5 * i;
        r[0] = std::get<0>(all[i]);
        r[1] = std::get<1>(all[i]);
        r[2] = std::get<2>(all[i]);
        r[3] = std::get<3>(all[i]);
        r[4] = std::get<4>(all[i]);
    }
    return VISQOL_OK;
}

void visqol_b200_trace_free(visqol_b200_trace *t) {
    if (!t) return;
    delete reinterpret_cast<TraceBox *>(t);
}

int visqol_b200_last_timing(visqol_ctx *c, visqol_b200_timing *out) {
    if (!c || !out) return fail(VISQOL_E_INVALID_ARGUMENT, "NULL argument");
    const vqb::Timing &t = c->timing;
    out->total_ms = t.total_ms;
    out->lag_ms = t.lag_ms;
    out->spectrogram_ms = t.spectrogram_ms;
    out->prep_ms = t.prep_ms;
    out->nsim_ms = t.nsim_ms;
    out->realign_ms = t.realign_ms;
    out->gammatone_kernel_ms = t.gammatone_kernel_ms;
    out->gammatone_launches = t.gammatone_launches;
    out->gammatone_rms = t.gammatone_rms;
    out->gammatone_window = t.gammatone_window;
    out->kernel_launches = t.kernel_launches;
    out->h2d_bytes = t.h2d_bytes;
    out->d2h_bytes = t.d2h_bytes;
    out->host_syncs = t.host_syncs;
    out->lag_kernel_ms = t.lag_kernel_ms;
    out->lag_bytes = t.lag_bytes;
    out->lag_reruns = t.lag_reruns;
    return VISQOL_OK;
}

int visqol_b200_device_info(int device, char *name, size_t name_len, int *sm_count, int *cc_major, int *cc_minor) {
    if (device_count() <= device) return fail(VISQOL_E_BACKEND, "no such CUDA device");
    cudaDeviceProp p;
    if (cudaGetDeviceProperties(&p, device) != cudaSuccess) return fail(VISQOL_E_BACKEND, "cudaGetDeviceProperties failed");
    if (name && name_len) std::snprintf(name, name_len, "%s", p.name);
    if (sm_count) *sm_count = p.multiProcessorCount;
    if (cc_major) *cc_major = p.major;
    if (cc_minor) *cc_minor = p.minor;
    return VISQOL_OK;
}

}  // extern "C"
