// Request server: continuous batching of ViSQOL pairs on one GPU
// (include/visqol_b200.h, visqol_b200_server_*).
//
// Requests enter one FIFO queue. A fixed pool of lanes runs on the GPU side
// by side; each lane owns one engine per mode (its own streams and device
// arena) and a host thread. A lane that is free takes the oldest queued
// request, then every further queued request of the same mode and sample
// rate, oldest first, while the batch stays within max_batch pairs and the
// HBM the other lanes leave free, and runs the batch through its engine. A
// lane that finishes goes straight back to the queue, so requests that
// arrived while others were on the GPU are admitted as soon as a lane and
// memory free up, and up to `lanes` batches overlap on the device. Under
// light load batches are small (low latency); under heavy load they grow to
// max_batch (high throughput).
//
// HBM is one pool: the budget is shared by all lanes, each counting what its
// engines hold (their arenas grow to the largest batch they ran and are
// reused) or, while it runs a batch, the larger of that and the batch's
// footprint (pair footprints are upper bounds estimated from the signal
// lengths). A request larger than what the other lanes leave makes idle
// lanes give their memory back, then waits for the busy ones; only a pair
// larger than the whole budget is refused.
//
// The pipeline's results for a pair do not depend on the other pairs of its
// batch (each kernel job reads and writes only its own pair's buffers), so a
// request scores the same alone and in any mix.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/visqol_b200.h"
#include "capi_internal.h"
#include "engine.h"

namespace {

using Clock = std::chrono::steady_clock;

double ms_between(Clock::time_point a, Clock::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
}

struct Request {
    uint64_t ticket = 0;
    uint32_t mode = 0, sample_rate = 0;
    bool device = false;
    std::vector<double> ref, deg;       // host copies
    const double *ref_ptr = nullptr, *deg_ptr = nullptr;
    size_t ref_len = 0, deg_len = 0;
    size_t footprint = 0;
    Clock::time_point submitted, admitted;
};

struct Done {
    uint64_t ticket;
    int32_t status;
    visqol_result *result;
};

double percentile(std::vector<double> v, double q) {
    if (v.empty()) return 0.0;
    std::sort(v.begin(), v.end());
    const double pos = q * (double)(v.size() - 1);
    const size_t i = (size_t)pos;
    const double f = pos - (double)i;
    return i + 1 < v.size() ? v[i] * (1.0 - f) + v[i + 1] * f : v[i];
}

}  // namespace

struct visqol_b200_server {
    int device = 0;
    vqb::Options opt[2];  // audio, speech
    std::shared_ptr<const vqb::host::Svr> svr;
    std::shared_ptr<const vqb::host::LatticeMapper> lattice;  // speech requests, when enabled
    uint64_t budget = 0;
    uint32_t max_batch = 64;

    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    bool stopping = false;
    std::deque<std::unique_ptr<Request>> queue;
    std::deque<Done> done;
    uint64_t next_ticket = 1;
    uint64_t submitted = 0, completed = 0, failed = 0, in_flight = 0, in_flight_bytes = 0, batches = 0,
             batch_pairs = 0;
    uint64_t gen = 0;  // bumped (under mu) when the queue or a lane's memory changes
    std::vector<double> latency, queueing;

    struct Lane {
        std::unique_ptr<vqb::Engine> engine[2];
        std::thread thread;
        uint64_t reserved = 0;  // device memory its engines hold (under mu)
        uint64_t inflight = 0;  // footprint of the batch it runs (under mu)
        bool busy = false;
    };

    // HBM of the budget that the lanes other than `self` leave (under mu).
    uint64_t pool_available(const Lane &self) const {
        uint64_t held = 0;
        for (auto &l : lanes)
            if (l.get() != &self) held += l->busy ? std::max(l->reserved, l->inflight) : l->reserved;
        return budget > held ? budget - held : 0;
    }
    std::vector<std::unique_ptr<Lane>> lanes;

    // Stops the lanes (each finishes its batch in flight and what is still
    // queued) and joins them: visqol_b200_server_destroy, and the cleanup
    // when creation fails after some lanes started.
    ~visqol_b200_server() {
        {
            std::lock_guard<std::mutex> lock(mu);
            stopping = true;
        }
        cv_work.notify_all();
        for (auto &l : lanes)
            if (l->thread.joinable()) l->thread.join();
        for (auto &d : done) visqol_result_free(d.result);
    }

    vqb::Engine &engine(Lane &l, uint32_t mode) {
        auto &e = l.engine[mode];
        if (!e) e = std::make_unique<vqb::Engine>(device, opt[mode], mode == 0 ? svr : nullptr,
                                                  mode == 0 ? nullptr : lattice);
        return *e;
    }

    void lane_loop(Lane &lane) {
        cudaSetDevice(device);
        for (;;) {
            std::vector<std::unique_ptr<Request>> batch;
            bool release = false;
            {
                std::unique_lock<std::mutex> lock(mu);
                for (;;) {
                    if (queue.empty()) {
                        if (stopping) return;  // stopping and drained
                        const uint64_t g = gen;
                        cv_work.wait(lock, [&] { return stopping || gen != g; });
                        continue;
                    }
                    const uint64_t avail = pool_available(lane);
                    if (queue.front()->footprint <= avail) {
                        admit(lane, avail, batch);
                        break;
                    }
                    // The oldest request does not fit beside what the other
                    // lanes hold: hand this idle lane's memory back, or wait
                    // for another lane to finish or to hand its memory back
                    // (idle lanes holding memory are woken to do so).
                    if (lane.reserved > 0) {
                        release = true;
                        break;
                    }
                    const uint64_t g = gen;
                    cv_work.notify_all();
                    cv_work.wait(lock, [&] { return gen != g; });
                }
            }
            if (release) {
                for (auto &e : lane.engine)
                    if (e) e->release_device_memory();
                {
                    std::lock_guard<std::mutex> lock(mu);
                    lane.reserved = 0;
                    ++gen;
                }
                cv_work.notify_all();
                continue;
            }
            run(lane, batch);
        }
    }

    // The oldest request and every further queued one of its mode, sample
    // rate and input kind, oldest first, within max_batch pairs and `avail`
    // bytes (under mu; the oldest fits).
    void admit(Lane &lane, uint64_t avail, std::vector<std::unique_ptr<Request>> &batch) {
        const uint32_t mode = queue.front()->mode, sr = queue.front()->sample_rate;
        const bool dev = queue.front()->device;
        uint64_t bytes = 0;
        for (auto it = queue.begin(); it != queue.end() && batch.size() < max_batch;) {
            Request &r = **it;
            if (r.mode == mode && r.sample_rate == sr && r.device == dev && bytes + r.footprint <= avail) {
                bytes += r.footprint;
                batch.push_back(std::move(*it));
                it = queue.erase(it);
            } else {
                ++it;
            }
        }
        const auto now = Clock::now();
        for (auto &r : batch) {
            r->admitted = now;
            queueing.push_back(ms_between(r->submitted, now));
        }
        lane.busy = true;
        lane.inflight = bytes;
        in_flight += batch.size();
        in_flight_bytes += bytes;
        ++batches;
        batch_pairs += batch.size();
        ++gen;
    }

    void run(Lane &lane, std::vector<std::unique_ptr<Request>> &batch) {
        const size_t n = batch.size();
        std::vector<const double *> r(n), d(n);
        std::vector<size_t> rl(n), dl(n);
        uint64_t bytes = 0;
        for (size_t i = 0; i < n; ++i) {
            const Request &q = *batch[i];
            r[i] = q.device ? q.ref_ptr : q.ref.data();
            d[i] = q.device ? q.deg_ptr : q.deg.data();
            rl[i] = q.ref_len;
            dl[i] = q.deg_len;
            bytes += q.footprint;
        }
        std::vector<vqb::PairOutcome> out;
        int batch_code = VISQOL_OK;
        try {
            engine(lane, batch[0]->mode)
                .measure_batch(n, r.data(), rl.data(), d.data(), dl.data(), batch[0]->sample_rate,
                               batch[0]->device, out);
        } catch (const vqb::Error &e) {
            batch_code = e.code;
        } catch (const std::bad_alloc &) {
            batch_code = VISQOL_E_OUT_OF_MEMORY;
        } catch (const std::exception &) {
            batch_code = VISQOL_E_INTERNAL;
        }
        std::vector<Done> finished(n);
        for (size_t i = 0; i < n; ++i) {
            int32_t code = batch_code;
            visqol_result *res = nullptr;
            if (code == VISQOL_OK) {
                code = out[i].code;
                if (code == VISQOL_OK) {
                    try {
                        res = vqb::box_result(std::move(out[i].scores));
                    } catch (const std::bad_alloc &) {
                        code = VISQOL_E_OUT_OF_MEMORY;
                    }
                }
            }
            finished[i] = Done{batch[i]->ticket, code, res};
        }
        const auto now = Clock::now();
        {
            std::lock_guard<std::mutex> lock(mu);
            for (size_t i = 0; i < n; ++i) {
                latency.push_back(ms_between(batch[i]->submitted, now));
                if (finished[i].status == VISQOL_OK)
                    ++completed;
                else
                    ++failed;
                done.push_back(finished[i]);
            }
            in_flight -= n;
            in_flight_bytes -= bytes;
            lane.reserved = 0;
            for (auto &e : lane.engine)
                if (e) lane.reserved += e->reserved_bytes();
            lane.busy = false;
            lane.inflight = 0;
            ++gen;
        }
        cv_done.notify_all();
        cv_work.notify_all();
    }
};

namespace {

int fail(int code, const std::string &m) {
    vqb::set_last_error(m);
    return code;
}

}  // namespace

extern "C" {

int visqol_b200_server_create(const visqol_options *opts, const visqol_b200_serve_config *cfg,
                              visqol_b200_server **out) {
    if (!out) return fail(VISQOL_E_INVALID_ARGUMENT, "out is NULL");
    *out = nullptr;
    visqol_options o;
    visqol_options_default(&o);
    if (opts) o = *opts;
    if (o.backend != VISQOL_BACKEND_CUDA)
        return fail(VISQOL_E_BACKEND, "BackendUnavailable: this libvisqol serves backend cuda (2) only");
    if (o.precision > VISQOL_PRECISION_AUTO) return fail(VISQOL_E_INVALID_ARGUMENT, "invalid precision");
    visqol_b200_serve_config c{};
    if (cfg) c = *cfg;
    auto s = std::make_unique<visqol_b200_server>();
    try {
        std::string msg;
        visqol_options audio = o, speech = o;
        audio.mode = VISQOL_MODE_AUDIO;
        speech.mode = VISQOL_MODE_SPEECH;
        // one model_path: the lattice model's when speech uses the lattice, else the SVR's
        if (o.use_lattice_model) audio.model_path = nullptr;
        std::shared_ptr<const vqb::host::LatticeMapper> no_lattice;
        if (int rc = vqb::engine_options(audio, &s->opt[0], &s->svr, &no_lattice, &msg)) return fail(rc, msg);
        std::shared_ptr<const vqb::host::Svr> none;
        if (int rc = vqb::engine_options(speech, &s->opt[1], &none, &s->lattice, &msg)) return fail(rc, msg);
        if (int rc = vqb::context_device(&s->device, &msg)) return fail(rc, msg);
        VQB_CUDA(cudaSetDevice(s->device));
        size_t free_b = 0, total_b = 0;
        VQB_CUDA(cudaMemGetInfo(&free_b, &total_b));
        s->budget = c.hbm_budget_bytes ? c.hbm_budget_bytes : free_b / 2;
        if (s->budget > free_b) return fail(VISQOL_E_OUT_OF_MEMORY, "hbm_budget_bytes exceeds the free device memory");
        const uint32_t lanes = c.lanes ? std::min<uint32_t>(c.lanes, 16) : 4;
        s->max_batch = c.max_batch ? c.max_batch : 64;
        for (uint32_t l = 0; l < lanes; ++l) s->lanes.push_back(std::make_unique<visqol_b200_server::Lane>());
        visqol_b200_server *raw = s.get();
        for (auto &l : s->lanes) {
            auto *lane = l.get();
            lane->thread = std::thread([raw, lane] { raw->lane_loop(*lane); });
        }
    } catch (const vqb::Error &e) {
        return fail(e.code, e.what());
    } catch (const std::bad_alloc &) {
        return fail(VISQOL_E_OUT_OF_MEMORY, "OutOfMemory");
    } catch (const std::exception &e) {
        return fail(VISQOL_E_INTERNAL, e.what());
    }
    *out = s.release();
    return VISQOL_OK;
}

void visqol_b200_server_destroy(visqol_b200_server *s) { delete s; }

int visqol_b200_pair_footprint(size_t ref_len, size_t deg_len, uint32_t sample_rate, uint32_t mode,
                               uint64_t *bytes) {
    if (!bytes || sample_rate == 0 || mode > VISQOL_MODE_SPEECH)
        return fail(VISQOL_E_INVALID_ARGUMENT, "invalid argument");
    *bytes = vqb::Engine::pair_footprint(ref_len, deg_len, sample_rate, mode == VISQOL_MODE_SPEECH);
    return VISQOL_OK;
}

int visqol_b200_server_submit(visqol_b200_server *s, uint32_t mode, const double *ref, size_t ref_len,
                              const double *deg, size_t deg_len, uint32_t sample_rate, uint32_t flags,
                              uint64_t *ticket) {
    if (!s || !ticket) return fail(VISQOL_E_INVALID_ARGUMENT, "NULL argument");
    if (mode > VISQOL_MODE_SPEECH) return fail(VISQOL_E_INVALID_ARGUMENT, "invalid mode");
    if ((!ref && ref_len) || (!deg && deg_len)) return fail(VISQOL_E_INVALID_ARGUMENT, "signal pointer is NULL");
    if (sample_rate == 0) return fail(VISQOL_E_INVALID_ARGUMENT, "sample_rate is 0");
    auto r = std::make_unique<Request>();
    r->mode = mode;
    r->sample_rate = sample_rate;
    r->device = (flags & VISQOL_B200_DEVICE_INPUTS) != 0;
    r->ref_len = ref_len;
    r->deg_len = deg_len;
    try {
        r->footprint = vqb::Engine::pair_footprint(ref_len, deg_len, sample_rate, mode == VISQOL_MODE_SPEECH);
        if (r->footprint > s->budget)
            return fail(VISQOL_E_OUT_OF_MEMORY, "pair exceeds the server's HBM budget");
        if (r->device) {
            r->ref_ptr = ref;
            r->deg_ptr = deg;
        } else {
            r->ref.assign(ref, ref + ref_len);
            r->deg.assign(deg, deg + deg_len);
        }
    } catch (const vqb::Error &e) {
        return fail(e.code, e.what());
    } catch (const std::bad_alloc &) {
        return fail(VISQOL_E_OUT_OF_MEMORY, "OutOfMemory");
    }
    r->submitted = Clock::now();
    {
        std::lock_guard<std::mutex> lock(s->mu);
        r->ticket = s->next_ticket++;
        *ticket = r->ticket;
        if (s->stopping) return fail(VISQOL_E_INVALID_ARGUMENT, "server is stopping");
        ++s->submitted;
        s->queue.push_back(std::move(r));
        ++s->gen;
    }
    s->cv_work.notify_all();
    return VISQOL_OK;
}

int visqol_b200_server_next(visqol_b200_server *s, int32_t timeout_ms, uint64_t *ticket, int32_t *status,
                            visqol_result **out) {
    if (!s || !ticket || !status || !out) return fail(VISQOL_E_INVALID_ARGUMENT, "NULL argument");
    *out = nullptr;
    std::unique_lock<std::mutex> lock(s->mu);
    auto ready = [&] { return !s->done.empty(); };
    if (timeout_ms < 0)
        s->cv_done.wait(lock, ready);
    else if (!s->cv_done.wait_for(lock, std::chrono::milliseconds(timeout_ms), ready))
        return VISQOL_B200_PENDING;
    const Done d = s->done.front();
    s->done.pop_front();
    *ticket = d.ticket;
    *status = d.status;
    *out = d.result;
    return VISQOL_OK;
}

int visqol_b200_server_stats(visqol_b200_server *s, visqol_b200_serve_stats *out, int reset) {
    if (!s || !out) return fail(VISQOL_E_INVALID_ARGUMENT, "NULL argument");
    std::vector<double> lat, que;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        out->submitted = s->submitted;
        out->completed = s->completed;
        out->failed = s->failed;
        out->queued = s->queue.size();
        out->in_flight = s->in_flight;
        out->batches = s->batches;
        out->hbm_budget_bytes = s->budget;
        out->hbm_in_flight_bytes = s->in_flight_bytes;
        out->mean_batch = s->batches ? (double)s->batch_pairs / (double)s->batches : 0.0;
        lat = s->latency;
        que = s->queueing;
        if (reset) {
            s->latency.clear();
            s->queueing.clear();
            s->batches = 0;
            s->batch_pairs = 0;
        }
        uint64_t held = 0;
        for (auto &l : s->lanes) held += l->reserved;
        out->hbm_reserved_bytes = held;
    }
    out->latency_p50_ms = percentile(lat, 0.50);
    out->latency_p99_ms = percentile(lat, 0.99);
    double sum = 0;
    for (double v : lat) sum += v;
    out->latency_mean_ms = lat.empty() ? 0.0 : sum / (double)lat.size();
    out->queue_p50_ms = percentile(que, 0.50);
    out->queue_p99_ms = percentile(que, 0.99);
    return VISQOL_OK;
}

}  // extern "C"
