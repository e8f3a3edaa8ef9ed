// Batched ViSQOL pipeline on one GPU (exact f64 form).
//
// The reference's CPU model runs a pair's stages in sequence
// (src/visqol.zig:394-487); its data-dependent steps (frame counts follow the
// global lag, patch windows follow the frame counts, realignment slices
// follow the DP matches, trimmed lengths follow the per-patch lags) are
// planned here on the host between device phases, for all pairs of the batch
// at once, so every kernel launch covers the whole batch:
//
//   1. envelopes + FFT lag search, SPL energies        -> lags, energies
//   2. (host) SPL factors, frames, patches, search windows
//   3. aligned+scaled signals, gammatone spectrograms, dB/floors, NSIM
//      table, DP, per-match band statistics            -> matches
//   4. (host) realignment slices
//   5. slice envelopes + FFT lag search                 -> per-patch lags
//   6. (host) trimmed geometry, grid-frame reuse
//   7. realigned spectrograms, dB/floors, band statistics
//   8. (host) accept rule, pooled features, MOS
//
// Signals and intermediate spectrograms stay in HBM; only lags, energies,
// matches and statistics cross to the host.
#include <thread>
#include <cstdlib>
#include <map>
#include <tuple>
#include <mutex>
#include <functional>
#include <future>

#include "engine.h"

#include <algorithm>
#include <cmath>
#include <cstring>

#include "grad_host.h"
#include "kernels.h"

namespace vqb {

void cuda_check(cudaError_t e, const char *what) {
    if (e == cudaSuccess) return;
    cudaGetLastError();
    if (e == cudaErrorMemoryAllocation) throw Error(kOom, std::string(what) + ": " + cudaGetErrorString(e));
    throw Error(kBackend, std::string(what) + ": " + cudaGetErrorString(e));
}

// ---------------------------------------------------------------------------
// Arenas
// ---------------------------------------------------------------------------
namespace {
constexpr size_t kAlign = 256;
constexpr size_t kChunk = size_t(256) << 20;
inline size_t round_up(size_t x) { return (x + kAlign - 1) & ~(kAlign - 1); }

// Zero-fill on the compute stream as a kernel (no copy-engine work, so it
// cannot queue behind a signal upload that another stream has in flight).
__global__ void __launch_bounds__(256) zero_kernel(uint4 *__restrict__ dst, size_t n16) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n16; i += (size_t)gridDim.x * blockDim.x)
        dst[i] = make_uint4(0u, 0u, 0u, 0u);
}

// dst: an arena block (256-byte aligned and rounded, so whole 16-byte
// words may be written).
void launch_zero(void *dst, size_t bytes, cudaStream_t s) {
    const size_t n16 = (bytes + 15) / 16;
    const size_t blocks = std::min<size_t>((n16 + 255) / 256, 256);
    zero_kernel<<<(unsigned)std::max<size_t>(1, blocks), 256, 0, s>>>(static_cast<uint4 *>(dst), n16);
    launch_counter() += 1;
}
}  // namespace

Arena::~Arena() {
    for (auto &c : chunks_) cudaFree(c.base);
}
void Arena::reset() {
    for (auto &c : chunks_) c.used = 0;
    current_ = 0;
}
void *Arena::alloc(size_t bytes) {
    bytes = round_up(bytes ? bytes : 1);
    while (current_ < chunks_.size()) {
        Chunk &c = chunks_[current_];
        if (c.used + bytes <= c.size) {
            void *p = c.base + c.used;
            c.used += bytes;
            return p;
        }
        ++current_;
    }
    Chunk c{nullptr, std::max(bytes, kChunk), 0};
    VQB_CUDA(cudaMalloc(&c.base, c.size));
    c.used = bytes;
    chunks_.push_back(c);
    current_ = chunks_.size() - 1;
    return c.base;
}
void Arena::release() {
    for (auto &c : chunks_) cudaFree(c.base);
    chunks_.clear();
    current_ = 0;
}
size_t Arena::reserved() const {
    size_t s = 0;
    for (auto &c : chunks_) s += c.size;
    return s;
}

PinnedArena::~PinnedArena() {
    for (auto &c : chunks_) cudaFreeHost(c.base);
}
void PinnedArena::reset() {
    for (auto &c : chunks_) c.used = 0;
    current_ = 0;
}
void *PinnedArena::alloc(size_t bytes) {
    bytes = round_up(bytes ? bytes : 1);
    while (current_ < chunks_.size()) {
        Chunk &c = chunks_[current_];
        if (c.used + bytes <= c.size) {
            void *p = c.base + c.used;
            c.used += bytes;
            return p;
        }
        ++current_;
    }
    Chunk c{nullptr, std::max(bytes, size_t(64) << 20), 0};
    VQB_CUDA(cudaMallocHost(&c.base, c.size));
    c.used = bytes;
    chunks_.push_back(c);
    current_ = chunks_.size() - 1;
    return c.base;
}

// ---------------------------------------------------------------------------
// Engine
// ---------------------------------------------------------------------------
Engine::Engine(int device, const Options &opt, std::shared_ptr<const host::Svr> svr,
               std::shared_ptr<const host::LatticeMapper> lattice)
    : device_(device), opt_(opt), svr_(std::move(svr)), lattice_(std::move(lattice)) {
    nb_ = opt.speech ? 21 : 32;
    patch_ = opt.speech ? 20 : 30;
    max_freq_ = opt.speech ? 8000.0 : -1.0;
    VQB_CUDA(cudaSetDevice(device_));
    // The main stream carries the latency-critical chain (serial sums, FFTs,
    // read-backs): highest priority, so its CTAs take SMs first as the side
    // stream's long gammatone grid drains.
    int lo_prio = 0, hi_prio = 0;
    VQB_CUDA(cudaDeviceGetStreamPriorityRange(&lo_prio, &hi_prio));
    VQB_CUDA(cudaStreamCreateWithPriority(&stream_, cudaStreamNonBlocking, hi_prio));
    VQB_CUDA(cudaStreamCreateWithPriority(&side_, cudaStreamNonBlocking, lo_prio));
    VQB_CUDA(cudaEventCreateWithFlags(&ev_inputs_, cudaEventDisableTiming));
    VQB_CUDA(cudaEventCreateWithFlags(&ev_ref_done_, cudaEventDisableTiming));
    VQB_CUDA(cudaStreamCreateWithFlags(&copy_, cudaStreamNonBlocking));
    for (auto &e : ev_up_) VQB_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    VQB_CUDA(cudaEventCreateWithFlags(&ev_piece_, cudaEventDisableTiming));
    events_.resize(8);
    for (auto &e : events_) VQB_CUDA(cudaEventCreate(&e));
    for (auto &e : gt_events_) VQB_CUDA(cudaEventCreate(&e));
    for (auto &e : lag_events_) VQB_CUDA(cudaEventCreate(&e));
    fft_init_attributes();
    lag_init_attributes();
    lag32_init_attributes();
    nsim_init_attributes();
    VQB_CUDA(cudaGetLastError());
}

Engine::~Engine() {
    cudaSetDevice(device_);
    if (stream_) cudaStreamSynchronize(stream_);
    if (side_) cudaStreamSynchronize(side_);
    if (copy_) cudaStreamSynchronize(copy_);
    for (auto e : ev_up_)
        if (e) cudaEventDestroy(e);
    if (ev_piece_) cudaEventDestroy(ev_piece_);
    for (auto p : slot_) cudaFree(p);
    if (copy_) cudaStreamDestroy(copy_);
    if (ev_inputs_) cudaEventDestroy(ev_inputs_);
    if (ev_ref_done_) cudaEventDestroy(ev_ref_done_);
    if (side_) cudaStreamDestroy(side_);
    for (auto &kv : rates_) {
        cudaFree(kv.second.d_coeffs);
        cudaFree(kv.second.d_fast_coeffs);
        cudaFree(kv.second.d_hann);
    }
    for (auto &kv : twiddles_) cudaFree(const_cast<double2 *>(kv.second.top));
    for (auto e : events_) cudaEventDestroy(e);
    for (auto e : gt_events_)
        if (e) cudaEventDestroy(e);
    for (auto e : lag_events_)
        if (e) cudaEventDestroy(e);
    if (stream_) cudaStreamDestroy(stream_);
}

void Engine::release_device_memory() {
    VQB_CUDA(cudaSetDevice(device_));
    VQB_CUDA(cudaStreamSynchronize(stream_));
    VQB_CUDA(cudaStreamSynchronize(side_));
    VQB_CUDA(cudaStreamSynchronize(copy_));
    arena_.release();
    for (int k = 0; k < 2; ++k) {
        if (slot_[k]) cudaFree(slot_[k]);
        slot_[k] = nullptr;
        slot_bytes_[k] = 0;
    }
}

const Engine::RateCache &Engine::rate_cache(uint32_t sr) {
    auto it = rates_.find(sr);
    if (it != rates_.end()) return it->second;
    RateCache rc;
    rc.fb = host::make_filterbank(nb_, sr, 50.0, max_freq_ > 0 ? max_freq_ : (double)sr / 2.0);
    rc.geo = host::analysis_geometry(sr);
    const std::vector<double> w = host::hann(rc.geo.window);
    VQB_CUDA(cudaMalloc(&rc.d_coeffs, nb_ * sizeof(BandCoeffs)));
    VQB_CUDA(cudaMalloc(&rc.d_hann, std::max<size_t>(1, w.size()) * sizeof(double)));
    // Copies from pageable memory are ordered on this engine's stream (a
    // plain cudaMemcpy may return before its DMA lands, and the engine's
    // non-blocking streams would not wait for it).
    std::vector<FastBandCoeffs> fast(nb_);
    fill_fast_band_coeffs(rc.fb.run.data(), rc.fb.cf.data(), (int)nb_, fast.data());
    VQB_CUDA(cudaMalloc(&rc.d_fast_coeffs, nb_ * sizeof(FastBandCoeffs)));
    VQB_CUDA(cudaMemcpyAsync(rc.d_coeffs, rc.fb.run.data(), nb_ * sizeof(BandCoeffs), cudaMemcpyHostToDevice, stream_));
    VQB_CUDA(cudaMemcpyAsync(rc.d_fast_coeffs, fast.data(), nb_ * sizeof(FastBandCoeffs), cudaMemcpyHostToDevice,
                             stream_));
    if (!w.empty())
        VQB_CUDA(cudaMemcpyAsync(rc.d_hann, w.data(), w.size() * sizeof(double), cudaMemcpyHostToDevice, stream_));
    VQB_CUDA(cudaStreamSynchronize(stream_));
    return rates_.emplace(sr, std::move(rc)).first->second;
}

Engine::Twiddles Engine::twiddles(size_t n) {
    auto it = twiddles_.find(n);
    if (it != twiddles_.end()) return it->second;
    // top[k] = W_n^k (k < n/2), then the block passes' W_B^k = top[k * n/B].
    // then the fused lag search's stage-major column twiddles.
    std::vector<double2> t = host::twiddles(n);
    const size_t B = (size_t)fft_block_size((int64_t)n), half = t.size();
    for (size_t k = 0; k < B / 2; ++k) t.push_back(t[k * (n / B)]);
    const size_t cols_at = t.size();
    t.resize(cols_at + column_twiddle_count((int64_t)n));
    fill_column_twiddles(t.data(), (int64_t)n, t.data() + cols_at);
    // the 4096-point block stages' stage-major table (fused search, n > 4096)
    const size_t stages_at = t.size();
    if (B == 4096) {
        t.resize(stages_at + block_stage_twiddle_count());
        fill_block_stage_twiddles(t.data() + half, t.data() + stages_at);
    }
    // f32 copies of the block, column and stage tables (the f32 search)
    std::vector<float2> t32(t.size() - half);
    for (size_t k = half; k < t.size(); ++k) t32[k - half] = make_float2((float)t[k].x, (float)t[k].y);
    // one allocation: the f64 tables, then the f32 ones at a 16-byte boundary
    const size_t bytes64 = std::max<size_t>(1, t.size()) * sizeof(double2);
    double2 *d = nullptr;
    VQB_CUDA(cudaMalloc(&d, bytes64 + std::max<size_t>(1, t32.size()) * sizeof(float2)));
    float2 *d32 = reinterpret_cast<float2 *>(reinterpret_cast<char *>(d) + bytes64);
    if (!t.empty()) {
        VQB_CUDA(cudaMemcpyAsync(d, t.data(), t.size() * sizeof(double2), cudaMemcpyHostToDevice, stream_));
        VQB_CUDA(cudaMemcpyAsync(d32, t32.data(), t32.size() * sizeof(float2), cudaMemcpyHostToDevice, stream_));
        VQB_CUDA(cudaStreamSynchronize(stream_));
    }
    Twiddles tw{d, d + half, d + cols_at, d + stages_at, d32, d32 + (cols_at - half), d32 + (stages_at - half)};
    twiddles_[n] = tw;
    return tw;
}

template <class T>
T *Engine::upload(const std::vector<T> &v) {
    return static_cast<T *>(upload_bytes(v.data(), v.size() * sizeof(T)));
}

void *Engine::upload_bytes(const void *src, size_t bytes) {
    void *h = pinned_.alloc(bytes);
    if (bytes) std::memcpy(h, src, bytes);
    void *d = arena_.alloc(bytes);
    if (bytes) VQB_CUDA(cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, stream_));
    timing_.h2d_bytes += bytes;
    return d;
}

void Engine::d2h(void *dst, const void *src, size_t bytes) {
    if (!bytes) return;
    VQB_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, stream_));
    timing_.d2h_bytes += bytes;
}

void Engine::sync() {
    VQB_CUDA(cudaGetLastError());
    VQB_CUDA(cudaStreamSynchronize(stream_));
    ++timing_.host_syncs;
}

void Engine::record(cudaEvent_t e) { VQB_CUDA(cudaEventRecord(e, stream_)); }

float Engine::elapsed(cudaEvent_t a, cudaEvent_t b) {
    float ms = 0;
    VQB_CUDA(cudaEventElapsedTime(&ms, a, b));
    return ms;
}

uint64_t lag_search_bytes(const LagJob &j, bool f32) {
    // signals read by the forward pass (and by the f32 search's rescoring),
    // then the transform written, read and written, read: 4 passes over z
    const uint64_t sig = 8 * (uint64_t)(j.a.avail + j.b.avail);
    return f32 ? 2 * sig + 4 * 8 * (uint64_t)j.n : sig + 4 * 16 * (uint64_t)j.n;
}

int32_t *Engine::launch_lag_jobs(std::vector<LagJob> &jobs, bool raw, bool exact) {
    if (jobs.empty()) return nullptr;
    // Group by FFT size; bound each submission's buffer.
    std::map<int64_t, std::vector<size_t>> groups;
    for (size_t i = 0; i < jobs.size(); ++i) groups[jobs[i].n].push_back(i);
    const size_t budget = size_t(4) << 30;
    const bool f32 = !exact && !opt_.exact_lag_search;
    int32_t *d_status = nullptr;
    if (f32) {
        d_status = arena_.alloc_n<int32_t>(jobs.size());
        launch_zero(d_status, jobs.size() * sizeof(int32_t), stream_);
    }
    for (auto &g : groups) {
        const int64_t n = g.first;
        const Twiddles tw = twiddles((size_t)n);
        const size_t per = std::max<size_t>(1, budget / ((size_t)n * sizeof(double2)));
        for (size_t c0 = 0; c0 < g.second.size(); c0 += per) {
            const size_t cnt = std::min(per, g.second.size() - c0);
            if (f32 && fused_lag_supported(n)) {
                // The f32 search (half the transform's bytes, FP32 arithmetic),
                // then f64 rescoring of its candidates.
                const size_t parts = lag32_parts(n);
                int64_t max_b = 1;
                for (size_t k = 0; k < cnt; ++k) max_b = std::max(max_b, jobs[g.second[c0 + k]].b.len);
                const int nchunks = lag32_rescore_chunks(max_b);
                float2 *z = arena_.alloc_n<float2>((size_t)n * cnt);
                double2 *energy = arena_.alloc_n<double2>(parts * cnt);
                LagCands *cands = arena_.alloc_n<LagCands>(parts * cnt);
                int32_t *ncand = arena_.alloc_n<int32_t>(cnt);
                int32_t *keys = arena_.alloc_n<int32_t>((size_t)kLagCandCap * cnt);
                double *rescore = arena_.alloc_n<double>((size_t)kLagCandCap * nchunks * cnt);
                std::vector<LagJob> chunk(cnt);
                for (size_t k = 0; k < cnt; ++k) {
                    const size_t i = g.second[c0 + k];
                    LagJob j = jobs[i];
                    j.z32 = z + (int64_t)k * n;
                    j.energy = energy + k * parts;
                    j.cands = cands + k * parts;
                    j.status = d_status + i;
                    j.ncand = ncand + k;
                    j.cand_key = keys + (size_t)kLagCandCap * k;
                    j.rescore = rescore + (size_t)kLagCandCap * nchunks * k;
                    chunk[k] = j;
                }
                LagJob *d_chunk = upload(chunk);
                auto launch32 = [&](int columns) {
                    launch_lag32(d_chunk, (int)cnt, n, raw, tw.cols32, tw.block32, tw.stages32, nchunks, columns,
                                 stream_);
                };
                // forward samples staged in shared memory, or loaded into
                // registers: measured per transform size
                const char *env = std::getenv("VISQOL_LAG_COLUMNS");
                const int columns = !fused_lag_register_columns(n) ? 0
                                    : env && (env[0] == '0' || env[0] == '1' || env[0] == '2')
                                        ? env[0] - '0'
                                        : tuned(kTuneLagColumns, (int)std::log2((double)n), raw ? 3 : 2, {2, 1},
                                                launch32, stream_);
                launch32(columns);
                continue;
            }
            // (above 2^24 points the exact search decides in every form; status stays 0)
            double2 *z = arena_.alloc_n<double2>((size_t)n * cnt);
            std::vector<LagJob> chunk(cnt);
            for (size_t k = 0; k < cnt; ++k) {
                chunk[k] = jobs[g.second[c0 + k]];
                chunk[k].z = z + (int64_t)k * n;
            }
            LagJob *d_jobs = upload(chunk);
            if (fused_lag_supported(n)) {
                const size_t parts = fused_lag_parts(n);
                double *pv = arena_.alloc_n<double>(parts * cnt);
                int64_t *pk = arena_.alloc_n<int64_t>(parts * cnt);
                auto launch = [&](int columns) {
                    launch_fused_lag(d_jobs, (int)cnt, n, raw, tw.cols, tw.block, tw.stages, pv, pk, columns, stream_);
                };
                // column passes: shared-memory tiles, registers, or registers
                // with the forward samples staged, measured per transform size
                // (VISQOL_LAG_COLUMNS=0/1/2 fixes the choice)
                int columns = 0;
                if (fused_lag_register_columns(n)) {
                    const char *env = std::getenv("VISQOL_LAG_COLUMNS");
                    columns = env && (env[0] == '0' || env[0] == '1' || env[0] == '2')
                                  ? env[0] - '0'
                                  : tuned(kTuneLagColumns, (int)std::log2((double)n), raw ? 1 : 0, {1, 2, 0},
                                          launch, stream_);
                }
                launch(columns);
                continue;
            }
            const int parts = argmax_parts(n);
            double *pv = arena_.alloc_n<double>((size_t)parts * cnt);
            int64_t *pk = arena_.alloc_n<int64_t>((size_t)parts * cnt);
            launch_pack(d_jobs, (int)cnt, n, raw, stream_);
            launch_fft(z, n, false, tw.top, tw.block, (int)cnt, n, stream_);
            launch_cross(z, n, (int)cnt, n, stream_);
            launch_fft(z, n, true, tw.top, tw.block, (int)cnt, n, stream_);
            launch_argmax(z, d_jobs, (int)cnt, n, n, pv, pk, stream_);
        }
    }
    return d_status;
}

std::vector<size_t> Engine::rerun_undecided(const std::vector<LagJob> &jobs, const int32_t *h_status, bool raw) {
    std::vector<size_t> idx;
    if (!h_status) return idx;
    std::vector<LagJob> rerun;
    for (size_t i = 0; i < jobs.size(); ++i)
        if (h_status[i]) idx.push_back(i), rerun.push_back(jobs[i]);
    if (!rerun.empty()) launch_lag_jobs(rerun, raw, true);
    timing_.lag_reruns += idx.size();
    return idx;
}

size_t Engine::pair_footprint(size_t rl, size_t dl, uint32_t sample_rate, bool speech) {
    const size_t H = std::max<size_t>(1, host::analysis_geometry(sample_rate).hop);
    const size_t NB = speech ? 21 : 32, P = speech ? 20 : 30;
    const size_t al = dl + rl / 2 + 1;  // aligned degraded length bound (|lag| <= ref/2)
    const size_t nfr = rl / H + 1, nfd = al / H + 1;
    const size_t width = nfd + 2 * P + 2;
    const size_t np = nfr / std::max<size_t>(1, P) + 1;
    const size_t n_global = host::fft_size_for(std::max(rl, dl));
    const size_t n_slice = host::fft_size_for(2 * P * H + 2);
    size_t b = 8 * (rl + dl)                                   // inputs
               + 16 * n_global + 16 * 1024                     // lag search and argmax parts
               + 8 * al                                        // aligned, scaled degraded signal
               + 8 * NB * (2 * nfr + 2 * nfd + 4 * width)      // spectrograms, prepared copies, plane
               + np * (8 * 4 * NB * P + 24 * nfd + 8 * (3 * NB + 1) + 16)  // terms, table, DP, stats
               + np * (16 * n_slice + 8 * 4 * NB * (2 * P + 2) + 256);     // realignment slices
    b += b / 4 + (size_t(1) << 20);  // job tables, tiles, rounding slack
    return b;
}

uint64_t Engine::launch_spectrograms(const std::vector<SpecJob> &jobs, const RateCache &rc, cudaStream_t st,
                                     cudaEvent_t begin, cudaEvent_t end) {
    if (jobs.empty()) return 0;
    const int nbi = (int)nb_;
    const int W = (int)rc.geo.window, H = (int)rc.geo.hop;
    SpecJob *d_jobs = upload(jobs);
    uint64_t rms = 0;
    for (const SpecJob &j : jobs) rms += (uint64_t)j.nf * nb_;
    // Tiles of F frames (the FP32 kernel's shape is fixed), uploaded on the
    // main stream; a side stream waits for them.
    auto tiles_of = [&](int F, int *ntiles) {
        const size_t tsz = gammatone_tile_size();
        std::vector<char> tiles;
        *ntiles = 0;
        for (size_t j = 0; j < jobs.size(); ++j)
            for (int64_t f = 0; f < jobs[j].nf; f += F, ++*ntiles) {
                tiles.resize(tiles.size() + tsz);
                fill_gammatone_tile(tiles.data() + tiles.size() - tsz, (int)j, (int)f);
            }
        void *d = upload_bytes(tiles.data(), tiles.size());
        if (st != stream_) {
            record(ev_inputs_);
            VQB_CUDA(cudaStreamWaitEvent(st, ev_inputs_, 0));
        }
        return d;
    };
    auto launch_frames = [&](int F) {
        int ntiles = 0;
        const void *d_tiles = tiles_of(F, &ntiles);
        if (opt_.form == kFormF64)
            launch_gammatone_f64fma(d_jobs, d_tiles, ntiles, rc.d_fast_coeffs, nbi, rc.d_hann, W, H, F, st);
        else
            launch_gammatone(d_jobs, d_tiles, ntiles, rc.d_coeffs, nbi, rc.d_hann, W, H, F, st);
    };
    if (opt_.form == kFormF32) {
        int ntiles = 0;
        const void *d_tiles = tiles_of(gammatone_fast_frames_per_cta(), &ntiles);
        int *queue = arena_.alloc_n<int>(1);  // the persistent form's work counter
        auto launch = [&](int shape) {
            if (shape >= 100) launch_zero(queue, sizeof(int), st);
            launch_gammatone_fast(d_jobs, d_tiles, ntiles, rc.d_fast_coeffs, nbi, rc.d_hann, W, H, shape, queue, st);
        };
        static const std::vector<int> all_shapes = gammatone_fast_shapes();
        const int shape =
            tuned(kTuneGammatoneFastCtas, opt_.form, nbi, gammatone_fast_shape_candidates(), launch, st, &all_shapes);
        if (begin) VQB_CUDA(cudaEventRecord(begin, st));
        launch(shape);
    } else {
        const int F = tuned(kTuneGammatone, opt_.form, nbi,
                            opt_.form == kFormF64 ? gammatone_f64fma_frames_candidates(nbi)
                                                  : gammatone_frames_candidates(nbi),
                            launch_frames, st);
        if (opt_.form == kFormF64) {
            // the FP64-FMA kernel at that shape, or the same form on the FP32
            // kernel's staged tiles (same bits); tile lists uploaded on first use
            int ntiles[2] = {0, 0};
            const void *d_tiles[2] = {nullptr, nullptr};
            auto ensure_tiles = [&](int staged) {
                if (!d_tiles[staged])
                    d_tiles[staged] = tiles_of(staged ? gammatone_fast_frames_per_cta() : F, &ntiles[staged]);
            };
            auto launch = [&](int staged) {
                ensure_tiles(staged);
                if (staged)
                    launch_gammatone_f64_staged(d_jobs, d_tiles[1], ntiles[1], rc.d_fast_coeffs, nbi, rc.d_hann, W, H,
                                                st);
                else
                    launch_gammatone_f64fma(d_jobs, d_tiles[0], ntiles[0], rc.d_fast_coeffs, nbi, rc.d_hann, W, H, F,
                                            st);
            };
            const int staged =
                tuned(kTuneGammatoneF64Staged, opt_.form, nbi, gammatone_f64_staged_candidates(), launch, st);
            ensure_tiles(staged);
            if (begin) VQB_CUDA(cudaEventRecord(begin, st));
            launch(staged);
        } else {
            int ntiles = 0;
            const void *d_tiles = tiles_of(F, &ntiles);
            if (begin) VQB_CUDA(cudaEventRecord(begin, st));
            launch_gammatone(d_jobs, d_tiles, ntiles, rc.d_coeffs, nbi, rc.d_hann, W, H, F, st);
        }
    }
    if (end) VQB_CUDA(cudaEventRecord(end, st));
    return rms;
}

namespace {

// Launch shapes chosen by measurement, per (device, kernel, variant): shared
// by every engine of the process. VISQOL_AUTOTUNE=0 keeps the defaults.
std::mutex g_tune_mu;
std::map<std::tuple<int, int, int, int>, int> g_tune;

bool autotune_enabled() {
    static const bool on = [] {
        const char *e = std::getenv("VISQOL_AUTOTUNE");
        return !e || std::atoi(e) != 0;
    }();
    return on;
}

}  // namespace

int Engine::tuned(int kernel, int a, int b, const std::vector<int> &candidates,
                  const std::function<void(int)> &launch, cudaStream_t st, const std::vector<int> *allowed) {
    // VISQOL_TUNE_<kernel>=<choice> fixes a kernel class's shape (one of its
    // candidates), e.g. to check that every shape gives the same results.
    if (const char *env = std::getenv(("VISQOL_TUNE_" + std::to_string(kernel)).c_str())) {
        const int forced = std::atoi(env);
        const std::vector<int> &ok = allowed ? *allowed : candidates;
        if (std::find(ok.begin(), ok.end(), forced) != ok.end()) return forced;
    }
    if (!autotune_enabled() || candidates.size() < 2) return candidates.at(0);
    const auto key = std::make_tuple(device_, kernel, a, b);
    {
        std::lock_guard<std::mutex> lock(g_tune_mu);
        auto it = g_tune.find(key);
        if (it != g_tune.end()) return it->second;
    }
    // The candidates run on this batch's real jobs (the kernels write the
    // same values whatever their shape), one warm-up each, then five timed
    // rounds in turn so that other work on the GPU (other lanes' kernels)
    // touches them alike; each keeps its fastest run. A candidate replaces
    // the default only when it is at least 5% faster: the defaults are the
    // shapes measured best in isolation, and a first batch timed beside other
    // lanes is noisy.
    cudaEvent_t e0, e1;
    VQB_CUDA(cudaEventCreate(&e0));
    VQB_CUDA(cudaEventCreate(&e1));
    std::vector<float> best_ms(candidates.size(), 0.0f);
    for (int c : candidates) launch(c);
    for (int round = 0; round < 5; ++round)
        for (size_t i = 0; i < candidates.size(); ++i) {
            VQB_CUDA(cudaEventRecord(e0, st));
            launch(candidates[i]);
            VQB_CUDA(cudaEventRecord(e1, st));
            VQB_CUDA(cudaEventSynchronize(e1));
            float ms = 0.0f;
            VQB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            if (round == 0 || ms < best_ms[i]) best_ms[i] = ms;
        }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    int best = candidates[0];
    float best_t = best_ms[0] * 0.95f;
    for (size_t i = 1; i < candidates.size(); ++i)
        if (best_ms[i] < best_t) best = candidates[i], best_t = best_ms[i];
    std::lock_guard<std::mutex> lock(g_tune_mu);
    return g_tune.emplace(key, best).first->second;
}

std::vector<std::tuple<int, int, int, int, int>> autotune_choices() {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    std::vector<std::tuple<int, int, int, int, int>> out;
    for (const auto &kv : g_tune)
        out.emplace_back(std::get<0>(kv.first), std::get<1>(kv.first), std::get<2>(kv.first), std::get<3>(kv.first),
                         kv.second);
    return out;
}

PreparedRef::~PreparedRef() {
    if (!d_sig && !d_stats && !d_spec) return;
    int cur = 0;
    cudaGetDevice(&cur);
    cudaSetDevice(device);
    cudaFree(d_sig);
    cudaFree(d_stats);
    cudaFree(d_spec);
    cudaSetDevice(cur);
}

void Engine::prepare(size_t n, const double *const *refs, const size_t *ref_lens, uint32_t sample_rate,
                     bool device_inputs, std::vector<std::unique_ptr<PreparedRef>> &out) {
    out.clear();
    VQB_CUDA(cudaSetDevice(device_));
    arena_.reset();
    pinned_.reset();
    const RateCache &rc = rate_cache(sample_rate);
    const size_t W = rc.geo.window, H = rc.geo.hop, P = patch_;
    std::vector<SumJob> sums;
    std::vector<SpecJob> specs;
    for (size_t i = 0; i < n; ++i) {
        auto p = std::make_unique<PreparedRef>();
        p->device = device_;
        p->len = ref_lens[i];
        if (p->len && !refs[i]) {
            p->code = kInvalid;
            p->message = "signal pointer is NULL";
        } else if (p->len <= W) {
            p->code = kSignal;
            p->message = "SpectrogramTooShort";
        } else {
            p->nf = host::num_frames(p->len, W, H);
            VQB_CUDA(cudaMalloc(&p->d_sig, p->len * sizeof(double)));
            VQB_CUDA(cudaMalloc(&p->d_stats, 4 * sizeof(double)));
            VQB_CUDA(cudaMalloc(&p->d_spec, nb_ * p->nf * sizeof(double)));
            VQB_CUDA(cudaMemcpyAsync(p->d_sig, refs[i], p->len * sizeof(double),
                                     device_inputs ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, stream_));
            const VSig sig{p->d_sig, 0, (int64_t)p->len, (int64_t)p->len};
            sums.push_back(SumJob{sig, p->d_stats});
            specs.push_back(SpecJob{sig, (int64_t)p->nf, p->d_spec});
        }
        out.push_back(std::move(p));
    }
    launch_sums(sums);
    launch_spectrograms(specs, rc, stream_);
    std::vector<double> h(4 * n, 0.0);
    for (size_t i = 0; i < n; ++i)
        if (out[i]->d_stats) VQB_CUDA(cudaMemcpyAsync(h.data() + 4 * i, out[i]->d_stats, 4 * sizeof(double),
                                                      cudaMemcpyDeviceToHost, stream_));
    sync();
    for (size_t i = 0; i < n; ++i) {
        PreparedRef &p = *out[i];
        if (p.code) continue;
        std::copy(h.begin() + 4 * i, h.begin() + 4 * i + 4, p.stats);
        if (opt_.speech) {
            std::vector<double> tmp;
            const double *hr = refs[i];
            if (device_inputs) {
                tmp.resize(p.len);
                VQB_CUDA(cudaMemcpy(tmp.data(), refs[i], p.len * sizeof(double), cudaMemcpyDeviceToHost));
                hr = tmp.data();
            }
            p.idx = host::vad_patch_indices(hr, p.len, p.nf, P, W, 0.25);
        } else {
            p.idx = host::ref_patch_indices(p.nf, P);
        }
        if (p.idx.empty()) {
            p.code = kSignal;
            p.message = "NoPatches";
        }
    }
}

void Engine::launch_sums(const std::vector<SumJob> &sums) {
    if (sums.empty()) return;
    const SumJob *d = upload(sums);
    if (opt_.form != kFormExact)
        launch_envelope_stats_tree(d, (int)sums.size(), arena_.alloc_n<double>(sums.size() * kTreeParts * 3), stream_);
    else
        launch_envelope_stats(d, (int)sums.size(), stream_);
}

void Engine::lags(size_t njobs, const VSig *a, const VSig *b, bool raw, int64_t *h_lags, int32_t *status_out,
                  float *d_corr) {
    arena_.reset();
    pinned_.reset();
    std::vector<LagJob> jobs(njobs);
    int64_t *d_lags = arena_.alloc_n<int64_t>(njobs);
    double *d_stats = arena_.alloc_n<double>(8 * njobs);
    std::vector<SumJob> sums;
    for (size_t i = 0; i < njobs; ++i) {
        LagJob &j = jobs[i];
        j.a = a[i];
        j.b = b[i];
        j.biggest = std::max(a[i].len, b[i].len);
        j.n = (int64_t)host::fft_size_for((size_t)j.biggest);
        j.stats_a = d_stats + 8 * i;
        j.stats_b = d_stats + 8 * i + 4;
        j.lag_out = d_lags + i;
        j.corr_out = i == 0 ? d_corr : nullptr;
        sums.push_back(SumJob{a[i], j.stats_a});
        sums.push_back(SumJob{b[i], j.stats_b});
    }
    VQB_CUDA(cudaMemsetAsync(d_lags, 0, njobs * sizeof(int64_t), stream_));
    std::vector<size_t> empty;
    std::vector<LagJob> run;
    std::vector<size_t> where;
    for (size_t i = 0; i < njobs; ++i)
        if (jobs[i].biggest > 0) run.push_back(jobs[i]), where.push_back(i);
    if (!raw && !sums.empty()) launch_envelope_stats(upload(sums), (int)sums.size(), stream_);
    int32_t *d_status = launch_lag_jobs(run, raw);
    int64_t *h = pinned_.alloc_n<int64_t>(njobs);
    int32_t *h_status = d_status ? pinned_.alloc_n<int32_t>(run.size()) : nullptr;
    d2h(h, d_lags, njobs * sizeof(int64_t));
    if (h_status && !run.empty()) d2h(h_status, d_status, run.size() * sizeof(int32_t));
    sync();
    if (!rerun_undecided(run, h_status, raw).empty()) {
        d2h(h, d_lags, njobs * sizeof(int64_t));
        sync();
    }
    std::memcpy(h_lags, h, njobs * sizeof(int64_t));
    if (status_out)
        for (size_t k = 0; k < run.size(); ++k) status_out[where[k]] = h_status ? h_status[k] : 0;
}

bool Engine::refine_approx(const VSig &a, const VSig &b, const float *d_approx, int64_t n, double slack,
                           double energy, int64_t *lag) {
    arena_.reset();
    pinned_.reset();
    LagJob j{};
    j.a = a;
    j.b = b;
    j.n = n;
    j.biggest = std::max(a.len, b.len);
    const int nchunks = lag32_rescore_chunks(std::max<int64_t>(1, b.len));
    const size_t parts = (size_t)((n + 4095) / 4096);
    j.corr_out = const_cast<float *>(d_approx);
    j.slack_fixed = slack;
    j.cands = arena_.alloc_n<LagCands>(parts);
    std::vector<double2> e(parts, make_double2(0.0, 0.0));
    e[0].x = energy;  // the rescoring's tie margin scales with it
    j.energy = upload(e);
    j.status = arena_.alloc_n<int32_t>(1);
    j.ncand = arena_.alloc_n<int32_t>(1);
    j.cand_key = arena_.alloc_n<int32_t>(kLagCandCap);
    j.rescore = arena_.alloc_n<double>((size_t)kLagCandCap * nchunks);
    j.lag_out = arena_.alloc_n<int64_t>(1);
    launch_zero(j.lag_out, sizeof(int64_t), stream_);
    launch_refine_approx(upload(std::vector<LagJob>{j}), n, nchunks, stream_);
    int64_t *h = pinned_.alloc_n<int64_t>(1);
    int32_t *st = pinned_.alloc_n<int32_t>(1);
    d2h(h, j.lag_out, sizeof(int64_t));
    d2h(st, j.status, sizeof(int32_t));
    sync();
    *lag = *h;
    return *st == 0;
}

void Engine::spectrogram(const host::Filterbank &fb, const double *d_hann, size_t window, size_t hop,
                         const double *d_x, size_t len, double *d_out, size_t nf) {
    arena_.reset();
    pinned_.reset();
    if (nf == 0) return;
    BandCoeffs *d_coeffs = upload(fb.run);
    SpecJob job{VSig{d_x, 0, (int64_t)len, (int64_t)len}, (int64_t)nf, d_out};
    SpecJob *d_job = upload(std::vector<SpecJob>{job});
    const int nbi = (int)fb.nb;
    const int F = gammatone_frames_per_cta(nbi);
    const size_t tsz = gammatone_tile_size();
    std::vector<char> tiles;
    int ntiles = 0;
    for (size_t f = 0; f < nf; f += F, ++ntiles) {
        tiles.resize(tiles.size() + tsz);
        fill_gammatone_tile(tiles.data() + tiles.size() - tsz, 0, (int)f);
    }
    void *d_tiles = upload_bytes(tiles.data(), tiles.size());
    launch_gammatone(d_job, d_tiles, ntiles, d_coeffs, nbi, d_hann, (int)window, (int)hop, F, stream_);
    sync();
}

namespace detail {

struct RealignPatch {
    size_t mi;
    host::Slice rl, dl;
    int64_t rlen, dlen;
    int64_t lag = 0;
    host::Trim trim{};
    size_t nf = 0;
    double *stats = nullptr;  // 8: slice envelope stats
    double *rs_raw = nullptr, *ds_raw = nullptr, *rs = nullptr, *ds = nullptr, *st = nullptr;
    uint8_t reused = 0;
};

struct PairState {
    const PreparedRef *prep = nullptr;
    bool live = true;
    int code = 0;
    std::string msg;
    const double *ref = nullptr, *deg = nullptr;  // device
    const double *h_ref = nullptr;                // host (VAD)
    size_t rl = 0, dl = 0;
    bool lag_job = false;
    double *stats = nullptr;  // device: ref[4], deg[4], aligned energy, aligned length
    host::Aligned al{};
    double factor = 1.0;
    double al_energy = 0.0;  // energy of the aligned degraded signal (its SPL)
    double ref_energy = 0.0;
    size_t nf_ref = 0, nf_deg = 0;
    std::vector<int64_t> idx;
    host::Search search;
    size_t width = 0;
    double *deg_al = nullptr, *ref_raw = nullptr, *deg_raw = nullptr, *ref_prep = nullptr, *deg_prep = nullptr;
    double *pad = nullptr, *mu = nullptr, *dms = nullptr, *sds = nullptr, *terms = nullptr, *sims = nullptr;
    double *dp = nullptr;
    int64_t *bt = nullptr, *offs = nullptr;
    uint8_t *valid = nullptr;
    double *mstats = nullptr;
    std::vector<host::Match> matches;
    bool grad_ok = false;  // scored, and its gradient requested
    std::vector<RealignPatch> rps;
    PairTrace trace;
    void fail(int c, const std::string &m) {
        live = false;
        code = c;
        msg = m;
    }
};

}  // namespace detail

using detail::PairState;
using detail::RealignPatch;

void Engine::measure_batch(size_t n, const double *const *refs, const size_t *ref_lens, const double *const *degs,
                           const size_t *deg_lens, uint32_t sample_rate, bool device_inputs,
                           std::vector<PairOutcome> &out, const PreparedRef *const *prepared,
                           const double *const *host_refs, bool grads) {
    out.assign(n, PairOutcome{});
    timing_ = Timing{};
    if (n == 0) return;
    VQB_CUDA(cudaSetDevice(device_));
    if (sample_rate == 0) {
        for (auto &o : out) o.code = kInvalid, o.message = "InvalidInput";
        return;
    }
    arena_.reset();
    pinned_.reset();
    const RateCache &rc = rate_cache(sample_rate);
    const size_t W = rc.geo.window, H = rc.geo.hop, NB = nb_, P = patch_;
    const double fd = rc.geo.frame_duration;
    const int nbi = (int)NB;
    std::vector<PairState> ps(n);
    const uint64_t launches0 = launch_counter();
    record(events_[0]);

    // ---- inputs -----------------------------------------------------------
    for (size_t i = 0; i < n; ++i) {
        PairState &s = ps[i];
        s.prep = prepared ? prepared[i] : nullptr;
        if (s.prep && s.prep->code) {
            s.fail(s.prep->code, s.prep->message);
            continue;
        }
        s.rl = s.prep ? s.prep->len : ref_lens[i];
        s.dl = deg_lens[i];
        if ((!s.prep && s.rl && !refs[i]) || (s.dl && !degs[i])) {
            s.fail(kInvalid, "signal pointer is NULL");
            continue;
        }
        if (device_inputs) {
            s.ref = s.prep ? s.prep->d_sig : refs[i];
            s.deg = degs[i];
            if (host_refs && !s.prep) s.h_ref = host_refs[i];
        } else {
            double *d = arena_.alloc_n<double>(s.dl);
            if (s.dl) VQB_CUDA(cudaMemcpyAsync(d, degs[i], s.dl * sizeof(double), cudaMemcpyHostToDevice, stream_));
            timing_.h2d_bytes += s.dl * sizeof(double);
            s.deg = d;
            if (s.prep) {
                s.ref = s.prep->d_sig;
            } else {
                double *r = arena_.alloc_n<double>(s.rl);
                if (s.rl)
                    VQB_CUDA(cudaMemcpyAsync(r, refs[i], s.rl * sizeof(double), cudaMemcpyHostToDevice, stream_));
                timing_.h2d_bytes += s.rl * sizeof(double);
                s.ref = r;
                s.h_ref = refs[i];
            }
        }
        s.stats = arena_.alloc_n<double>(10);
    }

    auto launch_prep_jobs = [&](const std::vector<PrepJob> &jobs) {
        int max_frames = 0;
        for (const PrepJob &j : jobs) max_frames = std::max({max_frames, (int)j.nfr, (int)j.nfd});
        double *scratch = arena_.alloc_n<double>(prep_scratch_count((int)jobs.size(), max_frames));
        launch_prep(upload(jobs), (int)jobs.size(), nbi, max_frames, scratch, stream_);
    };
    auto run_gammatone = [&](const std::vector<SpecJob> &jobs, cudaStream_t st) {
        if (jobs.empty()) return;
        const size_t slot = 2 * timing_.gammatone_launches;
        const uint64_t rms = launch_spectrograms(jobs, rc, st, gt_events_[slot], gt_events_[slot + 1]);
        timing_.gammatone_launches += 1;
        timing_.gammatone_rms += rms;
        timing_.gammatone_window = W;
    };

    // Reference spectrograms need only the reference signal: they run on a
    // side stream while the main stream does the serial lag-phase work.
    {
        std::vector<SpecJob> ref_jobs;
        for (size_t i = 0; i < n; ++i) {
            PairState &s = ps[i];
            if (!s.live || s.rl <= W) continue;
            if (s.prep) {
                s.nf_ref = s.prep->nf;
                s.ref_raw = s.prep->d_spec;
                continue;
            }
            s.nf_ref = host::num_frames(s.rl, W, H);
            s.ref_raw = arena_.alloc_n<double>(NB * s.nf_ref);
            ref_jobs.push_back(SpecJob{VSig{s.ref, 0, (int64_t)s.rl, (int64_t)s.rl}, (int64_t)s.nf_ref, s.ref_raw});
        }
        run_gammatone(ref_jobs, side_);
        VQB_CUDA(cudaEventRecord(ev_ref_done_, side_));
    }

    // ---- 1: global lag and SPL energies --------------------------------
    int64_t *d_lags = arena_.alloc_n<int64_t>(n);
    launch_zero(d_lags, n * sizeof(int64_t), stream_);
    std::vector<LagJob> lag_jobs;
    std::vector<size_t> lag_pair;  // pair of each lag job
    int32_t *d_lstat = nullptr;    // FP32 form: per lag job, 1 when the f32 search left it undecided
    // aligned energies (read the lags on the device) of the listed pairs
    auto launch_aligned = [&](const std::vector<size_t> &pairs) {
        std::vector<char> args;
        const size_t asz = aligned_energy_args_size();
        int na = 0;
        for (size_t i : pairs) {
            PairState &s = ps[i];
            if (!s.live) continue;
            args.resize(args.size() + asz);
            fill_aligned_energy_args(args.data() + args.size() - asz, VSig{s.deg, 0, (int64_t)s.dl, (int64_t)s.dl},
                                     (int64_t)s.rl, d_lags + i, s.stats + 8, s.lag_job ? s.stats + 4 : nullptr);
            ++na;
        }
        if (na && opt_.form != kFormExact)
            launch_aligned_energy_tree(upload_bytes(args.data(), args.size()), na,
                                       arena_.alloc_n<double>((size_t)na * kTreeParts * 3), stream_);
        else if (na)
            launch_aligned_energy(upload_bytes(args.data(), args.size()), na, stream_);
    };
    {
        std::vector<SumJob> sums;
        for (size_t i = 0; i < n; ++i) {
            PairState &s = ps[i];
            if (!s.live) continue;
            const VSig r{s.ref, 0, (int64_t)s.rl, (int64_t)s.rl}, d{s.deg, 0, (int64_t)s.dl, (int64_t)s.dl};
            if (!s.prep) sums.push_back(SumJob{r, s.stats});
            if (!opt_.disable_global_alignment && s.rl > 0 && s.dl > 0) {
                s.lag_job = true;
                sums.push_back(SumJob{d, s.stats + 4});
                LagJob j{};
                j.a = r;
                j.b = d;
                j.biggest = (int64_t)std::max(s.rl, s.dl);
                j.n = (int64_t)host::fft_size_for((size_t)j.biggest);
                j.stats_a = s.prep ? s.prep->d_stats : s.stats;
                j.stats_b = s.stats + 4;
                j.lag_out = d_lags + i;
                lag_jobs.push_back(j);
                lag_pair.push_back(i);
                s.trace.fft_nlogn += 2.0 * (double)j.n * std::log2((double)j.n);
                timing_.lag_bytes += lag_search_bytes(j, !opt_.exact_lag_search);
            }
        }
        launch_sums(sums);
        record(lag_events_[0]);
        d_lstat = launch_lag_jobs(lag_jobs, false);
        record(lag_events_[1]);
        std::vector<size_t> all(n);
        for (size_t i = 0; i < n; ++i) all[i] = i;
        launch_aligned(all);
    }
    int64_t *h_lags = pinned_.alloc_n<int64_t>(n);
    double *h_stats = pinned_.alloc_n<double>(10 * n);
    int32_t *h_lstat = d_lstat ? pinned_.alloc_n<int32_t>(lag_jobs.size()) : nullptr;
    d2h(h_lags, d_lags, n * sizeof(int64_t));
    for (size_t i = 0; i < n; ++i)
        if (ps[i].live) d2h(h_stats + 10 * i, ps[i].stats, 10 * sizeof(double));
    if (h_lstat) d2h(h_lstat, d_lstat, lag_jobs.size() * sizeof(int32_t));
    record(events_[1]);
    sync();
    {
        // searches the f32 pass left undecided: the exact search, then those
        // pairs' aligned energies again
        const std::vector<size_t> redo = rerun_undecided(lag_jobs, h_lstat, false);
        if (!redo.empty()) {
            std::vector<size_t> pairs;
            for (size_t k : redo) pairs.push_back(lag_pair[k]);
            launch_aligned(pairs);
            for (size_t i : pairs) {
                d2h(h_lags + i, d_lags + i, sizeof(int64_t));
                d2h(h_stats + 10 * i, ps[i].stats, 10 * sizeof(double));
            }
            sync();
        }
    }
    for (size_t i = 0; i < n; ++i)
        if (ps[i].live && ps[i].prep) std::copy(ps[i].prep->stats, ps[i].prep->stats + 4, h_stats + 10 * i);

    // ---- 2: plan frames, patches and search windows (host) --------------
    std::vector<SpecJob> spec_jobs;
    std::vector<char> scale_args;
    int nscale = 0;
    int64_t max_al = 0;
    std::vector<PrepJob> prep_jobs;
    std::vector<PlaneJob> plane_jobs;
    std::vector<RefTermsJob> term_jobs;
    std::vector<TableTask> table_rows;  // one per patch: offsets [off0, hi]
    std::vector<DpJob> dp_jobs;
    std::vector<int64_t> all_lohi;  // per DP job: its patches' lo, then hi
    std::vector<size_t> lohi_at;
    std::vector<StatsJob> stat_jobs;
    int max_width = 0;
    for (size_t i = 0; i < n; ++i) {
        PairState &s = ps[i];
        if (!s.live) continue;
        try {
            const int64_t lag = s.lag_job ? h_lags[i] : 0;
            s.trace.global_lag = lag;
            s.al = opt_.disable_global_alignment ? host::Aligned{0, 0, (int64_t)s.dl, 0.0}
                                                 : host::apply_lag_geometry(s.rl, s.dl, lag, sample_rate);
            const double *st = h_stats + 10 * i;
            s.factor = host::spl_factor(st[2], s.rl, st[8], (size_t)s.al.len);
            s.al_energy = st[8];
            s.ref_energy = st[2];
            s.trace.spl_factor = s.factor;
            s.trace.deg_len = (uint64_t)s.al.len;
            if (s.rl <= W || (size_t)s.al.len <= W) throw Error(kSignal, "SpectrogramTooShort");
            s.nf_ref = host::num_frames(s.rl, W, H);
            s.nf_deg = host::num_frames((size_t)s.al.len, W, H);
            s.trace.nf_ref = s.nf_ref;
            s.trace.nf_deg = s.nf_deg;
            if (s.prep) {
                s.idx = s.prep->idx;
            } else if (opt_.speech) {
                std::vector<double> tmp;
                const double *hr = s.h_ref;
                if (!hr) {
                    tmp.resize(s.rl);
                    VQB_CUDA(cudaMemcpy(tmp.data(), s.ref, s.rl * sizeof(double), cudaMemcpyDeviceToHost));
                    hr = tmp.data();
                }
                s.idx = host::vad_patch_indices(hr, s.rl, s.nf_ref, P, W, 0.25);
            } else {
                s.idx = host::ref_patch_indices(s.nf_ref, P);
            }
            if (s.idx.empty()) throw Error(kSignal, "NoPatches");
            s.search = host::plan_search(s.idx, s.nf_ref, s.nf_deg, P, opt_.radius);
        } catch (const Error &e) {
            s.fail(e.code, e.what());
            continue;
        }
        const size_t np = s.search.np;
        s.width = s.nf_deg;
        for (size_t p = 0; p < np; ++p) s.width = std::max(s.width, (size_t)s.search.hi[p] + P);
        max_width = std::max(max_width, (int)s.width);
        s.deg_al = arena_.alloc_n<double>((size_t)s.al.len);
        s.deg_raw = arena_.alloc_n<double>(NB * s.nf_deg);
        s.ref_prep = arena_.alloc_n<double>(NB * s.nf_ref);
        s.deg_prep = arena_.alloc_n<double>(NB * s.nf_deg);
        const size_t plane = NB * s.width;
        s.pad = arena_.alloc_n<double>(4 * plane);
        s.mu = s.pad + plane;
        s.dms = s.mu + plane;
        s.sds = s.dms + plane;
        s.terms = arena_.alloc_n<double>(np * 4 * NB * P);
        s.sims = arena_.alloc_n<double>(np * s.nf_deg);
        s.dp = arena_.alloc_n<double>(np * s.nf_deg);
        s.bt = arena_.alloc_n<int64_t>(np * s.nf_deg);
        s.offs = arena_.alloc_n<int64_t>(np);
        s.valid = arena_.alloc_n<uint8_t>(np);
        s.mstats = arena_.alloc_n<double>(np * (3 * NB + 1));
        // aligned[i] = deg[i - lead + skip] (applyLag), scaled (scaleToMatchSpl)
        const VSig src{s.deg + s.al.skip, s.al.lead, (int64_t)s.dl - s.al.skip, s.al.len};
        scale_args.resize(scale_args.size() + scale_args_size());
        fill_scale_args(scale_args.data() + scale_args.size() - scale_args_size(), src, s.factor, s.deg_al);
        ++nscale;
        max_al = std::max(max_al, s.al.len);
        spec_jobs.push_back(SpecJob{VSig{s.deg_al, 0, s.al.len, s.al.len}, (int64_t)s.nf_deg, s.deg_raw});
        s.trace.n_rms += NB * (s.nf_ref + s.nf_deg);
        prep_jobs.push_back(PrepJob{s.ref_raw, s.deg_raw, s.ref_prep, s.deg_prep, (int32_t)s.nf_ref, (int32_t)s.nf_deg});
        plane_jobs.push_back(PlaneJob{s.deg_prep, (int32_t)s.nf_deg, (int32_t)s.width, s.pad, s.mu, s.dms, s.sds,
                                      opt_.form != kFormExact ? 1 : 0});
        lohi_at.push_back(all_lohi.size());
        all_lohi.insert(all_lohi.end(), s.search.lo.begin(), s.search.lo.end());
        all_lohi.insert(all_lohi.end(), s.search.hi.begin(), s.search.hi.end());
        for (size_t p = 0; p < np; ++p) {
            double *terms = s.terms + p * 4 * NB * P;
            term_jobs.push_back(RefTermsJob{s.ref_prep, (int32_t)s.nf_ref, (int32_t)s.idx[p], terms,
                                            opt_.form != kFormExact ? 1 : 0});
            table_rows.push_back(TableTask{terms, s.pad, s.mu, s.dms, s.sds, (int32_t)s.width,
                                           (int32_t)s.search.lo[p], (int32_t)s.search.hi[p], s.sims + p * s.nf_deg});
            s.trace.n_cells += (uint64_t)(s.search.hi[p] - s.search.lo[p] + 1) * NB * P;
            double *ms = s.mstats + p * (3 * NB + 1);
            stat_jobs.push_back(StatsJob{s.ref_prep, (int32_t)s.nf_ref, (int32_t)s.idx[p], s.deg_prep,
                                         (int32_t)s.nf_deg, 0, (int32_t)s.nf_deg, (int32_t)P, s.offs + p,
                                         s.valid + p, ms, ms + NB, ms + 2 * NB, ms + 3 * NB});
            s.trace.n_cells += NB * P;
        }
        dp_jobs.push_back(DpJob{s.sims, nullptr, nullptr, (int32_t)np, (int64_t)s.nf_deg, s.dp, s.bt, s.offs, s.valid});
    }
    // every pair's search windows in one upload
    if (!dp_jobs.empty()) {
        const int64_t *d_lohi = upload(all_lohi);
        for (size_t k = 0; k < dp_jobs.size(); ++k) {
            dp_jobs[k].lo = d_lohi + lohi_at[k];
            dp_jobs[k].hi = dp_jobs[k].lo + dp_jobs[k].np;
        }
    }

    // ---- 3: spectrograms, prep, NSIM table, DP, match statistics ----------
    if (nscale) launch_scale(upload_bytes(scale_args.data(), scale_args.size()), nscale, max_al, stream_);
    record(events_[2]);
    run_gammatone(spec_jobs, stream_);
    record(events_[3]);
    VQB_CUDA(cudaStreamWaitEvent(stream_, ev_ref_done_, 0));
    if (!prep_jobs.empty()) launch_prep_jobs(prep_jobs);
    record(events_[4]);
    if (!plane_jobs.empty()) launch_plane(upload(plane_jobs), (int)plane_jobs.size(), nbi, max_width, stream_);
    if (!term_jobs.empty()) launch_ref_terms(upload(term_jobs), (int)term_jobs.size(), nbi, (int)P, stream_);
    if (!table_rows.empty()) {
        const bool fast_cells = opt_.form != kFormExact;
        auto launch_width = [&](int w) {
            std::vector<TableTask> tasks;
            for (const TableTask &row : table_rows)
                for (int64_t off0 = row.off0; off0 <= row.hi; off0 += w) {
                    TableTask t = row;
                    t.off0 = (int32_t)off0;
                    tasks.push_back(t);
                }
            launch_table(upload(tasks), (int)tasks.size(), nbi, (int)P, fast_cells, w, stream_);
        };
        const int w = tuned(kTuneTable, fast_cells ? 1 : 0, nbi, table_width_candidates((int)P), launch_width, stream_);
        launch_width(w);
    }
    if (!dp_jobs.empty()) launch_dp(upload(dp_jobs), (int)dp_jobs.size(), stream_);
    if (!stat_jobs.empty()) launch_stats(upload(stat_jobs), (int)stat_jobs.size(), nbi, stream_);
    std::vector<int64_t *> h_offs(n, nullptr);
    std::vector<uint8_t *> h_valid(n, nullptr);
    std::vector<double *> h_ms(n, nullptr);
    for (size_t i = 0; i < n; ++i) {
        PairState &s = ps[i];
        if (!s.live) continue;
        const size_t np = s.search.np;
        h_offs[i] = pinned_.alloc_n<int64_t>(np);
        h_valid[i] = pinned_.alloc_n<uint8_t>(np);
        h_ms[i] = pinned_.alloc_n<double>(np * (3 * NB + 1));
        d2h(h_offs[i], s.offs, np * sizeof(int64_t));
        d2h(h_valid[i], s.valid, np);
        d2h(h_ms[i], s.mstats, np * (3 * NB + 1) * sizeof(double));
    }
    record(events_[5]);
    sync();

    // ---- 4: matches and realignment slices (host) ----------------------
    const double patch_dur = fd * (double)P;
    std::vector<SumJob> slice_sums;
    std::vector<LagJob> slice_lags;
    int64_t *d_slice_lags = nullptr;
    size_t n_slices = 0;
    for (size_t i = 0; i < n; ++i) {
        PairState &s = ps[i];
        if (!s.live) continue;
        const size_t np = s.search.np;
        s.matches.resize(np);
        for (size_t p = 0; p < np; ++p) {
            host::Match &m = s.matches[p];
            const double *ms = h_ms[i] + p * (3 * NB + 1);
            m.means.assign(ms, ms + NB);
            m.stddevs.assign(ms + NB, ms + 2 * NB);
            m.energy.assign(ms + 2 * NB, ms + 3 * NB);
            m.similarity = ms[3 * NB];
            const int64_t off = h_offs[i][p];
            if (off >= 0) {
                m.valid = h_valid[i][p] != 0;
                if (m.valid) {
                    m.deg_start = (double)off * fd;
                    m.deg_end = m.deg_start + patch_dur;
                }
                m.ref_start = (double)s.idx[p] * fd;
                m.ref_end = m.ref_start + patch_dur;
            }
            s.trace.ref_index.push_back(s.idx[p]);
            s.trace.deg_offset.push_back(off);
            s.trace.valid.push_back(m.valid ? 1 : 0);
            s.trace.realign_lag.push_back(0);
            s.trace.realign_frames.push_back(-1);
            s.trace.realign_reused.push_back(0);
            s.trace.realign_accepted.push_back(0);
        }
        if (opt_.disable_realignment) continue;
        for (size_t p = 0; p < np; ++p) {
            const host::Match &m = s.matches[p];
            if (!m.valid) continue;
            RealignPatch rp;
            rp.mi = p;
            rp.rl = host::slice_layout(s.rl, sample_rate, m.ref_start, m.ref_end);
            rp.dl = host::slice_layout((size_t)s.al.len, sample_rate, m.deg_start, m.deg_end);
            rp.rlen = rp.rl.pad + rp.rl.len;
            rp.dlen = rp.dl.pad + rp.dl.len;
            if (rp.rlen < (int64_t)W || rp.dlen < (int64_t)W) continue;
            s.rps.push_back(rp);
            ++n_slices;
        }
    }
    if (n_slices) {
        d_slice_lags = arena_.alloc_n<int64_t>(n_slices);
        double *d_sst = arena_.alloc_n<double>(8 * n_slices);
        size_t k = 0;
        for (auto &s : ps) {
            if (!s.live) continue;
            for (auto &rp : s.rps) {
                rp.stats = d_sst + 8 * k;
                const VSig a{s.ref + rp.rl.base, rp.rl.pad, rp.rl.len, rp.rlen};
                const VSig b{s.deg_al + rp.dl.base, rp.dl.pad, rp.dl.len, rp.dlen};
                slice_sums.push_back(SumJob{a, rp.stats});
                slice_sums.push_back(SumJob{b, rp.stats + 4});
                LagJob j{};
                j.a = a;
                j.b = b;
                j.biggest = std::max(rp.rlen, rp.dlen);
                j.n = (int64_t)host::fft_size_for((size_t)j.biggest);
                j.stats_a = rp.stats;
                j.stats_b = rp.stats + 4;
                j.lag_out = d_slice_lags + k;
                slice_lags.push_back(j);
                s.trace.fft_nlogn += 2.0 * (double)j.n * std::log2((double)j.n);
                ++k;
            }
        }
        // ---- 5: slice lags --------------------------------------------------
        launch_sums(slice_sums);
        int32_t *d_sstat = launch_lag_jobs(slice_lags, false);
        int64_t *h_sl = pinned_.alloc_n<int64_t>(n_slices);
        int32_t *h_sstat = d_sstat ? pinned_.alloc_n<int32_t>(n_slices) : nullptr;
        d2h(h_sl, d_slice_lags, n_slices * sizeof(int64_t));
        if (h_sstat) d2h(h_sstat, d_sstat, n_slices * sizeof(int32_t));
        sync();
        if (!rerun_undecided(slice_lags, h_sstat, false).empty()) {
            d2h(h_sl, d_slice_lags, n_slices * sizeof(int64_t));
            sync();
        }

        // ---- 6: trimmed geometry, frame reuse (host) -------------------------
        std::vector<SpecJob> rjobs;
        std::vector<CopyJob> copies;
        std::vector<PrepJob> rprep;
        std::vector<StatsJob> rstats;
        int max_cols = 0;
        k = 0;
        for (auto &s : ps) {
            if (!s.live) continue;
            for (auto &rp : s.rps) {
                rp.lag = h_sl[k++];
                s.trace.realign_lag[rp.mi] = rp.lag;
                rp.trim = host::trim_geometry(rp.rlen, rp.dlen, rp.lag, sample_rate);
                rp.nf = host::num_frames((size_t)rp.trim.len, W, H);
                s.trace.realign_frames[rp.mi] = (int64_t)rp.nf;
                if (rp.nf == 0) continue;
                max_cols = std::max(max_cols, (int)rp.nf);
                rp.rs_raw = arena_.alloc_n<double>(NB * rp.nf);
                rp.ds_raw = arena_.alloc_n<double>(NB * rp.nf);
                rp.rs = arena_.alloc_n<double>(NB * rp.nf);
                rp.ds = arena_.alloc_n<double>(NB * rp.nf);
                rp.st = arena_.alloc_n<double>(3 * NB + 1);
                const int64_t g_ref = host::reuse_frame(rp.rl, rp.trim.ref_off, H, rp.nf, s.nf_ref);
                if (g_ref >= 0) {
                    copies.push_back(CopyJob{s.ref_raw, (int32_t)s.nf_ref, (int32_t)g_ref, rp.rs_raw, (int32_t)rp.nf});
                    rp.reused |= 1;
                } else {
                    rjobs.push_back(SpecJob{VSig{s.ref + rp.rl.base, rp.rl.pad - rp.trim.ref_off, rp.rl.len, rp.trim.len},
                                            (int64_t)rp.nf, rp.rs_raw});
                    s.trace.n_rms += NB * rp.nf;
                }
                const int64_t g_deg = host::reuse_frame(rp.dl, rp.trim.deg_off, H, rp.nf, s.nf_deg);
                if (g_deg >= 0) {
                    copies.push_back(CopyJob{s.deg_raw, (int32_t)s.nf_deg, (int32_t)g_deg, rp.ds_raw, (int32_t)rp.nf});
                    rp.reused |= 2;
                } else {
                    rjobs.push_back(SpecJob{VSig{s.deg_al + rp.dl.base, rp.dl.pad - rp.trim.deg_off, rp.dl.len, rp.trim.len},
                                            (int64_t)rp.nf, rp.ds_raw});
                    s.trace.n_rms += NB * rp.nf;
                }
                s.trace.realign_reused[rp.mi] = rp.reused;
                rprep.push_back(PrepJob{rp.rs_raw, rp.ds_raw, rp.rs, rp.ds, (int32_t)rp.nf, (int32_t)rp.nf});
                rstats.push_back(StatsJob{rp.rs, (int32_t)rp.nf, 0, rp.ds, (int32_t)rp.nf, 0, (int32_t)rp.nf,
                                          (int32_t)rp.nf, nullptr, nullptr, rp.st, rp.st + NB, rp.st + 2 * NB,
                                          rp.st + 3 * NB});
                s.trace.n_cells += NB * rp.nf;
            }
        }
        // ---- 7: realigned spectrograms and statistics ------------------------
        if (!copies.empty()) launch_copy_frames(upload(copies), (int)copies.size(), nbi, max_cols, stream_);
        run_gammatone(rjobs, stream_);
        if (!rprep.empty()) launch_prep_jobs(rprep);
        if (!rstats.empty()) launch_stats(upload(rstats), (int)rstats.size(), nbi, stream_);
        std::vector<double *> h_rst;
        for (auto &s : ps) {
            if (!s.live) continue;
            for (auto &rp : s.rps) {
                if (rp.nf == 0) continue;
                double *h = pinned_.alloc_n<double>(3 * NB + 1);
                d2h(h, rp.st, (3 * NB + 1) * sizeof(double));
                h_rst.push_back(h);
            }
        }
        record(events_[6]);
        sync();

        // ---- 8: accept rule (reference src/realign.zig:398-460) --------------
        size_t q = 0;
        for (auto &s : ps) {
            if (!s.live) continue;
            for (auto &rp : s.rps) {
                if (rp.nf == 0) continue;
                const double *st = h_rst[q++];
                host::Match &m = s.matches[rp.mi];
                const double sim = st[3 * NB];
                if (!(sim < m.similarity)) {
                    m.means.assign(st, st + NB);
                    m.stddevs.assign(st + NB, st + 2 * NB);
                    m.energy.assign(st + 2 * NB, st + 3 * NB);
                    m.similarity = sim;
                    const double dur = (double)rp.trim.len / (double)sample_rate;
                    if (rp.trim.lag_seconds > 0.0)
                        m.ref_start += rp.trim.lag_seconds;
                    else
                        m.deg_start -= rp.trim.lag_seconds;
                    m.ref_end = m.ref_start + dur;
                    m.deg_end = m.deg_start + dur;
                    s.trace.realign_accepted[rp.mi] = 1;
                }
            }
        }
    }
    record(events_[7]);
    VQB_CUDA(cudaEventSynchronize(events_[7]));
    for (uint64_t g = 0; g < timing_.gammatone_launches; ++g)
        timing_.gammatone_kernel_ms += elapsed(gt_events_[2 * g], gt_events_[2 * g + 1]);
    if (!lag_jobs.empty()) timing_.lag_kernel_ms = elapsed(lag_events_[0], lag_events_[1]);
    timing_.kernel_launches = launch_counter() - launches0;

    auto finish = [&](size_t i) {
        PairState &s = ps[i];
        PairOutcome &o = out[i];
        if (!s.live) {
            o.code = s.code;
            o.message = s.msg;
            return;
        }
        try {
            s.trace.n_rms_window = W;
            o.scores = host::build_scores(std::move(s.matches), NB, fd, svr_.get(), opt_.speech, opt_.unscaled_speech,
                                          rc.fb.cf, s.al.lag_seconds, lattice_.get());
            o.trace = std::move(s.trace);
        } catch (const Error &e) {
            o.code = e.code;
            o.message = e.what();
        } catch (const std::exception &e) {
            o.code = kInternal;
            o.message = e.what();
        }
    };
    // The lattice mapping runs a few milliseconds of host interpreter per
    // pair: spread it over host threads (results are per pair).
    const size_t workers = lattice_ ? std::min<size_t>(n, std::max(1u, std::thread::hardware_concurrency() / 2)) : 1;
    if (workers > 1) {
        std::vector<std::thread> pool;
        for (size_t w = 0; w < workers; ++w)
            pool.emplace_back([&, w] {
                for (size_t i = w; i < n; i += workers) finish(i);
            });
        for (auto &t : pool) t.join();
    } else {
        for (size_t i = 0; i < n; ++i) finish(i);
    }
    if (grads) {
        for (size_t i = 0; i < n; ++i)
            if (ps[i].live && out[i].code == 0) ps[i].grad_ok = true;
        gradients(ps.data(), n, deg_lens, rc, out);
    }
    timing_.total_ms = elapsed(events_[0], events_[7]);
    timing_.lag_ms = elapsed(events_[0], events_[1]);
    timing_.spectrogram_ms = elapsed(events_[2], events_[3]);
    timing_.prep_ms = elapsed(events_[3], events_[4]);
    timing_.nsim_ms = elapsed(events_[4], events_[5]);
    timing_.realign_ms = n_slices ? elapsed(events_[5], events_[6]) : 0.0;
}

void Engine::measure_batch_streamed(size_t n, const double *const *refs, const size_t *ref_lens,
                                    const double *const *degs, const size_t *deg_lens, uint32_t sample_rate,
                                    std::vector<PairOutcome> &out, const PreparedRef *const *prepared) {
    // Bytes each pair uploads, each signal at a 256-byte boundary of its slot.
    auto up = [](size_t len) { return (len * sizeof(double) + 255) & ~size_t(255); };
    auto ref_up = [&](size_t i) {
        return (prepared && prepared[i]) || !refs[i] ? size_t(0) : up(ref_lens[i]);
    };
    auto deg_up = [&](size_t i) { return degs[i] ? up(deg_lens[i]) : size_t(0); };
    size_t total = 0;
    for (size_t i = 0; i < n; ++i) total += ref_up(i) + deg_up(i);
    // Below ~64 MiB the exposed first upload and the per-chunk host work
    // outweigh the overlap (VISQOL_STREAMED_MIN_BYTES overrides the bound).
    size_t min_bytes = size_t(64) << 20;
    if (const char *env = std::getenv("VISQOL_STREAMED_MIN_BYTES")) min_bytes = (size_t)std::strtoull(env, nullptr, 10);
    if (n < 2 || total < min_bytes) {
        measure_batch(n, refs, ref_lens, degs, deg_lens, sample_rate, false, out, prepared);
        return;
    }
    // Chunks of 1/16, 1/8, 1/4 ... of the bytes (a small first chunk keeps
    // the exposed first upload short; each later upload has the previous,
    // half-as-large chunk's scoring to hide behind); a tail smaller than
    // half the next target joins the last chunk.
    std::vector<size_t> bounds{0};
    {
        size_t target = std::max<size_t>(1, total / 16), acc = 0, left = total;
        for (size_t i = 0; i < n; ++i) {
            const size_t b = ref_up(i) + deg_up(i);
            acc += b;
            left -= b;
            if (acc >= target && i + 1 < n) {
                if (left < target) continue;  // the rest is small: keep it in this chunk
                bounds.push_back(i + 1);
                acc = 0;
                target *= 2;
            }
        }
        bounds.push_back(n);
    }
    const size_t K = bounds.size() - 1;
    std::vector<size_t> chunk_bytes(K, 0);
    for (size_t k = 0; k < K; ++k)
        for (size_t i = bounds[k]; i < bounds[k + 1]; ++i) chunk_bytes[k] += ref_up(i) + deg_up(i);
    VQB_CUDA(cudaSetDevice(device_));
    for (int sl = 0; sl < 2; ++sl) {
        size_t need = 0;
        for (size_t k = sl; k < K; k += 2) need = std::max(need, chunk_bytes[k]);
        if (need > slot_bytes_[sl]) {
            VQB_CUDA(cudaStreamSynchronize(copy_));
            if (slot_[sl]) VQB_CUDA(cudaFree(slot_[sl]));
            slot_[sl] = nullptr;
            slot_bytes_[sl] = 0;
            VQB_CUDA(cudaMalloc(&slot_[sl], need));
            slot_bytes_[sl] = need;
        }
    }
    // Device views of chunk k's signals in slot k & 1 (NULL where the pair
    // has nothing to upload, so measure_batch reports it as the host path does).
    std::vector<const double *> d_ref(n, nullptr), d_deg(n, nullptr);
    for (size_t k = 0; k < K; ++k) {
        char *base = reinterpret_cast<char *>(slot_[k & 1]);
        size_t off = 0;
        for (size_t i = bounds[k]; i < bounds[k + 1]; ++i) {
            if (ref_up(i)) d_ref[i] = reinterpret_cast<const double *>(base + off), off += ref_up(i);
            if (deg_up(i)) d_deg[i] = reinterpret_cast<const double *>(base + off), off += deg_up(i);
        }
    }
    // A chunk goes up one copy at a time (each signal, in pieces of at most
    // 64 MiB), the next issued when the previous has landed: the scoring
    // streams' own small uploads (job arrays) share the copy engines, and
    // behind a whole queued chunk they would stall their kernels until the
    // chunk had landed. Measured on the 10 s 48 kHz batch, one copy in flight
    // beat finer pieces with more in flight and the whole chunk queued at
    // once.
    constexpr size_t kPiece = size_t(64) << 20;
    auto upload_chunk = [&](size_t k) {
        VQB_CUDA(cudaSetDevice(device_));
        size_t pieces = 0;
        auto copy = [&](const double *dst, const double *src, size_t len) {
            const char *s8 = reinterpret_cast<const char *>(src);
            char *d8 = reinterpret_cast<char *>(const_cast<double *>(dst));
            const size_t bytes = len * sizeof(double);
            for (size_t o = 0; o < bytes; o += kPiece, ++pieces) {
                if (pieces) VQB_CUDA(cudaEventSynchronize(ev_piece_));
                VQB_CUDA(cudaMemcpyAsync(d8 + o, s8 + o, std::min(kPiece, bytes - o), cudaMemcpyHostToDevice, copy_));
                VQB_CUDA(cudaEventRecord(ev_piece_, copy_));
            }
        };
        for (size_t i = bounds[k]; i < bounds[k + 1]; ++i) {
            if (d_ref[i] && ref_lens[i]) copy(d_ref[i], refs[i], ref_lens[i]);
            if (d_deg[i] && deg_lens[i]) copy(d_deg[i], degs[i], deg_lens[i]);
        }
        VQB_CUDA(cudaEventRecord(ev_up_[k & 1], copy_));
    };
    out.assign(n, PairOutcome{});
    Timing sum{};
    uint64_t h2d = 0;
    for (size_t i = 0; i < n; ++i)
        h2d += (d_ref[i] ? ref_lens[i] : 0) * sizeof(double) + (d_deg[i] ? deg_lens[i] : 0) * sizeof(double);
    std::vector<PairOutcome> part;
    upload_chunk(0);
    for (size_t k = 0; k < K; ++k) {
        // Chunk k+1 goes into the other slot, last read by chunk k-1, whose
        // scoring has returned (measure_batch ends with its stream drained).
        std::future<void> next;
        if (k + 1 < K) next = std::async(std::launch::async, upload_chunk, k + 1);
        VQB_CUDA(cudaStreamWaitEvent(stream_, ev_up_[k & 1], 0));
        const size_t b0 = bounds[k], m = bounds[k + 1] - b0;
        measure_batch(m, d_ref.data() + b0, ref_lens + b0, d_deg.data() + b0, deg_lens + b0, sample_rate, true,
                      part, prepared ? prepared + b0 : nullptr, refs + b0);
        if (next.valid()) next.get();
        for (size_t j = 0; j < m; ++j) out[b0 + j] = std::move(part[j]);
        const Timing &t = timing_;
        sum.total_ms += t.total_ms;
        sum.lag_ms += t.lag_ms;
        sum.spectrogram_ms += t.spectrogram_ms;
        sum.prep_ms += t.prep_ms;
        sum.nsim_ms += t.nsim_ms;
        sum.realign_ms += t.realign_ms;
        sum.gammatone_kernel_ms += t.gammatone_kernel_ms;
        sum.gammatone_launches += t.gammatone_launches;
        sum.gammatone_rms += t.gammatone_rms;
        sum.gammatone_window = std::max(sum.gammatone_window, t.gammatone_window);
        sum.kernel_launches += t.kernel_launches;
        sum.h2d_bytes += t.h2d_bytes;
        sum.d2h_bytes += t.d2h_bytes;
        sum.host_syncs += t.host_syncs;
        sum.lag_kernel_ms += t.lag_kernel_ms;
        sum.lag_bytes += t.lag_bytes;
        sum.lag_reruns += t.lag_reruns;
    }
    sum.h2d_bytes += h2d;
    timing_ = sum;
}

}  // namespace vqb

namespace vqb {

void Engine::gradients(detail::PairState *ps, size_t n, const size_t *deg_lens, const RateCache &rc,
                       std::vector<PairOutcome> &out) {
    const size_t NB = nb_, P = patch_, W = rc.geo.window, H = rc.geo.hop;
    const double fd = rc.geo.frame_duration;
    // 1. the raw spectrograms the statistics came from, and the degraded samples
    struct HostCopy {
        std::vector<double> ref, deg, sig;
        std::vector<std::vector<double>> rs, ds;  // per realignment patch
    };
    std::vector<HostCopy> hc(n);
    auto fetch = [&](std::vector<double> &dst, const double *src, size_t count) {
        dst.resize(count);
        if (count) VQB_CUDA(cudaMemcpyAsync(dst.data(), src, count * sizeof(double), cudaMemcpyDeviceToHost, stream_));
        timing_.d2h_bytes += count * sizeof(double);
    };
    for (size_t i = 0; i < n; ++i) {
        PairState &s = ps[i];
        if (!s.grad_ok) continue;
        HostCopy &h = hc[i];
        fetch(h.ref, s.ref_raw, NB * s.nf_ref);
        fetch(h.deg, s.deg_raw, NB * s.nf_deg);
        fetch(h.sig, s.deg, s.dl);
        h.rs.resize(s.rps.size());
        h.ds.resize(s.rps.size());
        for (size_t k = 0; k < s.rps.size(); ++k)
            if (s.rps[k].nf) {
                fetch(h.rs[k], s.rps[k].rs_raw, NB * s.rps[k].nf);
                fetch(h.ds[k], s.rps[k].ds_raw, NB * s.rps[k].nf);
            }
    }
    sync();

    // 2. host reverses: MOS -> match statistics -> prepared cells -> raw
    // degraded cells, for the global spectrograms and each accepted
    // realignment slice
    std::vector<std::vector<double>> g_glob(n);
    struct SliceGrad {
        size_t pair, rp;
        std::vector<double> g;
    };
    std::vector<SliceGrad> slice_grads;
    for (size_t i = 0; i < n; ++i) {
        PairState &s = ps[i];
        if (!s.grad_ok) continue;
        const HostCopy &h = hc[i];
        const std::vector<host::Match> &matches = out[i].scores.patches;
        const PairTrace &tr = out[i].trace;
        const size_t nfr = s.nf_ref, nfd = s.nf_deg;
        std::vector<host::MatchGrad> mg;
        host::scores_grad(matches, NB, fd, svr_.get(), opt_.speech, opt_.unscaled_speech, lattice_.get(), mg);
        std::vector<double> rprep, dprep;
        host::prepare_forward(h.ref.data(), h.deg.data(), NB, nfr, nfd, rprep, dprep);
        std::vector<double> g_ref(NB * nfr, 0.0), g_deg(NB * nfd, 0.0);
        g_glob[i].assign(NB * nfd, 0.0);
        std::vector<double> pr(NB * P), pd(NB * P), dr(NB * P), dd(NB * P);
        for (size_t p = 0; p < matches.size(); ++p) {
            if (!tr.valid[p] || tr.deg_offset[p] < 0) continue;  // statistics are constants
            const host::MatchGrad &g = mg[p];
            if (tr.realign_accepted[p]) {
                size_t k = 0;
                while (k < s.rps.size() && !(s.rps[k].mi == p && s.rps[k].nf)) ++k;
                if (k == s.rps.size()) continue;
                const RealignPatch &rp = s.rps[k];
                const size_t nf = rp.nf;
                std::vector<double> a, b, da(NB * nf, 0.0), db(NB * nf, 0.0), gds(NB * nf, 0.0);
                host::prepare_forward(h.rs[k].data(), h.ds[k].data(), NB, nf, nf, a, b);
                host::patch_similarity_grad(a.data(), b.data(), NB, nf, g.dmeans.data(), g.dstddevs.data(),
                                            g.denergy.data(), da.data(), db.data());
                host::prepare_grad(h.rs[k].data(), h.ds[k].data(), NB, nf, nf, da.data(), db.data(), gds.data());
                if (rp.reused & 2) {
                    // the slice's degraded frames were the global spectrogram's
                    const int64_t g0 = host::reuse_frame(rp.dl, rp.trim.deg_off, H, nf, nfd);
                    for (size_t bb = 0; bb < NB; ++bb)
                        for (size_t f = 0; f < nf; ++f) g_glob[i][bb * nfd + g0 + f] += gds[bb * nf + f];
                } else {
                    slice_grads.push_back(SliceGrad{i, k, std::move(gds)});
                }
                continue;
            }
            const size_t idx = (size_t)tr.ref_index[p], off = (size_t)tr.deg_offset[p];
            for (size_t bb = 0; bb < NB; ++bb)
                for (size_t c = 0; c < P; ++c) {
                    pr[bb * P + c] = rprep[bb * nfr + idx + c];
                    pd[bb * P + c] = off + c < nfd ? dprep[bb * nfd + off + c] : 0.0;
                }
            std::fill(dr.begin(), dr.end(), 0.0);
            std::fill(dd.begin(), dd.end(), 0.0);
            host::patch_similarity_grad(pr.data(), pd.data(), NB, P, g.dmeans.data(), g.dstddevs.data(),
                                        g.denergy.data(), dr.data(), dd.data());
            for (size_t bb = 0; bb < NB; ++bb)
                for (size_t c = 0; c < P; ++c) {
                    g_ref[bb * nfr + idx + c] += dr[bb * P + c];
                    if (off + c < nfd) g_deg[bb * nfd + off + c] += dd[bb * P + c];
                }
        }
        host::prepare_grad(h.ref.data(), h.deg.data(), NB, nfr, nfd, g_ref.data(), g_deg.data(), g_glob[i].data());
    }

    // 3. the gammatone reverse on the device, into each pair's gradient with
    // respect to its scaled, aligned degraded signal
    std::vector<GradSpecJob> jobs;
    std::vector<double *> d_g(n, nullptr);
    for (size_t i = 0; i < n; ++i) {
        PairState &s = ps[i];
        if (!s.grad_ok) continue;
        d_g[i] = arena_.alloc_n<double>((size_t)s.al.len);
        launch_zero(d_g[i], (size_t)s.al.len * sizeof(double), stream_);
        jobs.push_back(GradSpecJob{VSig{s.deg_al, 0, s.al.len, s.al.len}, (int64_t)s.nf_deg, upload(g_glob[i]), d_g[i]});
    }
    for (const SliceGrad &sg : slice_grads) {
        PairState &s = ps[sg.pair];
        const RealignPatch &rp = s.rps[sg.rp];
        jobs.push_back(GradSpecJob{VSig{s.deg_al + rp.dl.base, rp.dl.pad - rp.trim.deg_off, rp.dl.len, rp.trim.len},
                                   (int64_t)rp.nf, upload(sg.g), d_g[sg.pair] + rp.dl.base});
    }
    if (!jobs.empty()) {
        const int F = gammatone_bwd_frames_per_cta();
        const size_t tsz = gammatone_tile_size();
        std::vector<char> tiles;
        int ntiles = 0;
        for (size_t j = 0; j < jobs.size(); ++j)
            for (int64_t f = 0; f < jobs[j].nf; f += F, ++ntiles) {
                tiles.resize(tiles.size() + tsz);
                fill_gammatone_tile(tiles.data() + tiles.size() - tsz, (int)j, (int)f);
            }
        const GradSpecJob *d_jobs = upload(jobs);
        const void *d_tiles = upload_bytes(tiles.data(), tiles.size());
        double *scratch = arena_.alloc_n<double>(gammatone_bwd_scratch_count(ntiles, (int)W));
        launch_gammatone_bwd(d_jobs, d_tiles, ntiles, rc.d_fast_coeffs, (int)NB, rc.d_hann, (int)W, (int)H, scratch,
                             stream_);
    }
    std::vector<std::vector<double>> g_al(n);
    for (size_t i = 0; i < n; ++i)
        if (ps[i].grad_ok) fetch(g_al[i], d_g[i], (size_t)ps[i].al.len);
    sync();

    // 4. the SPL scaling (scaled = factor x aligned, factor ~ |aligned|^-1)
    // and the lag (aligned[i] = deg[i - lead + skip]) reversed
    for (size_t i = 0; i < n; ++i) {
        PairState &s = ps[i];
        if (!s.grad_ok) continue;
        const std::vector<double> &x = hc[i].sig, &g = g_al[i];
        const int64_t lead = s.al.lead, skip = s.al.skip, L = s.al.len;
        auto aligned = [&](int64_t k) {
            const int64_t d = k - lead + skip;
            return k >= lead && d >= 0 && d < (int64_t)s.dl ? x[(size_t)d] : 0.0;
        };
        const double f = s.factor, E = s.al_energy;
        const bool depends = s.ref_energy > 0.0 && E > 0.0 && s.rl > 0 && L > 0;
        double dldf = 0.0;
        if (depends)
            for (int64_t k = 0; k < L; ++k) dldf += g[(size_t)k] * aligned(k);
        std::vector<double> &gd = out[i].grad;
        gd.assign(deg_lens[i], 0.0);
        for (int64_t k = lead; k < L; ++k) {
            const int64_t d = k - lead + skip;
            if (d < 0 || d >= (int64_t)s.dl) continue;
            gd[(size_t)d] = f * g[(size_t)k] - (depends ? dldf * f * aligned(k) / E : 0.0);
        }
    }
}

}  // namespace vqb
