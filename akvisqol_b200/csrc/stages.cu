// Single-stage entry points of include/visqol_b200.h: each copies host
// buffers in, runs one kernel family of the batch pipeline, and copies the
// result out. They exist so that each kernel can be checked on its own
// against the CPU model; the batch pipeline does not use them.
#include <algorithm>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/visqol_b200.h"
#include "engine.h"
#include "grad_host.h"
#include "host_model.h"
#include "kernels.h"

using vqb::Error;

namespace {

int stage_fail(int code, const char *m) {
    vqb::set_last_error(m);
    return code;
}

// Device buffer freed on scope exit.
template <class T>
struct DBuf {
    T *p = nullptr;
    explicit DBuf(size_t n) { VQB_CUDA(cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T))); }
    DBuf(const T *h, size_t n) : DBuf(n) {
        // A copy from pageable memory may return before its DMA lands; the
        // kernels run on a non-blocking stream, so wait for it.
        if (n) {
            VQB_CUDA(cudaMemcpy(p, h, n * sizeof(T), cudaMemcpyHostToDevice));
            VQB_CUDA(cudaDeviceSynchronize());
        }
    }
    ~DBuf() { cudaFree(p); }
    void get(T *h, size_t n) const {
        if (n) VQB_CUDA(cudaMemcpy(h, p, n * sizeof(T), cudaMemcpyDeviceToHost));
    }
};

// One engine per process and arithmetic form for the stage calls (its
// stream and caches).
vqb::Engine &stage_engine(int form = vqb::kFormExact) {
    static std::mutex mu;
    static std::unique_ptr<vqb::Engine> e[3];
    std::lock_guard<std::mutex> lock(mu);
    if (!e[form]) {
        int dev = 0;
        cudaGetDevice(&dev);
        vqb::Options o;
        o.form = form;
        o.exact_lag_search = form == vqb::kFormExact;  // the stage lag calls' exact search
        e[form] = std::make_unique<vqb::Engine>(dev, o, nullptr);
    }
    return *e[form];
}

template <class F>
int guarded(F &&f) {
    try {
        f();
        VQB_CUDA(cudaGetLastError());
        VQB_CUDA(cudaDeviceSynchronize());
        return VISQOL_OK;
    } catch (const Error &e) {
        stage_fail(e.code, e.what());
        return e.code;
    } catch (const std::exception &e) {
        stage_fail(VISQOL_E_INTERNAL, e.what());
        return VISQOL_E_INTERNAL;
    }
}

}  // namespace

extern "C" {

int visqol_b200_spectrogram(size_t nb, const double *coeffs, const double *hann, size_t window, size_t hop,
                            const double *x, size_t len, double *out, size_t *nf_out) {
    if (!coeffs || !hann || (!x && len) || !out || !nf_out || nb == 0 || nb > 32 || hop == 0)
        return stage_fail(VISQOL_E_INVALID_ARGUMENT, "invalid argument");
    return guarded([&] {
        vqb::host::Filterbank fb;
        fb.nb = nb;
        fb.coeffs.assign(coeffs, coeffs + 8 * nb);
        for (size_t b = 0; b < nb; ++b) fb.run.push_back(vqb::host::band_coeffs(coeffs + 8 * b));
        const size_t nf = vqb::host::num_frames(len, window, hop);
        *nf_out = nf;
        DBuf<double> dx(x, len), dh(hann, window), dout(nb * nf);
        stage_engine().spectrogram(fb, dh.p, window, hop, dx.p, len, dout.p, nf);
        dout.get(out, nb * nf);
    });
}

static int lag_stage(const double *a, size_t la, const double *b, size_t lb, int64_t *lag, bool raw) {
    if ((!a && la) || (!b && lb) || !lag) return stage_fail(VISQOL_E_INVALID_ARGUMENT, "invalid argument");
    return guarded([&] {
        DBuf<double> da(a, la), db(b, lb);
        const vqb::VSig va{da.p, 0, (int64_t)la, (int64_t)la}, vb{db.p, 0, (int64_t)lb, (int64_t)lb};
        stage_engine().lags(1, &va, &vb, raw, lag);
    });
}

int visqol_b200_envelope_lag(const double *a, size_t la, const double *b, size_t lb, int64_t *lag) {
    return lag_stage(a, la, b, lb, lag, false);
}

int visqol_b200_signal_sums(const double *x, size_t len, size_t skip, double *out) {
    if ((!x && len) || !out || skip > len) return stage_fail(VISQOL_E_INVALID_ARGUMENT, "invalid argument");
    return guarded([&] {
        DBuf<double> dx(x, len), dout(8);
        const int64_t n = (int64_t)len, k = (int64_t)skip;
        const vqb::SumJob whole{vqb::VSig{dx.p, 0, n, n}, dout.p};
        // x[skip..] as a window: sample(i) = x[i + skip]
        const vqb::SumJob tail{vqb::VSig{dx.p, -k, n, n - k}, dout.p + 4};
        DBuf<vqb::SumJob> dw(&whole, 1), dt(&tail, 1);
        vqb::launch_envelope_stats(dw.p, 1, 0);
        vqb::launch_energy(dt.p, 1, 0);
        VQB_CUDA(cudaDeviceSynchronize());
        double h[8];
        dout.get(h, 8);
        out[0] = h[0];
        out[1] = h[1];
        out[2] = h[2];
        out[3] = h[3];
        out[4] = h[6];
    });
}

int visqol_b200_best_lag(const double *a, size_t la, const double *b, size_t lb, int64_t *lag) {
    return lag_stage(a, la, b, lb, lag, true);
}

int visqol_b200_lag_search(const double *a, size_t la, const double *b, size_t lb, int raw, int form, int64_t *lag,
                           int32_t *undecided, float *corr, size_t corr_len) {
    if ((!a && la) || (!b && lb) || !lag || (form != 0 && form != 1))
        return stage_fail(VISQOL_E_INVALID_ARGUMENT, "invalid argument");
    const size_t n = vqb::host::fft_size_for(std::max(la, lb));
    if (corr && (form != 1 || corr_len != n || std::max(la, lb) == 0 || n > ((size_t)1 << 24)))
        return stage_fail(VISQOL_E_INVALID_ARGUMENT, "corr needs form 1 and corr_len = fftSizeFor(max(la, lb))");
    return guarded([&] {
        DBuf<double> da(a, la), db(b, lb);
        std::unique_ptr<DBuf<float>> dc;
        if (corr) dc = std::make_unique<DBuf<float>>(n);
        const vqb::VSig va{da.p, 0, (int64_t)la, (int64_t)la}, vb{db.p, 0, (int64_t)lb, (int64_t)lb};
        int32_t st = 0;
        stage_engine(form == 1 ? vqb::kFormF32 : vqb::kFormExact)
            .lags(1, &va, &vb, raw != 0, lag, &st, dc ? dc->p : nullptr);
        if (undecided) *undecided = st;
        if (dc) dc->get(corr, n);
    });
}

int visqol_b200_refine_lag(const double *s1, size_t l1, const double *s2, size_t l2, const float *approx, size_t n,
                           double scale, double tol, int64_t *lag, int32_t *decided) {
    if ((!s1 && l1) || (!s2 && l2) || !approx || !lag || !decided || l1 == 0 || l2 == 0 ||
        n < 2 * std::max(l1, l2) - 1 || n > ((size_t)1 << 31))
        return stage_fail(VISQOL_E_INVALID_ARGUMENT, "invalid argument (n must be at least 2 max(l1, l2) - 1)");
    return guarded([&] {
        double e1 = 0.0, e2 = 0.0;
        for (size_t i = 0; i < l1; ++i) e1 += s1[i] * s1[i];
        for (size_t i = 0; i < l2; ++i) e2 += s2[i] * s2[i];
        const double slack = 2.0 * tol * (e1 + e2) * scale;
        DBuf<double> da(s1, l1), db(s2, l2);
        DBuf<float> dx(approx, n);
        const vqb::VSig va{da.p, 0, (int64_t)l1, (int64_t)l1}, vb{db.p, 0, (int64_t)l2, (int64_t)l2};
        *decided = stage_engine(vqb::kFormF32).refine_approx(va, vb, dx.p, (int64_t)n, slack, e1 + e2, lag) ? 1 : 0;
    });
}

int visqol_b200_nsim_quotient(const double *num, const double *den, size_t n, double *out) {
    if ((!num || !den || !out) && n) return stage_fail(VISQOL_E_INVALID_ARGUMENT, "invalid argument");
    return guarded([&] {
        vqb::Engine &e = stage_engine();
        DBuf<double> dn(num, n), dd(den, n), dq(n);
        vqb::launch_fast_quotient(dn.p, dd.p, dq.p, n, e.stream());
        VQB_CUDA(cudaStreamSynchronize(e.stream()));
        dq.get(out, n);
    });
}

int visqol_b200_patch_similarity_grad(const double *ref, const double *deg, size_t nrows, size_t ncols,
                                      const double *dmeans, const double *dstddevs, const double *denergy,
                                      double *dref, double *ddeg) {
    if (!ref || !deg || !dref || !ddeg || nrows == 0 || ncols == 0)
        return stage_fail(VISQOL_E_INVALID_ARGUMENT, "invalid argument");
    try {
        vqb::host::patch_similarity_grad(ref, deg, nrows, ncols, dmeans, dstddevs, denergy, dref, ddeg);
    } catch (const std::exception &e) {
        return stage_fail(VISQOL_E_INTERNAL, e.what());
    }
    return VISQOL_OK;
}

int visqol_b200_prepare_grad(const double *ref_raw, const double *deg_raw, size_t nb, size_t nfr, size_t nfd,
                             const double *g_ref, const double *g_deg, double *g_deg_raw) {
    if (!ref_raw || !deg_raw || !g_ref || !g_deg || !g_deg_raw || nb == 0)
        return stage_fail(VISQOL_E_INVALID_ARGUMENT, "invalid argument");
    try {
        vqb::host::prepare_grad(ref_raw, deg_raw, nb, nfr, nfd, g_ref, g_deg, g_deg_raw);
    } catch (const std::exception &e) {
        return stage_fail(VISQOL_E_INTERNAL, e.what());
    }
    return VISQOL_OK;
}

int visqol_b200_fft(double *buf, size_t n, int inverse) {
    if (!buf || n == 0 || (n & (n - 1))) return stage_fail(VISQOL_E_INVALID_ARGUMENT, "n must be a power of two");
    return guarded([&] {
        vqb::Engine &e = stage_engine();
        DBuf<double2> z(reinterpret_cast<const double2 *>(buf), n);
        const auto tw = e.twiddles(n);
        vqb::launch_fft(z.p, (int64_t)n, inverse != 0, tw.top, tw.block, 1, (int64_t)n, e.stream());
        VQB_CUDA(cudaStreamSynchronize(e.stream()));
        z.get(reinterpret_cast<double2 *>(buf), n);
    });
}

int visqol_b200_prepare_for_comparison(double *ref, double *deg, size_t nb, size_t nfr, size_t nfd) {
    if ((!ref && nfr) || (!deg && nfd) || nb == 0 || nb > 32)
        return stage_fail(VISQOL_E_INVALID_ARGUMENT, "invalid argument (1 <= nb <= 32)");
    return guarded([&] {
        vqb::Engine &e = stage_engine();
        DBuf<double> ri(ref, nb * nfr), di(deg, nb * nfd), ro(nb * nfr), dout(nb * nfd);
        vqb::PrepJob pj{ri.p, di.p, ro.p, dout.p, (int32_t)nfr, (int32_t)nfd};
        DBuf<vqb::PrepJob> dj(&pj, 1);
        const int max_frames = (int)std::max(nfr, nfd);
        DBuf<double> scratch(std::max<size_t>(1, vqb::prep_scratch_count(1, max_frames)));
        vqb::launch_prep(dj.p, 1, (int)nb, max_frames, scratch.p, e.stream());
        VQB_CUDA(cudaStreamSynchronize(e.stream()));
        ro.get(ref, nb * nfr);
        dout.get(deg, nb * nfd);
    });
}

int visqol_b200_log10(const double *x, size_t n, double *out) {
    if ((!x || !out) && n) return stage_fail(VISQOL_E_INVALID_ARGUMENT, "invalid argument");
    return guarded([&] {
        vqb::Engine &e = stage_engine();
        DBuf<double> dx(x, n), dy(n);
        vqb::launch_log10(dx.p, (int64_t)n, dy.p, e.stream());
        VQB_CUDA(cudaStreamSynchronize(e.stream()));
        dy.get(out, n);
    });
}

int visqol_b200_nsim_table(const double *ref_spec, size_t nf_ref, const double *deg_spec, size_t nf_deg, size_t nb,
                           size_t patch, size_t np, const int64_t *ref_idx, const int64_t *lo, const int64_t *hi,
                           double *out) {
    if (!ref_spec || !deg_spec || !ref_idx || !lo || !hi || !out || nb == 0 || patch == 0)
        return stage_fail(VISQOL_E_INVALID_ARGUMENT, "invalid argument");
    for (size_t p = 0; p < np; ++p)
        if (lo[p] < 0 || hi[p] < lo[p] || (size_t)hi[p] >= nf_deg || ref_idx[p] < 0 ||
            (size_t)ref_idx[p] + patch > nf_ref)
            return stage_fail(VISQOL_E_INVALID_ARGUMENT, "patch window out of range");
    return guarded([&] {
        vqb::Engine &e = stage_engine();
        size_t width = nf_deg;
        for (size_t p = 0; p < np; ++p) width = std::max(width, (size_t)hi[p] + patch);
        DBuf<double> rs(ref_spec, nb * nf_ref), ds(deg_spec, nb * nf_deg), plane(4 * nb * width),
            terms(np * 4 * nb * patch), sims(np * nf_deg);
        VQB_CUDA(cudaMemsetAsync(sims.p, 0, std::max<size_t>(1, np * nf_deg) * sizeof(double), e.stream()));
        const size_t pl = nb * width;
        vqb::PlaneJob pj{ds.p, (int32_t)nf_deg, (int32_t)width, plane.p, plane.p + pl, plane.p + 2 * pl, plane.p + 3 * pl,
                         0};
        std::vector<vqb::RefTermsJob> tj;
        std::vector<vqb::TableTask> tasks;
        for (size_t p = 0; p < np; ++p) {
            double *t = terms.p + p * 4 * nb * patch;
            tj.push_back(vqb::RefTermsJob{rs.p, (int32_t)nf_ref, (int32_t)ref_idx[p], t, 0});
            for (int64_t o = lo[p]; o <= hi[p]; o += vqb::table_offsets_per_cta())
                tasks.push_back(vqb::TableTask{t, pj.pad, pj.mu, pj.dms, pj.sds, (int32_t)width, (int32_t)o,
                                               (int32_t)hi[p], sims.p + p * nf_deg});
        }
        DBuf<vqb::PlaneJob> dpj(&pj, 1);
        DBuf<vqb::RefTermsJob> dtj(tj.data(), tj.size());
        DBuf<vqb::TableTask> dtasks(tasks.data(), tasks.size());
        vqb::launch_plane(dpj.p, 1, (int)nb, (int)width, e.stream());
        vqb::launch_ref_terms(dtj.p, (int)tj.size(), (int)nb, (int)patch, e.stream());
        vqb::launch_table(dtasks.p, (int)tasks.size(), (int)nb, (int)patch, false, vqb::table_offsets_per_cta(),
                          e.stream());
        VQB_CUDA(cudaStreamSynchronize(e.stream()));
        sims.get(out, np * nf_deg);
    });
}

int visqol_b200_dp(const double *sims, size_t np, size_t nf_deg, const int64_t *lo, const int64_t *hi,
                   int64_t *offset, uint8_t *valid, size_t *reached) {
    if (!sims || !lo || !hi || !offset || !valid || np == 0) return stage_fail(VISQOL_E_INVALID_ARGUMENT, "invalid argument");
    for (size_t p = 0; p < np; ++p)
        if (lo[p] < 0 || hi[p] < lo[p] || (size_t)hi[p] >= nf_deg || (p && lo[p] < lo[p - 1]))
            return stage_fail(VISQOL_E_INVALID_ARGUMENT, "window out of range");
    return guarded([&] {
        vqb::Engine &e = stage_engine();
        DBuf<double> ds(sims, np * nf_deg), dpb(np * nf_deg);
        DBuf<int64_t> dlo(lo, np), dhi(hi, np), bt(np * nf_deg), off(np);
        DBuf<uint8_t> val(np);
        vqb::DpJob job{ds.p, dlo.p, dhi.p, (int32_t)np, (int64_t)nf_deg, dpb.p, bt.p, off.p, val.p};
        DBuf<vqb::DpJob> dj(&job, 1);
        vqb::launch_dp(dj.p, 1, e.stream());
        VQB_CUDA(cudaStreamSynchronize(e.stream()));
        off.get(offset, np);
        val.get(valid, np);
        size_t r = 0;
        for (size_t p = 0; p < np; ++p) r += offset[p] >= 0;
        if (reached) *reached = r;
    });
}

int visqol_b200_patch_similarity(const double *ref, const double *deg, size_t nrows, size_t ncols, double *means,
                                 double *stddevs, double *deg_energy, double *mean) {
    if (!ref || !deg || !means || !stddevs || !deg_energy || !mean || nrows == 0 || nrows > 32 || ncols == 0)
        return stage_fail(VISQOL_E_INVALID_ARGUMENT, "invalid argument");
    return guarded([&] {
        vqb::Engine &e = stage_engine();
        DBuf<double> dr(ref, nrows * ncols), dd(deg, nrows * ncols), st(3 * nrows + 1);
        vqb::StatsJob job{dr.p, (int32_t)ncols, 0, dd.p, (int32_t)ncols, 0, (int32_t)ncols, (int32_t)ncols,
                          nullptr, nullptr, st.p, st.p + nrows, st.p + 2 * nrows, st.p + 3 * nrows};
        DBuf<vqb::StatsJob> dj(&job, 1);
        vqb::launch_stats(dj.p, 1, (int)nrows, e.stream());
        VQB_CUDA(cudaStreamSynchronize(e.stream()));
        std::vector<double> h(3 * nrows + 1);
        st.get(h.data(), h.size());
        std::memcpy(means, h.data(), nrows * sizeof(double));
        std::memcpy(stddevs, h.data() + nrows, nrows * sizeof(double));
        std::memcpy(deg_energy, h.data() + 2 * nrows, nrows * sizeof(double));
        *mean = h[3 * nrows];
    });
}

}  // extern "C"
