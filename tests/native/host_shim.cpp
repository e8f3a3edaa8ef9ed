// Test-only C wrappers over the product's host model
// (akvisqol_b200/csrc/host_model.cpp), so the CPU test suite can compare
// its planning and filter design with the oracle without a GPU.
#include <cstring>
#include <string>

#include "../../akvisqol_b200/csrc/host_model.h"

using namespace vqb;

extern "C" {

void hs_filterbank(size_t nb, uint32_t sr, double low, double high, double *coeffs, double *cf, double *run) {
    host::Filterbank fb = host::make_filterbank(nb, sr, low, high);
    std::memcpy(coeffs, fb.coeffs.data(), 8 * nb * sizeof(double));
    std::memcpy(cf, fb.cf.data(), nb * sizeof(double));
    std::memcpy(run, fb.run.data(), nb * sizeof(BandCoeffs));
}

void hs_hann(size_t size, double *out) {
    auto w = host::hann(size);
    std::memcpy(out, w.data(), size * sizeof(double));
}

void hs_twiddles(size_t n, double *out) {
    auto t = host::twiddles(n);
    std::memcpy(out, t.data(), t.size() * sizeof(double2));
}

double hs_zig_pow(double x, double y) { return host::zig_pow(x, y); }

void hs_geometry(uint32_t sr, size_t *window, size_t *hop, double *fd) {
    auto g = host::analysis_geometry(sr);
    *window = g.window, *hop = g.hop, *fd = g.frame_duration;
}

int hs_ref_patch_indices(size_t nf, size_t patch, int64_t *out, size_t *count) {
    try {
        auto v = host::ref_patch_indices(nf, patch);
        std::memcpy(out, v.data(), v.size() * sizeof(int64_t));
        *count = v.size();
        return 0;
    } catch (const Error &e) {
        *count = 0;
        return e.code;
    }
}

void hs_vad(const double *ref, size_t len, size_t nf, size_t patch, size_t window, double overlap, int64_t *out,
            size_t *count) {
    auto v = host::vad_patch_indices(ref, len, nf, patch, window, overlap);
    std::memcpy(out, v.data(), v.size() * sizeof(int64_t));
    *count = v.size();
}

int hs_plan_search(const int64_t *idx, size_t n, size_t nfr, size_t nfd, size_t patch, int32_t radius, int64_t *lo,
                   int64_t *hi, size_t *np) {
    try {
        auto s = host::plan_search(std::vector<int64_t>(idx, idx + n), nfr, nfd, patch, radius);
        std::memcpy(lo, s.lo.data(), s.np * sizeof(int64_t));
        std::memcpy(hi, s.hi.data(), s.np * sizeof(int64_t));
        *np = s.np;
        return 0;
    } catch (const Error &e) {
        *np = 0;
        return e.code;
    }
}

void hs_slice_layout(size_t len, uint32_t sr, double t0, double t1, int64_t *pad, int64_t *base, int64_t *n) {
    auto l = host::slice_layout(len, sr, t0, t1);
    *pad = l.pad, *base = l.base, *n = l.len;
}

void hs_trim_geometry(int64_t rl, int64_t dl, int64_t lag, uint32_t sr, int64_t *len, int64_t *ro, int64_t *dof,
                      double *ls) {
    auto t = host::trim_geometry(rl, dl, lag, sr);
    *len = t.len, *ro = t.ref_off, *dof = t.deg_off, *ls = t.lag_seconds;
}

int64_t hs_reuse_frame(int64_t pad, int64_t base, int64_t len, int64_t off, size_t hop, size_t nf_local,
                       size_t nf_global) {
    return host::reuse_frame(host::Slice{pad, base, len}, off, hop, nf_local, nf_global);
}

double hs_spl_factor(double er, size_t rl, double ed, size_t dl) { return host::spl_factor(er, rl, ed, dl); }

int hs_svr_predict(const char *text, size_t len, const double *x, double *y) {
    try {
        auto m = host::parse_svr(text ? std::string(text, len) : host::default_svr_text());
        *y = m.predict(x);
        return 0;
    } catch (const Error &e) {
        return e.code;
    }
}

int64_t hs_decode_wav(const char *bytes, size_t n, double *out, size_t cap, uint32_t *rate) {
    try {
        auto v = host::decode_wav(std::string(bytes, n), rate);
        if (v.size() <= cap) std::memcpy(out, v.data(), v.size() * sizeof(double));
        return (int64_t)v.size();
    } catch (const Error &e) {
        return e.code;
    }
}

// out holds n + 1 entries; returns the number of bounds written.
size_t hs_chunk_bounds(const size_t *sizes, size_t n, size_t chunks, size_t lanes, size_t front, size_t *out) {
    const auto b = host::chunk_bounds(std::vector<size_t>(sizes, sizes + n), chunks, lanes, front);
    std::memcpy(out, b.data(), b.size() * sizeof(size_t));
    return b.size();
}

}  // extern "C"
