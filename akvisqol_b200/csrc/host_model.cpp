// Host-side parts of the model (see host_model.h). Compiled with
// -ffp-contract=off: every expression rounds as the reference's Zig code.
#include "host_model.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>

#ifndef VQB_MODEL_PATH
#error "VQB_MODEL_PATH must name the bundled libsvm_nu_svr_model.txt"
#endif
#define VQB_STR2(x) #x
#define VQB_STR(x) VQB_STR2(x)
// The bundled SVR model, embedded at build time.
__asm__(".section .rodata\n"
        ".balign 16\n"
        "vqb_svr_model_begin:\n"
        ".incbin \"" VQB_STR(VQB_MODEL_PATH) "\"\n"
        "vqb_svr_model_finish:\n"
        ".byte 0\n"
        ".previous\n");
extern "C" const char vqb_svr_model_begin[];
extern "C" const char vqb_svr_model_finish[];

namespace vqb {
namespace host {

namespace {
constexpr double kPi = 3.14159265358979323846;
constexpr double kInf = std::numeric_limits<double>::infinity();
}  // namespace

double zig_pow(double x, double y) {
    if (y == 0.0 || x == 1.0) return 1.0;
    if (std::isnan(x) || std::isnan(y)) return std::nan("");
    if (y == 1.0) return x;
    if (x == 0.0 || std::isinf(x) || std::isinf(y)) return std::pow(x, y);  // edge cases; unused by the model
    if (y == 0.5) return std::sqrt(x);
    if (y == -0.5) return 1.0 / std::sqrt(x);
    double ipart;
    double frac = std::modf(std::fabs(y), &ipart);
    if (frac != 0.0 && x < 0.0) return std::nan("");
    if (ipart >= 9223372036854775808.0) return std::pow(x, y);
    double a = 1.0;
    int64_t exp2 = 0;
    if (frac != 0.0) {
        if (frac > 0.5) {
            frac -= 1.0;
            ipart += 1.0;
        }
        a = std::exp(frac * std::log(x));
    }
    int e = 0;
    double m = std::frexp(x, &e);
    int64_t me = e;
    for (int64_t bits = (int64_t)ipart; bits != 0; bits >>= 1) {
        if (me < -4096 || 4096 < me) {
            exp2 += me;
            break;
        }
        if (bits & 1) {
            a *= m;
            exp2 += me;
        }
        m *= m;
        me <<= 1;
        if (m < 0.5) {
            m += m;
            me -= 1;
        }
    }
    if (y < 0.0) {
        a = 1.0 / a;
        exp2 = -exp2;
    }
    exp2 = std::max<int64_t>(-100000, std::min<int64_t>(100000, exp2));
    return std::scalbn(a, (int)exp2);
}

namespace {

// ERB constants (reference src/dsp/erb.zig:8-10).
constexpr double kEarQ = 9.26449;
constexpr double kMinBw = 24.7;

struct C {
    double re, im;
};
inline C add(C a, C b) { return {a.re + b.re, a.im + b.im}; }
inline C sub(C a, C b) { return {a.re - b.re, a.im - b.im}; }
inline C mul(C a, C b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
inline C scale(C a, double s) { return {a.re * s, a.im * s}; }
inline C divide(C a, C b) {
    const double d = b.re * b.re + b.im * b.im;
    return {(a.re * b.re + a.im * b.im) / d, (a.im * b.re - a.re * b.im) / d};
}
inline C cexp(C z) {
    const double e = std::exp(z.re);
    return {e * std::cos(z.im), e * std::sin(z.im)};
}

// computeBand (reference src/gammatone.zig:76-153): coefficients of one
// 4th-order gammatone as four biquads sharing a denominator, gain from the
// complex transfer function at the centre frequency.
void design_band(double cf, double t, double pi, double *out) {
    const double erb = cf / kEarQ + kMinBw;
    const double big_b = 1.019 * 2.0 * pi * erb;
    const double exp_bt = std::exp(big_b * t);
    const double inv = 1.0 / exp_bt;
    const double exp_m2bt = std::exp(-2.0 * big_b * t);
    const double omega = 2.0 * cf * pi * t;
    const double cw = std::cos(omega), sw = std::sin(omega);
    const double p15 = zig_pow(2.0, 1.5);
    const double sp = std::sqrt(3.0 + p15), sm = std::sqrt(3.0 - p15);
    const double sin_t = sw * t;
    const double bpos = sin_t * 2.0 * sp, bneg = sin_t * 2.0 * sm;
    const double aterm = cw * 2.0 * t;
    out[0] = t;
    out[1] = -(aterm * inv + bpos * inv) / 2.0;
    out[2] = -(aterm * inv - bpos * inv) / 2.0;
    out[3] = -(aterm * inv + bneg * inv) / 2.0;
    out[4] = -(aterm * inv - bneg * inv) / 2.0;
    out[5] = -2.0 * cw * inv;
    out[6] = exp_m2bt;
    // gain = |x1 x2 x3 x4 / x5^4|
    const C xexp = cexp(scale(C{0.0, 1.0}, 4.0 * cf * pi * t));
    const C x01 = scale(xexp, -2.0 * t);
    const C x02 = scale(cexp(C{-big_b * t, 2.0 * cf * pi * t}), 2.0 * t);
    const C xc{cw, 0.0}, xs{sw, 0.0};
    const double s1 = std::sqrt(3.0 - p15), s2 = std::sqrt(3.0 + p15);
    const C x1 = add(x01, mul(x02, sub(xc, scale(xs, s1))));
    const C x2 = add(x01, mul(x02, add(xc, scale(xs, s1))));
    const C x3 = add(x01, mul(x02, sub(xc, scale(xs, s2))));
    const C x4 = add(x01, mul(x02, add(xc, scale(xs, s2))));
    const C t1 = divide(C{-2.0, 0.0}, C{std::exp(2.0 * big_b * t), 0.0});
    const C t2 = scale(xexp, -2.0);
    const C t3 = scale(divide(add(C{1.0, 0.0}, xexp), C{exp_bt, 0.0}), 2.0);
    const C x5 = add(add(t1, t2), t3);
    const C x5p4 = mul(mul(x5, x5), mul(x5, x5));
    const C r = divide(mul(mul(x1, x2), mul(x3, x4)), x5p4);
    out[7] = std::sqrt(r.re * r.re + r.im * r.im);
}

}  // namespace

BandCoeffs band_coeffs(const double *c) {
    const double gi = 1.0 / c[7];
    return BandCoeffs{c[0] * gi, c[1] * gi, c[2], c[3], c[4], c[0], c[5], c[6]};
}

Filterbank make_filterbank(size_t nb, uint32_t sample_rate, double low, double high_in) {
    const double fs = (double)sample_rate;
    const double high = std::min(high_in, fs / 2.0);
    // uniformCenterFreqs, descending (reference src/dsp/erb.zig:30-52).
    const double q = kEarQ, m = kMinBw;
    const double a = -(q * m);
    const double b = -std::log(high + q * m);
    const double c = std::log(low + q * m);
    const double d = high + q * m;
    const double e = (b + c) / (double)nb;
    std::vector<double> desc(nb);
    for (size_t i = 0; i < nb; ++i) desc[i] = a + std::exp(((double)i + 1.0) * e) * d;
    Filterbank fb;
    fb.nb = nb;
    fb.coeffs.resize(8 * nb);
    fb.cf.resize(nb);
    fb.run.resize(nb);
    const double t = 1.0 / fs;
    for (size_t i = 0; i < nb; ++i) {
        const double cf = desc[nb - 1 - i];
        fb.cf[i] = cf;
        design_band(cf, t, kPi, &fb.coeffs[8 * i]);
        fb.run[i] = band_coeffs(&fb.coeffs[8 * i]);
    }
    return fb;
}

std::vector<double> hann(size_t size) {
    std::vector<double> w(size);
    const double denom = std::max(1.0, (double)size - 1.0);
    for (size_t i = 0; i < size; ++i) w[i] = 0.5 - 0.5 * std::cos(2.0 * kPi * (double)i / denom);
    return w;
}

std::vector<double2> twiddles(size_t n) {
    std::vector<double2> top(n / 2);
    const double two_pi = 2.0 * kPi;
    const double nf = (double)n;
    for (size_t k = 0; k < n / 2; ++k) {
        const double angle = -two_pi * (double)k / nf;
        top[k] = double2{std::cos(angle), std::sin(angle)};
    }
    return top;
}

size_t num_frames(size_t len, size_t window, size_t hop) { return len < window ? 0 : 1 + (len - window) / hop; }

size_t fft_size_for(size_t biggest) {
    const size_t need = biggest == 0 ? 1 : 2 * biggest - 1;
    size_t n = 1;
    while (n < need) n <<= 1;
    return n;
}

Geometry analysis_geometry(uint32_t sample_rate) {
    const double fs = (double)sample_rate;
    Geometry g;
    g.window = (size_t)std::round(fs * 0.08);
    g.hop = (size_t)((double)g.window * 0.25);
    if (g.hop == 0) g.hop = 1;
    g.frame_duration = (double)g.hop / fs;
    return g;
}

std::vector<int64_t> ref_patch_indices(size_t nf, size_t patch) {
    const size_t first = patch / 2;
    if (nf < patch + first) throw Error(kSignal, "ReferenceSpectrogramTooSmall");
    const size_t stop = first < nf - patch ? nf - patch : first + 1;
    std::vector<int64_t> idx;
    for (size_t i = first; i < stop; i += patch) idx.push_back((int64_t)i - 1);
    return idx;
}

std::vector<int64_t> vad_patch_indices(const double *ref, size_t len, size_t nf, size_t patch, size_t window,
                                       double overlap) {
    const double frame_size = (double)window * overlap;
    const size_t frame_len = (size_t)frame_size;
    const size_t patch_len = (size_t)((double)patch * frame_size);
    const size_t first = patch / 2 - 1;
    std::vector<int64_t> out;
    if (nf <= first || frame_len == 0) return out;
    const size_t patches = (nf - first) / patch;
    const size_t chunks = patches * patch_len / frame_len;
    double peak = -kInf;
    for (size_t i = 0; i < len; ++i) peak = std::fmax(peak, ref[i]);
    // RMS of int16-scaled chunks, starting at *sample* `first` (upstream quirk).
    std::vector<char> loud(chunks);
    for (size_t c = 0; c < chunks; ++c) {
        double sq = 0.0;
        for (size_t j = 0; j < frame_len; ++j) {
            const size_t k = first + c * frame_len + j;
            const double x = k < len ? ref[k] / peak : 0.0;
            const double s = std::trunc(std::min(std::max(x * 32768.0, -32768.0), 32767.0));
            sq += s * s;
        }
        loud[c] = std::sqrt(sq / (double)frame_len) >= 5000.0;
    }
    // A chunk is silent only when it and the two before it are quiet; the
    // first two always count as active.
    std::vector<double> vad(std::max<size_t>(chunks, 2), 0.0);
    vad[0] = vad[1] = 1.0;
    for (size_t i = 2; i < chunks; ++i) vad[i] = (!loud[i] && !loud[i - 1] && !loud[i - 2]) ? 0.0 : 1.0;
    size_t start = first;
    for (size_t p = 0; p < patches; ++p, start += patch) {
        double act = 0.0;
        for (size_t k = p * patch; k < p * patch + patch; ++k)
            if (k < vad.size()) act += vad[k];
        if (act >= 1.0) out.push_back((int64_t)start);
    }
    return out;
}

size_t max_num_patches(const std::vector<int64_t> &idx, size_t nf_deg, size_t patch) {
    size_t n = idx.size();
    const size_t half = patch / 2;
    while (n > 0) {
        const size_t last = (size_t)idx[n - 1];
        if (last < half || last - half <= nf_deg) break;
        --n;
    }
    return n;
}

Search plan_search(const std::vector<int64_t> &idx, size_t nf_ref, size_t nf_deg, size_t patch, int32_t radius) {
    Search s;
    s.np = max_num_patches(idx, nf_deg, patch);
    if (s.np == 0 || nf_deg == 0) throw Error(kSignal, "SignalsTooDifferent");
    for (size_t i = 0; i < s.np; ++i)
        if ((size_t)idx[i] + patch > nf_ref) throw Error(kSignal, "SignalsTooDifferent");
    const int64_t reach = (int64_t)radius * (int64_t)patch;
    const int64_t last = (int64_t)nf_deg - 1;
    s.lo.resize(s.np);
    s.hi.resize(s.np);
    for (size_t i = 0; i < s.np; ++i) {
        const int64_t lo = std::max<int64_t>(0, idx[i] - reach);
        s.lo[i] = lo;
        s.hi[i] = std::max(lo, std::min(idx[i] + reach, last));
    }
    return s;
}

Slice slice_layout(size_t signal_len, uint32_t sample_rate, double t0, double t1) {
    const double fs = (double)sample_rate;
    const int64_t n = (int64_t)signal_len;
    const int64_t first = std::max<int64_t>(0, (int64_t)(t0 * fs));
    const int64_t last = std::min<int64_t>(n - 1, (int64_t)(t1 * fs));
    const int64_t len = last > first ? last - first : 0;
    const double over = t1 * fs - (double)signal_len;
    const int64_t post = over > 0.0 ? (int64_t)over : 0;
    const int64_t pre = t0 < 0.0 ? (int64_t)(-t0 * fs) : 0;
    return Slice{pre + post, len > 0 ? first : 0, len};
}

Trim trim_geometry(int64_t ref_len, int64_t deg_len, int64_t lag, uint32_t sample_rate) {
    const int64_t mag = lag < 0 ? -lag : lag;
    const int64_t shift = (lag == 0 || mag > ref_len / 2) ? 0 : lag;
    const int64_t dl = shift < 0 ? deg_len - std::min(-shift, deg_len) : deg_len + shift;
    const double fs = (double)sample_rate;
    int64_t head = 0, len = ref_len;
    if (ref_len > dl) {
        len = dl;
    } else if (ref_len < dl && shift > 0) {
        // lag -> seconds -> samples truncates (27 becomes 26 at 48 kHz).
        const double secs = (double)shift / fs;
        head = std::max<int64_t>((int64_t)(secs * fs), 0);
        len = ref_len - head;
    }
    return Trim{len, head, head - shift, shift == 0 ? 0.0 : (double)shift / fs};
}

int64_t reuse_frame(const Slice &l, int64_t off, size_t hop, size_t nf_local, size_t nf_global) {
    if (off < l.pad) return -1;
    const int64_t start = l.base + off - l.pad;
    if (start % (int64_t)hop != 0) return -1;
    const int64_t g0 = start / (int64_t)hop;
    if ((size_t)g0 + nf_local > nf_global) return -1;
    return g0;
}

Aligned apply_lag_geometry(size_t ref_len, size_t deg_len, int64_t lag, uint32_t sample_rate) {
    const int64_t mag = lag < 0 ? -lag : lag;
    Aligned a{0, 0, (int64_t)deg_len, 0.0};
    if (lag == 0 || mag > (int64_t)(ref_len / 2)) return a;
    a.lag_seconds = (double)lag / (double)sample_rate;
    if (lag < 0) {
        a.skip = std::min<int64_t>(-lag, (int64_t)deg_len);
        a.len = (int64_t)deg_len - a.skip;
    } else {
        a.lead = lag;
        a.len = (int64_t)deg_len + lag;
    }
    return a;
}

double spl_of_energy(double energy, size_t len) {
    if (len == 0) return -kInf;
    const double rms = std::sqrt(energy / (double)len);
    return 20.0 * std::log10(rms / 0.00002);
}

double spl_factor(double ref_energy, size_t ref_len, double deg_energy, size_t deg_len) {
    const double r = spl_of_energy(ref_energy, ref_len), d = spl_of_energy(deg_energy, deg_len);
    if (!std::isfinite(r) || !std::isfinite(d)) return 1.0;
    return zig_pow(10.0, (r - d) / 20.0);
}

double Svr::predict(const double *x) const {
    double acc = 0.0;
    for (size_t i = 0; i < coeff.size(); ++i) {
        double dist = 0.0;
        for (size_t f = 0; f < nf; ++f) {
            const double d = sv[i * nf + f] - x[f];
            dist += d * d;
        }
        acc += coeff[i] * std::exp(-gamma * dist);
    }
    return acc - rho;
}

namespace {
std::vector<std::string> split_ws(const std::string &s) {
    std::vector<std::string> out;
    size_t i = 0;
    while (i < s.size()) {
        while (i < s.size() && (s[i] == ' ' || s[i] == '\t')) ++i;
        size_t j = i;
        while (j < s.size() && s[j] != ' ' && s[j] != '\t') ++j;
        if (j > i) out.push_back(s.substr(i, j - i));
        i = j;
    }
    return out;
}
bool parse_double(const std::string &s, double *v) {
    if (s.empty()) return false;
    char *end = nullptr;
    *v = std::strtod(s.c_str(), &end);
    return end && *end == 0;
}
bool parse_index(const std::string &s, size_t *v) {
    if (s.empty()) return false;
    char *end = nullptr;
    const unsigned long long x = std::strtoull(s.c_str(), &end, 10);
    if (!end || *end != 0 || s[0] == '-' || s[0] == '+') return false;
    *v = (size_t)x;
    return true;
}
}  // namespace

// parseModel (reference src/svr.zig:80-165): header keys, then one line per
// support vector ("coef idx:val ..."); features are 1-indexed, zero-filled.
Svr parse_svr(const std::string &text) {
    Svr m;
    bool in_sv = false;
    std::vector<std::string> rows;
    size_t max_feat = 0;
    size_t pos = 0;
    while (pos < text.size()) {
        size_t nl = text.find('\n', pos);
        if (nl == std::string::npos) nl = text.size();
        std::string line = text.substr(pos, nl - pos);
        pos = nl + 1;
        if (!line.empty() && line.back() == '\r') line.pop_back();
        if (line.empty()) continue;
        if (!in_sv) {
            if (line == "SV") {
                in_sv = true;
                continue;
            }
            const size_t sp = line.find(' ');
            if (sp == std::string::npos) continue;
            const std::string key = line.substr(0, sp);
            std::string val = line.substr(sp + 1);
            val.erase(0, val.find_first_not_of(" \t"));
            val.erase(val.find_last_not_of(" \t") + 1);
            if (key == "svm_type" && val != "nu_svr" && val != "epsilon_svr")
                throw Error(kModel, "UnsupportedSvmType");
            if (key == "kernel_type" && val != "rbf") throw Error(kModel, "UnsupportedKernel");
            if (key == "gamma" && !parse_double(val, &m.gamma)) throw Error(kModel, "InvalidModelFile");
            if (key == "rho" && !parse_double(val, &m.rho)) throw Error(kModel, "InvalidModelFile");
            continue;
        }
        rows.push_back(line);
        const auto toks = split_ws(line);
        for (size_t t = 1; t < toks.size(); ++t) {
            const size_t colon = toks[t].find(':');
            size_t idx;
            if (colon != std::string::npos && parse_index(toks[t].substr(0, colon), &idx)) max_feat = std::max(max_feat, idx);
        }
    }
    if (rows.empty()) throw Error(kModel, "NoSupportVectors");
    if (max_feat == 0) throw Error(kModel, "InvalidModelFile");
    m.nf = max_feat;
    m.sv.assign(rows.size() * max_feat, 0.0);
    m.coeff.resize(rows.size());
    for (size_t r = 0; r < rows.size(); ++r) {
        const auto toks = split_ws(rows[r]);
        if (toks.empty() || !parse_double(toks[0], &m.coeff[r])) throw Error(kModel, "InvalidModelFile");
        for (size_t t = 1; t < toks.size(); ++t) {
            const size_t colon = toks[t].find(':');
            if (colon == std::string::npos) continue;
            size_t idx;
            double v;
            if (!parse_index(toks[t].substr(0, colon), &idx)) continue;
            if (!parse_double(toks[t].substr(colon + 1), &v)) continue;
            if (idx == 0 || idx > max_feat) throw Error(kModel, "InvalidFeatureIndex");
            m.sv[r * max_feat + idx - 1] = v;
        }
    }
    return m;
}

const std::string &default_svr_text() {
    static const std::string text(vqb_svr_model_begin, vqb_svr_model_finish - vqb_svr_model_begin);
    return text;
}

Scores build_scores(std::vector<Match> matches, size_t nb, double frame_duration, const Svr *svr, bool speech,
                    bool unscaled_speech, const std::vector<double> &cf, double lag_s,
                    const LatticeMapper *lattice) {
    Scores s;
    const size_t n = matches.size();
    const double nf = (double)n;
    s.fvnsim.assign(nb, 0.0);
    s.fvdegenergy.assign(nb, 0.0);
    s.fvnsim10.assign(nb, 0.0);
    s.fstdnsim.assign(nb, 0.0);
    for (const Match &m : matches)
        for (size_t b = 0; b < nb; ++b) {
            s.fvnsim[b] += m.means[b];
            s.fvdegenergy[b] += m.energy[b];
        }
    for (size_t b = 0; b < nb; ++b) {
        s.fvnsim[b] /= nf;
        s.fvdegenergy[b] /= nf;
    }
    // Mean of the lowest 10% (at least one) per band.
    const size_t k = std::max<size_t>(1, (size_t)std::trunc(nf * 0.10));
    std::vector<double> col(n);
    for (size_t b = 0; b < nb; ++b) {
        for (size_t i = 0; i < n; ++i) col[i] = matches[i].means[b];
        std::sort(col.begin(), col.end());
        double acc = 0.0;
        for (size_t i = 0; i < k; ++i) acc += col[i];
        s.fvnsim10[b] = acc / (double)k;
    }
    // Pooled standard deviation over patches weighted by their frames.
    std::vector<double> contrib(nb, 0.0);
    int64_t frames = 0;
    for (const Match &m : matches) {
        const int64_t fc_i = (int64_t)std::ceil((m.ref_end - m.ref_start) / frame_duration);
        frames += fc_i;
        const double fc = (double)fc_i;
        for (size_t b = 0; b < nb; ++b) {
            contrib[b] += (fc - 1.0) * m.stddevs[b] * m.stddevs[b];
            contrib[b] += fc * m.means[b] * m.means[b];
        }
    }
    const double total = (double)frames;
    for (size_t b = 0; b < nb; ++b) {
        const double v = (contrib[b] - s.fvnsim[b] * s.fvnsim[b] * total) / (total - 1.0);
        s.fstdnsim[b] = v < 0.0 ? 0.0 : std::sqrt(v);
    }
    double sum = 0.0;
    for (double x : s.fvnsim) sum += x;
    s.vnsim = sum / (double)nb;
    double mos;
    if (!speech) {
        mos = std::min(std::max(svr->predict(s.fvnsim.data()), 1.0), 5.0);
    } else if (lattice) {
        // widened without clamping, as the reference (src/lattice.zig:4-6)
        mos = lattice->predict(s.fvnsim.data(), s.fvnsim10.data(), s.fstdnsim.data(), s.fvdegenergy.data());
    } else {
        // Exponential fit over mean NSIM (reference src/visqol.zig:85-96).
        double acc = 0.0;
        for (double x : s.fvnsim) acc += x;
        const double mean = acc / (double)s.fvnsim.size();
        const double raw = -262.847869 + std::exp(0.0154302525 * (mean - -361.063949));
        const double gain = unscaled_speech ? 1.0 : (double)1.245063f;
        mos = std::min(std::max(raw * gain, 1.0), 5.0);
    }
    if (s.vnsim < 0.15) mos = 1.0;
    s.moslqo = mos;
    s.lag_s = lag_s;
    s.cf = cf;
    s.patches = std::move(matches);
    return s;
}

std::string read_file(const std::string &path) {
    FILE *f = std::fopen(path.c_str(), "rb");
    if (!f) throw Error(kIo, path + ": FileNotFound");
    std::string s;
    char buf[1 << 16];
    size_t k;
    while ((k = std::fread(buf, 1, sizeof buf, f)) > 0) s.append(buf, k);
    std::fclose(f);
    return s;
}

namespace {
uint32_t rd_u32(const unsigned char *p) { return (uint32_t)p[0] | (uint32_t)p[1] << 8 | (uint32_t)p[2] << 16 | (uint32_t)p[3] << 24; }
uint16_t rd_u16(const unsigned char *p) { return (uint16_t)(p[0] | p[1] << 8); }
}  // namespace

std::vector<double> decode_wav(const std::string &bytes, uint32_t *sample_rate) {
    const auto *d = reinterpret_cast<const unsigned char *>(bytes.data());
    const size_t n = bytes.size();
    if (n < 12 || std::memcmp(d, "RIFF", 4) != 0 || std::memcmp(d + 8, "WAVE", 4) != 0) throw Error(kIo, "NotRiffWave");
    uint16_t tag = 0, channels = 0, bits = 0;
    uint32_t rate = 0;
    bool fmt = false;
    const unsigned char *pcm = nullptr;
    size_t pcm_len = 0;
    size_t off = 12;
    while (off + 8 <= n) {
        const uint32_t size = rd_u32(d + off + 4);
        const size_t body = off + 8;
        const size_t end = std::min<size_t>(n, body + (size_t)size);
        if (std::memcmp(d + off, "fmt ", 4) == 0) {
            if (end - body < 16) throw Error(kIo, "UnsupportedFormat");
            tag = rd_u16(d + body);
            channels = rd_u16(d + body + 2);
            rate = rd_u32(d + body + 4);
            bits = rd_u16(d + body + 14);
            if (tag == 0xFFFE && end - body >= 26) tag = rd_u16(d + body + 24);
            fmt = true;
        } else if (std::memcmp(d + off, "data", 4) == 0) {
            pcm = d + body;
            pcm_len = end - body;
            break;
        }
        off = body + (size_t)size + (size & 1);
    }
    if (!fmt) throw Error(kIo, "MissingFmtChunk");
    if (!pcm) throw Error(kIo, "MissingDataChunk");
    if (channels == 0) throw Error(kSignal, "ChannelCountZero");
    const bool ok = (tag == 1 && (bits == 8 || bits == 16 || bits == 24 || bits == 32)) ||
                    (tag == 3 && (bits == 32 || bits == 64));
    if (!ok) throw Error(kIo, "UnsupportedFormat");
    const size_t bps = bits / 8;
    const size_t frames = pcm_len / (bps * channels);
    if (frames == 0) throw Error(kSignal, "EmptyAudio");
    std::vector<double> out(frames);
    for (size_t f = 0; f < frames; ++f) {
        double sum = 0.0;
        for (size_t ch = 0; ch < channels; ++ch) {
            const unsigned char *p = pcm + (f * channels + ch) * bps;
            double v;
            if (tag == 3) {
                if (bits == 32) {
                    float x;
                    std::memcpy(&x, p, 4);
                    v = x;
                } else {
                    std::memcpy(&v, p, 8);
                }
            } else if (bits == 8) {
                v = ((double)p[0] - 128.0) / 128.0;
            } else if (bits == 16) {
                v = (double)(int16_t)rd_u16(p) / 32768.0;
            } else if (bits == 24) {
                int32_t x = (int32_t)((uint32_t)p[0] | (uint32_t)p[1] << 8 | (uint32_t)p[2] << 16);
                if (x & 0x800000) x -= 0x1000000;
                v = (double)x / 8388608.0;
            } else {
                v = (double)(int32_t)rd_u32(p) / 2147483648.0;
            }
            sum += v;
        }
        out[f] = channels == 1 ? sum : sum / (double)channels;
    }
    *sample_rate = rate;
    return out;
}

std::vector<size_t> chunk_bounds(const std::vector<size_t> &sizes, size_t chunks, size_t lanes, size_t front) {
    const size_t n = sizes.size();
    std::vector<size_t> bounds{0};
    if (n == 0) return bounds;
    const size_t K = std::max<size_t>(1, std::min(n, chunks));
    size_t total = 0;
    for (size_t s : sizes) total += s;
    std::vector<size_t> target;  // cumulative size at each chunk's end
    if (front > 0 && front < 100 && K > lanes) {
        const double avg = (double)total / (double)K, small = avg * (double)front / 100.0;
        const double rest = ((double)total - small * (double)lanes) / (double)(K - lanes);
        double at = 0.0;
        for (size_t k = 0; k < K; ++k) target.push_back((size_t)(at += k < lanes ? small : rest));
    } else {
        for (size_t k = 0; k < K; ++k) target.push_back((size_t)((double)total * (double)(k + 1) / (double)K));
    }
    size_t acc = 0;
    for (size_t i = 0; i + 1 < n && bounds.size() < K; ++i) {
        acc += sizes[i];
        if (acc >= target[bounds.size() - 1]) bounds.push_back(i + 1);
    }
    bounds.push_back(n);
    return bounds;
}

}  // namespace host
}  // namespace vqb
