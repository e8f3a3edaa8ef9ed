// CPU oracle for the ViSQOL hot path (test infrastructure only).
//
// A plain C++17 restatement of the reference CPU model, jdek/akvisqol
// src/visqol.zig `Pipeline(NB).runBatch` and the stages it calls, in f64,
// compiled with -ffp-contract=off so that every product and sum rounds as
// the reference's Zig code does (Zig never contracts a*b+c). Host
// transcendentals are glibc's, as the reference links libc on Linux
// (build.zig:88); `pow` restates Zig's std.math.pow algorithm (the Go
// math.Pow method: exp/log for the fractional part, repeated squaring of
// the frexp mantissa for the integral part) over glibc exp/log.
//
// The product library never links or calls this file. Tests, the smoke
// check and bench.py's CPU-baseline leg use it as the checker.

#include "visqol_oracle.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <memory>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

// The default SVR model, embedded from the data file at build time.
#ifndef VQO_MODEL_PATH
#error "VQO_MODEL_PATH must name libsvm_nu_svr_model.txt"
#endif
#define VQO_STR2(x) #x
#define VQO_STR(x) VQO_STR2(x)
__asm__(".section .rodata\n"
        ".balign 16\n"
        "vqo_svr_model_start:\n"
        ".incbin \"" VQO_STR(VQO_MODEL_PATH) "\"\n"
        "vqo_svr_model_end:\n"
        ".byte 0\n"
        ".previous\n");
extern "C" const char vqo_svr_model_start[];
extern "C" const char vqo_svr_model_end[];

namespace {

constexpr double kPi = 3.14159265358979323846;
constexpr double kInf = std::numeric_limits<double>::infinity();

// Error codes as the C ABI classifies them (src/capi.zig:96-112).
constexpr int E_INVALID = -1;
constexpr int E_MODEL = -4;
constexpr int E_SIGNAL = -5;

struct VqError : std::runtime_error {
    int code;
    VqError(int c, const char *m) : std::runtime_error(m), code(c) {}
};

thread_local std::string g_last_error;

// ---------------------------------------------------------------------
// Zig std.math.pow (Go math.Pow method), f64. Reference call sites:
// src/audio.zig:148,156, src/gammatone.zig:91-92,116-117.
// ---------------------------------------------------------------------
double zig_pow(double x, double y) {
    if (y == 0.0 || x == 1.0) return 1.0;
    if (std::isnan(x) || std::isnan(y)) return std::nan("");
    if (y == 1.0) return x;
    if (x == 0.0) {
        if (y < 0.0) {
            double yi;
            bool odd = std::modf(y, &yi) == 0.0 && std::fmod(std::fabs(y), 2.0) == 1.0;
            if (odd && std::signbit(x)) return -kInf;
            return kInf;
        }
        if (y > 0.0) {
            bool odd = std::fmod(std::fabs(y), 2.0) == 1.0;
            if (odd) return x;
            return 0.0;
        }
    }
    if (std::isinf(y)) {
        if (x == -1.0) return 1.0;
        if ((std::fabs(x) < 1.0) == (y > 0.0)) return 0.0;
        return kInf;
    }
    if (std::isinf(x)) {
        if (x < 0.0) return zig_pow(1.0 / x, -y);
        if (y < 0.0) return 0.0;
        return kInf;
    }
    if (y == 0.5) return std::sqrt(x);
    if (y == -0.5) return 1.0 / std::sqrt(x);

    double yi;
    double yf = std::modf(std::fabs(y), &yi);
    if (yf != 0.0 && x < 0.0) return std::nan("");
    if (yi >= 9223372036854775808.0) {
        if (x == -1.0) return 1.0;
        if ((std::fabs(x) < 1.0) == (y > 0.0)) return 0.0;
        return kInf;
    }
    double a1 = 1.0;
    int64_t ae = 0;
    if (yf != 0.0) {
        if (yf > 0.5) {
            yf -= 1.0;
            yi += 1.0;
        }
        a1 = std::exp(yf * std::log(x));
    }
    int xe_i = 0;
    double x1 = std::frexp(x, &xe_i);
    int64_t xe = xe_i;
    for (int64_t i = (int64_t)yi; i != 0; i >>= 1) {
        const int64_t overflow_shift = 11 + 1;
        if (xe < -(int64_t(1) << overflow_shift) || (int64_t(1) << overflow_shift) < xe) {
            ae += xe;
            break;
        }
        if (i & 1) {
            a1 *= x1;
            ae += xe;
        }
        x1 *= x1;
        xe <<= 1;
        if (x1 < 0.5) {
            x1 += x1;
            xe -= 1;
        }
    }
    if (y < 0.0) {
        a1 = 1.0 / a1;
        ae = -ae;
    }
    if (ae > 100000) ae = 100000;
    if (ae < -100000) ae = -100000;
    return std::scalbn(a1, (int)ae);
}

// ---------------------------------------------------------------------
// ERB and gammatone coefficients (src/dsp/erb.zig, src/gammatone.zig).
// ---------------------------------------------------------------------
constexpr double EAR_Q = 9.26449;
constexpr double MIN_BW = 24.7;

// erbGeneralized at order 1 (src/dsp/erb.zig:20-27).
inline double erb_generalized(double f) { return f / EAR_Q + MIN_BW; }

// uniformCenterFreqs, descending (src/dsp/erb.zig:30-52).
void uniform_center_freqs(size_t n, double low, double high, double *out) {
    const double q = EAR_Q, m = MIN_BW;
    const double a = -(q * m);
    const double b = -std::log(high + q * m);
    const double c = std::log(low + q * m);
    const double d = high + q * m;
    const double e = (b + c) / (double)n;
    for (size_t i = 0; i < n; ++i) {
        const double idx = (double)i + 1.0;
        const double f = std::exp(idx * e) * d;
        out[i] = a + f;
    }
}

struct Cx {
    double re, im;
};
inline Cx cadd(Cx a, Cx b) { return {a.re + b.re, a.im + b.im}; }
inline Cx csub(Cx a, Cx b) { return {a.re - b.re, a.im - b.im}; }
inline Cx cmul(Cx a, Cx b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
inline Cx cmuls(Cx a, double s) { return {a.re * s, a.im * s}; }
inline Cx cdiv(Cx a, Cx b) {
    const double denom = b.re * b.re + b.im * b.im;
    return {(a.re * b.re + a.im * b.im) / denom, (a.im * b.re - a.re * b.im) / denom};
}
inline Cx cexp_(Cx z) {
    const double e = std::exp(z.re);
    return {e * std::cos(z.im), e * std::sin(z.im)};
}

struct Band {
    double a0, a11, a12, a13, a14, b1, b2, gain;
};

// computeBand (src/gammatone.zig:76-153).
Band compute_band(double cf, double t, double pi) {
    const double erb = erb_generalized(cf);
    const double big_b = 1.019 * 2.0 * pi * erb;
    const double exp_bt = std::exp(big_b * t);
    const double inv_exp_bt = 1.0 / exp_bt;
    const double exp_neg_2bt = std::exp(-2.0 * big_b * t);

    const double omega = 2.0 * cf * pi * t;
    const double cos_w = std::cos(omega);
    const double sin_w = std::sin(omega);

    const double b1_re = -2.0 * cos_w * inv_exp_bt;
    const double b2_re = exp_neg_2bt;

    const double sin_t = sin_w * t;
    const double sqrt_3p_p1 = std::sqrt(3.0 + zig_pow(2.0, 1.5));
    const double sqrt_3m_p1 = std::sqrt(3.0 - zig_pow(2.0, 1.5));
    const double b_pos = sin_t * 2.0 * sqrt_3p_p1;
    const double b_neg = sin_t * 2.0 * sqrt_3m_p1;
    const double a_term = cos_w * 2.0 * t;

    const double a11_re = -(a_term * inv_exp_bt + b_pos * inv_exp_bt) / 2.0;
    const double a12_re = -(a_term * inv_exp_bt - b_pos * inv_exp_bt) / 2.0;
    const double a13_re = -(a_term * inv_exp_bt + b_neg * inv_exp_bt) / 2.0;
    const double a14_re = -(a_term * inv_exp_bt - b_neg * inv_exp_bt) / 2.0;

    const Cx i_unit{0.0, 1.0};
    const Cx four_i_cf_pi_t = cmuls(i_unit, 4.0 * cf * pi * t);
    const Cx x_exp = cexp_(four_i_cf_pi_t);
    const Cx x01 = cmuls(x_exp, -2.0 * t);
    const Cx inner{-big_b * t, 2.0 * cf * pi * t};
    const Cx x02 = cmuls(cexp_(inner), 2.0 * t);
    const Cx xcos{cos_w, 0.0};
    const Cx xsin{sin_w, 0.0};
    const double s1 = std::sqrt(3.0 - zig_pow(2.0, 1.5));
    const double s2 = std::sqrt(3.0 + zig_pow(2.0, 1.5));
    const Cx x12 = csub(xcos, cmuls(xsin, s1));
    const Cx x22 = cadd(xcos, cmuls(xsin, s1));
    const Cx x32 = csub(xcos, cmuls(xsin, s2));
    const Cx x42 = cadd(xcos, cmuls(xsin, s2));
    const Cx x1 = cadd(x01, cmul(x02, x12));
    const Cx x2 = cadd(x01, cmul(x02, x22));
    const Cx x3 = cadd(x01, cmul(x02, x32));
    const Cx x4 = cadd(x01, cmul(x02, x42));

    const Cx exp_2bt{std::exp(2.0 * big_b * t), 0.0};
    const Cx exp_bt_c{exp_bt, 0.0};
    const Cx term1 = cdiv(Cx{-2.0, 0.0}, exp_2bt);
    const Cx term2 = cmuls(x_exp, -2.0);
    const Cx one_p_xexp = cadd(Cx{1.0, 0.0}, x_exp);
    const Cx term3 = cmuls(cdiv(one_p_xexp, exp_bt_c), 2.0);
    const Cx x5 = cadd(cadd(term1, term2), term3);

    const Cx x5_p4 = cmul(cmul(x5, x5), cmul(x5, x5));
    const Cx num = cmul(cmul(x1, x2), cmul(x3, x4));
    const Cx ratio = cdiv(num, x5_p4);
    const double gain = std::sqrt(ratio.re * ratio.re + ratio.im * ratio.im);
    return {t, a11_re, a12_re, a13_re, a14_re, b1_re, b2_re, gain};
}

struct Filters {
    std::vector<Band> bands;     // ascending
    std::vector<double> cf;      // ascending
};

// Filters.init (src/gammatone.zig:41-70).
Filters make_filters(size_t nb, uint32_t sample_rate, double low, double high_in) {
    const double sr_f = (double)sample_rate;
    const double high = std::min(high_in, sr_f / 2.0);
    std::vector<double> cf_desc(nb);
    uniform_center_freqs(nb, low, high, cf_desc.data());
    const double t = 1.0 / sr_f;
    const double pi = kPi;
    Filters f;
    f.bands.resize(nb);
    f.cf.resize(nb);
    for (size_t i = 0; i < nb; ++i) {
        f.bands[i] = compute_band(cf_desc[nb - 1 - i], t, pi);
        f.cf[i] = cf_desc[nb - 1 - i];
    }
    return f;
}

// hannWindow (src/gammatone.zig:309-316).
void hann_window(size_t size, double *out) {
    const double denom = std::max(1.0, (double)size - 1.0);
    for (size_t i = 0; i < size; ++i) out[i] = 0.5 - 0.5 * std::cos(2.0 * kPi * (double)i / denom);
}

// numFrames (src/gammatone.zig:320-323).
inline size_t num_frames(size_t len, size_t window, size_t hop) {
    if (len < window) return 0;
    return 1 + (len - window) / hop;
}

// filterBandRmsFresh (src/gammatone.zig:268-306).
double filter_band_rms_fresh(const Band &band, const double *x, size_t n) {
    const double gi = 1.0 / band.gain;
    const double s1n0 = band.a0 * gi, s1n1 = band.a11 * gi;
    const double s2n1 = band.a12, s3n1 = band.a13, s4n1 = band.a14;
    const double ca0 = band.a0, d1 = band.b1, d2 = band.b2;
    double s1c0 = 0, s1c1 = 0, s2c0 = 0, s2c1 = 0, s3c0 = 0, s3c1 = 0, s4c0 = 0, s4c1 = 0;
    double sum_sq = 0;
    for (size_t i = 0; i < n; ++i) {
        const double s = x[i];
        const double f1 = s1n0 * s + s1c0;
        s1c0 = s1n1 * s + s1c1 - d1 * f1;
        s1c1 = -(d2 * f1);
        const double f2 = ca0 * f1 + s2c0;
        s2c0 = s2n1 * f1 + s2c1 - d1 * f2;
        s2c1 = -(d2 * f2);
        const double f3 = ca0 * f2 + s3c0;
        s3c0 = s3n1 * f2 + s3c1 - d1 * f3;
        s3c1 = -(d2 * f3);
        const double f4 = ca0 * f3 + s4c0;
        s4c0 = s4n1 * f3 + s4c1 - d1 * f4;
        s4c1 = -(d2 * f4);
        sum_sq += f4 * f4;
    }
    const double inv_n = 1.0 / (double)n;
    return std::sqrt(sum_sq * inv_n);
}

// Frames run side by side in lanes, each lane the scalar recurrence above
// (src/gammatone.zig:336-408). Lane-wise IEEE ops, so bit-identical.
constexpr size_t LANES = 8;

void rms_fresh_lanes(const Band &band, const double *w /* window*LANES */, size_t window, double *rms) {
    const double gi = 1.0 / band.gain;
    const double s1n0 = band.a0 * gi, s1n1 = band.a11 * gi;
    const double s2n1 = band.a12, s3n1 = band.a13, s4n1 = band.a14;
    const double ca0 = band.a0, d1 = band.b1, d2 = band.b2;
    double s1c0[LANES] = {}, s1c1[LANES] = {}, s2c0[LANES] = {}, s2c1[LANES] = {};
    double s3c0[LANES] = {}, s3c1[LANES] = {}, s4c0[LANES] = {}, s4c1[LANES] = {};
    double sum[LANES] = {};
    for (size_t i = 0; i < window; ++i) {
        const double *s = w + i * LANES;
#pragma GCC ivdep
        for (size_t l = 0; l < LANES; ++l) {
            const double f1 = s1n0 * s[l] + s1c0[l];
            s1c0[l] = s1n1 * s[l] + s1c1[l] - d1 * f1;
            s1c1[l] = -(d2 * f1);
            const double f2 = ca0 * f1 + s2c0[l];
            s2c0[l] = s2n1 * f1 + s2c1[l] - d1 * f2;
            s2c1[l] = -(d2 * f2);
            const double f3 = ca0 * f2 + s3c0[l];
            s3c0[l] = s3n1 * f2 + s3c1[l] - d1 * f3;
            s3c1[l] = -(d2 * f3);
            const double f4 = ca0 * f3 + s4c0[l];
            s4c0[l] = s4n1 * f3 + s4c1[l] - d1 * f4;
            s4c1[l] = -(d2 * f4);
            sum[l] += f4 * f4;
        }
    }
    const double inv_n = 1.0 / (double)window;
    for (size_t l = 0; l < LANES; ++l) rms[l] = std::sqrt(sum[l] * inv_n);
}

// buildSpectrogramBands (src/gammatone.zig:432-467): out[b*nf + f].
size_t build_spectrogram(const std::vector<Band> &bands, const double *signal, size_t len, size_t window,
                         size_t hop, const double *hann, double *out) {
    const size_t nf = num_frames(len, window, hop);
    std::vector<double> w(window * LANES);
    double rms[LANES];
    for (size_t f = 0; f < nf; f += LANES) {
        const size_t lanes = std::min(LANES, nf - f);
        for (size_t i = 0; i < window; ++i)
            for (size_t l = 0; l < LANES; ++l)
                w[i * LANES + l] = l < lanes ? signal[(f + l) * hop + i] * hann[i] : 0.0;
        for (size_t b = 0; b < bands.size(); ++b) {
            rms_fresh_lanes(bands[b], w.data(), window, rms);
            for (size_t l = 0; l < lanes; ++l) out[b * nf + f + l] = rms[l];
        }
    }
    return nf;
}

// ---------------------------------------------------------------------
// Envelope, FFT and lag search (src/envelope.zig, src/dsp/fft.zig,
// src/xcorr.zig).
// ---------------------------------------------------------------------
size_t next_pow_two(size_t x) {
    if (x <= 1) return 1;
    size_t n = 1;
    while (n < x) n <<= 1;
    return n;
}

// upperEnvelope (src/envelope.zig:23-53).
void upper_envelope(const double *signal, size_t l, double *out) {
    if (l == 0) return;
    double sum = 0.0;
    for (size_t i = 0; i < l; ++i) sum += signal[i];
    const double mean = sum / (double)l;
    const size_t n = std::max(next_pow_two(l), (size_t)32);
    double nyquist = 0.0, sign = 1.0;
    for (size_t i = 0; i < l; ++i) {
        nyquist += sign * (signal[i] - mean);
        sign = -sign;
    }
    const double nyquist_over_n = nyquist / (double)n;
    const double eps = 0.000001;
    bool pos_sign = true;
    for (size_t idx = 0; idx < l; ++idx) {
        const double pad_centered = signal[idx] - mean;
        const double nyq_term = pos_sign ? nyquist_over_n : -nyquist_over_n;
        const double re = 2.0 * (pad_centered - nyq_term) - eps;
        out[idx] = std::fabs(re) + mean;
        pos_sign = !pos_sign;
    }
}

// fftSizeFor (src/xcorr.zig:64-69).
size_t fft_size_for(size_t biggest) {
    const size_t needed = biggest == 0 ? 1 : 2 * biggest - 1;
    size_t n = 1;
    while (n < needed) n <<= 1;
    return std::max(n, (size_t)1);
}

// Plan twiddles (src/dsp/fft.zig:55-66): W_S^j = top[j * n/S], where
// top[k] = exp(-2πik/n) computed as cos/sin of (-2π·k)/n.
struct FftPlan {
    size_t n = 0;
    std::vector<Cx> top;  // n/2 entries
    void init(size_t n_) {
        n = n_;
        top.resize(n / 2);
        const double two_pi = 2.0 * kPi;
        const double n_f = (double)n;
        for (size_t k = 0; k < n / 2; ++k) {
            const double angle = -two_pi * (double)k / n_f;
            top[k] = {std::cos(angle), std::sin(angle)};
        }
    }
    inline Cx tw(size_t span, size_t j) const { return top[j * (n / span)]; }
};

inline Cx cmul_tw(Cx x, Cx w) { return {x.re * w.re - x.im * w.im, x.re * w.im + x.im * w.re}; }
inline Cx cmul_conj(Cx x, Cx w) {
    const double wi = -w.im;
    return {x.re * w.re - x.im * wi, x.re * wi + x.im * w.re};
}

// One radix-2 DIF stage at span `size` over buf[base, base+len).
void dif_stage(const FftPlan &p, Cx *buf, size_t base, size_t len, size_t size) {
    const size_t h = size / 2, stride = p.n / size;
    for (size_t k = base; k < base + len; k += size)
        for (size_t j = 0; j < h; ++j) {
            const Cx a = buf[k + j], b = buf[k + j + h];
            buf[k + j] = cadd(a, b);
            buf[k + j + h] = cmul_tw(csub(a, b), p.top[j * stride]);
        }
}
void dit_stage(const FftPlan &p, Cx *buf, size_t base, size_t len, size_t size) {
    const size_t h = size / 2, stride = p.n / size;
    for (size_t k = base; k < base + len; k += size)
        for (size_t j = 0; j < h; ++j) {
            const Cx a = buf[k + j];
            const Cx b = cmul_conj(buf[k + j + h], p.top[j * stride]);
            buf[k + j] = cadd(a, b);
            buf[k + j + h] = csub(a, b);
        }
}

// Radix-4 fused DIF pass: spans S and S/2 applied as two radix-2 stages.
void dif_pass4(const FftPlan &p, Cx *buf, size_t len, size_t size) {
    const size_t q = size / 4, s1 = p.n / size, s2 = p.n / (size / 2);
    for (size_t k = 0; k < len; k += size)
        for (size_t j = 0; j < q; ++j) {
            Cx x0 = buf[k + j], x1 = buf[k + j + q], x2 = buf[k + j + 2 * q], x3 = buf[k + j + 3 * q];
            // span `size`: t pairs (0,2) and (1,3), twiddle index j + t*q
            Cx a = x0, b = x2;
            x0 = cadd(a, b);
            x2 = cmul_tw(csub(a, b), p.top[j * s1]);
            a = x1, b = x3;
            x1 = cadd(a, b);
            x3 = cmul_tw(csub(a, b), p.top[(j + q) * s1]);
            // span size/2: pairs (0,1) and (2,3), twiddle index j
            a = x0, b = x1;
            x0 = cadd(a, b);
            x1 = cmul_tw(csub(a, b), p.top[j * s2]);
            a = x2, b = x3;
            x2 = cadd(a, b);
            x3 = cmul_tw(csub(a, b), p.top[j * s2]);
            buf[k + j] = x0, buf[k + j + q] = x1, buf[k + j + 2 * q] = x2, buf[k + j + 3 * q] = x3;
        }
}
// Radix-4 fused DIT pass: spans S/2 then S.
void dit_pass4(const FftPlan &p, Cx *buf, size_t len, size_t size) {
    const size_t q = size / 4, s1 = p.n / size, s2 = p.n / (size / 2);
    for (size_t k = 0; k < len; k += size)
        for (size_t j = 0; j < q; ++j) {
            Cx x0 = buf[k + j], x1 = buf[k + j + q], x2 = buf[k + j + 2 * q], x3 = buf[k + j + 3 * q];
            Cx a = x0, b = cmul_conj(x1, p.top[j * s2]);
            x0 = cadd(a, b);
            x1 = csub(a, b);
            a = x2, b = cmul_conj(x3, p.top[j * s2]);
            x2 = cadd(a, b);
            x3 = csub(a, b);
            a = x0, b = cmul_conj(x2, p.top[j * s1]);
            x0 = cadd(a, b);
            x2 = csub(a, b);
            a = x1, b = cmul_conj(x3, p.top[(j + q) * s1]);
            x1 = cadd(a, b);
            x3 = csub(a, b);
            buf[k + j] = x0, buf[k + j + q] = x1, buf[k + j + 2 * q] = x2, buf[k + j + 3 * q] = x3;
        }
}

constexpr size_t CACHE_BLOCK = 4096;

// difForward: natural in, bit-reversed out, unscaled (src/dsp/fft.zig:127-145).
// Every schedule of the same radix-2 butterflies gives identical bits.
void dif_forward(const FftPlan &p, Cx *buf) {
    const size_t n = p.n;
    const size_t block = std::min(n, CACHE_BLOCK);
    size_t size = n;
    while (size > block) {
        if (size / 2 > block) {
            dif_pass4(p, buf, n, size);
            size >>= 2;
        } else {
            dif_stage(p, buf, 0, n, size);
            size >>= 1;
        }
    }
    for (size_t base = 0; base < n; base += block)
        for (size_t s = block; s > 1; s >>= 1) dif_stage(p, buf, base, block, s);
}

// ditInverse: bit-reversed in, natural out, unscaled (src/dsp/fft.zig:148-166).
void dit_inverse(const FftPlan &p, Cx *buf) {
    const size_t n = p.n;
    const size_t block = std::min(n, CACHE_BLOCK);
    for (size_t base = 0; base < n; base += block)
        for (size_t s = 2; s <= block; s <<= 1) dit_stage(p, buf, base, block, s);
    size_t done = block;
    while (done < n) {
        if (done * 4 <= n) {
            done <<= 2;
            dit_pass4(p, buf, n, done);
        } else {
            done <<= 1;
            dit_stage(p, buf, 0, n, done);
        }
    }
}

// crossTerm (src/xcorr.zig:182-192).
inline Cx cross_term(Cx x, Cx zy) {
    const Cx y{zy.re, -zy.im};
    const Cx sum{x.re + y.re, x.im + y.im};
    const Cx dif_c{x.re - y.re, -(x.im - y.im)};
    const Cx idc{-dif_c.im, dif_c.re};
    return {0.25 * (sum.re * idc.re - sum.im * idc.im), 0.25 * (sum.re * idc.im + sum.im * idc.re)};
}

struct Work {
    uint64_t n_rms = 0;
    uint64_t n_cells = 0;
    double fft_nlogn = 0;
};

// bestLagCached (src/xcorr.zig:197-251).
int64_t best_lag(const double *s1, size_t l1, const double *s2, size_t l2, Work *work) {
    const size_t biggest = std::max(l1, l2);
    if (biggest == 0) return 0;
    const size_t n = fft_size_for(biggest);
    FftPlan plan;
    plan.init(n);
    std::vector<Cx> z(n, Cx{0.0, 0.0});
    for (size_t i = 0; i < biggest; ++i) z[i] = {i < l1 ? s1[i] : 0.0, i < l2 ? s2[i] : 0.0};
    dif_forward(plan, z.data());
    z[0] = cross_term(z[0], z[0]);
    if (n > 1) z[1] = cross_term(z[1], z[1]);
    for (size_t h = 2; h < n; h <<= 1) {
        size_t a = h, b = 2 * h - 1;
        while (a < b) {
            const Cx za = z[a], zb = z[b];
            z[a] = cross_term(za, zb);
            z[b] = cross_term(zb, za);
            ++a, --b;
        }
    }
    dit_inverse(plan, z.data());
    if (work) work->fft_nlogn += 2.0 * (double)n * std::log2((double)n);
    const size_t max_lag = biggest - 1;
    double best_abs = -kInf;
    int64_t best = 0;
    for (size_t i = n - max_lag; i < n; ++i) {
        const double a = std::fabs(z[i].re);
        if (a > best_abs) best_abs = a, best = (int64_t)i - (int64_t)n;
    }
    for (size_t k = 0; k <= max_lag; ++k) {
        const double a = std::fabs(z[k].re);
        if (a > best_abs) best_abs = a, best = (int64_t)k;
    }
    return best;
}

// alignmentEnvelopes + bestLagCached (src/realign.zig:81-88, src/accel.zig:100-107).
int64_t envelope_lag(const double *a, size_t la, const double *b, size_t lb, Work *work) {
    std::vector<double> ea(la), eb(lb);
    upper_envelope(a, la, ea.data());
    upper_envelope(b, lb, eb.data());
    return best_lag(ea.data(), la, eb.data(), lb, work);
}

// ---------------------------------------------------------------------
// SPL (src/audio.zig:132-158).
// ---------------------------------------------------------------------
constexpr double SPL_REFERENCE_POINT = 0.00002;

double spl_of_energy(double energy, size_t len) {
    if (len == 0) return -kInf;
    const double rms = std::sqrt(energy / (double)len);
    return 20.0 * std::log10(rms / SPL_REFERENCE_POINT);
}
double sound_pressure_level(const double *x, size_t n) {
    double energy = 0.0;
    for (size_t i = 0; i < n; ++i) energy += x[i] * x[i];
    return spl_of_energy(energy, n);
}
// scaleToMatchSpl; returns the factor applied (1 when left as is).
double scale_to_match_spl(const double *ref, size_t rn, double *deg, size_t dn) {
    const double ref_spl = sound_pressure_level(ref, rn);
    const double deg_spl = sound_pressure_level(deg, dn);
    if (!std::isfinite(ref_spl) || !std::isfinite(deg_spl)) return 1.0;
    const double factor = zig_pow(10.0, (ref_spl - deg_spl) / 20.0);
    for (size_t i = 0; i < dn; ++i) deg[i] *= factor;
    return factor;
}

// ---------------------------------------------------------------------
// Spectrogram prep (src/spectrogram.zig:14-80).
// ---------------------------------------------------------------------
constexpr double NOISE_FLOOR_RELATIVE_TO_PEAK_DB = 45.0;
constexpr double NOISE_FLOOR_ABSOLUTE_DB = -45.0;

void convert_to_db(double *data, size_t n, double floor_db) {
    for (size_t i = 0; i < n; ++i) {
        const double sample = data[i] == 0.0 ? std::numeric_limits<double>::epsilon() : std::fabs(data[i]);
        const double db = 10.0 * std::log10(sample);
        data[i] = std::fmax(db, floor_db);  // Zig @max: IEEE maxNum
    }
}
void raise_floor_per_frame(double *ref, double *deg, size_t nb, size_t nfr, size_t nfd, double rel) {
    const size_t min_frames = std::min(nfr, nfd);
    for (size_t c = 0; c < min_frames; ++c) {
        double col_max = -kInf;
        for (size_t r = 0; r < nb; ++r) {
            const double m = std::fmax(ref[r * nfr + c], deg[r * nfd + c]);
            if (m > col_max) col_max = m;
        }
        const double floor_db = col_max - rel;
        for (size_t r = 0; r < nb; ++r) {
            double &rv = ref[r * nfr + c];
            if (rv < floor_db) rv = floor_db;
            double &dv = deg[r * nfd + c];
            if (dv < floor_db) dv = floor_db;
        }
    }
}
void subtract_joint_minimum(double *ref, size_t rn, double *deg, size_t dn) {
    double lo = kInf;
    for (size_t i = 0; i < rn; ++i)
        if (ref[i] < lo) lo = ref[i];
    for (size_t i = 0; i < dn; ++i)
        if (deg[i] < lo) lo = deg[i];
    for (size_t i = 0; i < rn; ++i) ref[i] -= lo;
    for (size_t i = 0; i < dn; ++i) deg[i] -= lo;
}
void prepare_for_comparison(double *ref, double *deg, size_t nb, size_t nfr, size_t nfd) {
    convert_to_db(ref, nb * nfr, NOISE_FLOOR_ABSOLUTE_DB);
    convert_to_db(deg, nb * nfd, NOISE_FLOOR_ABSOLUTE_DB);
    raise_floor_per_frame(ref, deg, nb, nfr, nfd, NOISE_FLOOR_RELATIVE_TO_PEAK_DB);
    subtract_joint_minimum(ref, nb * nfr, deg, nb * nfd);
}

// ---------------------------------------------------------------------
// NSIM (src/nsim.zig).
// ---------------------------------------------------------------------
constexpr double WINDOW[3][3] = {
    {0.0113033910173052, 0.0838251475442633, 0.0113033910173052},
    {0.0838251475442633, 0.619485845753726, 0.0838251475442633},
    {0.0113033910173052, 0.0838251475442633, 0.0113033910173052},
};

// Flipped taps and their fixed summation order (src/nsim.zig:119-155).
struct Taps {
    double w00, w01, w02, w10, w11, w12, w20, w21, w22;
    Taps()
        : w00(WINDOW[2][2]), w01(WINDOW[2][1]), w02(WINDOW[2][0]), w10(WINDOW[1][2]), w11(WINDOW[1][1]),
          w12(WINDOW[1][0]), w20(WINDOW[0][2]), w21(WINDOW[0][1]), w22(WINDOW[0][0]) {}
    inline double at(const double *in, size_t rm, size_t r0, size_t rp, size_t cm, size_t c, size_t cp) const {
        return w00 * in[rm + cm] + w01 * in[rm + c] + w02 * in[rm + cp] + w10 * in[r0 + cm] + w11 * in[r0 + c] +
               w12 * in[r0 + cp] + w20 * in[rp + cm] + w21 * in[rp + c] + w22 * in[rp + cp];
    }
    // Taps.row (src/nsim.zig:182-192).
    void row(const double *in, size_t rm, size_t r0, size_t rp, size_t ncols, double *out) const {
        if (ncols == 1) {
            out[0] = at(in, rm, r0, rp, 0, 0, 0);
            return;
        }
        out[0] = at(in, rm, r0, rp, 0, 0, 1);
        for (size_t c = 1; c + 1 < ncols; ++c) out[c] = at(in, rm, r0, rp, c - 1, c, c + 1);
        out[ncols - 1] = at(in, rm, r0, rp, ncols - 2, ncols - 1, ncols - 1);
    }
};
const Taps kTaps;

inline size_t row_above(size_t r) { return r == 0 ? 0 : r - 1; }
inline size_t row_below(size_t r, size_t nrows) { return r + 1 >= nrows ? nrows - 1 : r + 1; }

// conv2d3x3Replicate (src/nsim.zig:204-218).
void conv2d3x3(const double *in, double *out, size_t nrows, size_t ncols) {
    for (size_t r = 0; r < nrows; ++r) {
        const size_t r0 = r * ncols;
        kTaps.row(in, row_above(r) * ncols, r0, row_below(r, nrows) * ncols, ncols, out + r0);
    }
}

const double C1 = (0.01 * 1.0) * (0.01 * 1.0);
const double C3 = (0.03 * 1.0) * (0.03 * 1.0) / 2.0;

// simCell (src/nsim.zig:293-308).
inline double sim_cell(double mr, double rms, double srs, double md, double dms, double sds, double crd) {
    const double mrd = mr * md;
    const double srd = crd - mrd;
    const double intensity = (2.0 * mrd + C1) / (rms + dms + C1);
    const double prod = srs * sds;
    const double structure_denom = prod < 0.0 ? C3 : std::sqrt(prod) + C3;
    const double structure = (srd + C3) / structure_denom;
    return intensity * structure;
}

// DegPlane (src/nsim.zig:224-263).
struct DegPlane {
    size_t nrows, width;
    std::vector<double> pad, sq, mu, dms, sds;
    DegPlane(const double *spec, size_t nrows_, size_t nf, size_t width_) : nrows(nrows_), width(width_) {
        const size_t n = nrows * width;
        pad.assign(n, 0.0);
        sq.resize(n), mu.resize(n), dms.resize(n), sds.resize(n);
        for (size_t r = 0; r < nrows; ++r) std::memcpy(&pad[r * width], spec + r * nf, nf * sizeof(double));
        for (size_t i = 0; i < n; ++i) sq[i] = pad[i] * pad[i];
        conv2d3x3(pad.data(), mu.data(), nrows, width);
        conv2d3x3(sq.data(), sds.data(), nrows, width);
        for (size_t i = 0; i < n; ++i) {
            dms[i] = mu[i] * mu[i];
            sds[i] = sds[i] - dms[i];
        }
    }
};

// Scratch + Comparator (src/nsim.zig:46-108, 310-510).
struct Scratch {
    size_t nrows, ncols;
    std::vector<double> mu_ref, mu_deg, ref_sq, deg_sq, ref_deg, conv_ref_sq, conv_deg_sq, conv_rd, srs, rms;
    std::vector<double> row_crd, row_sim;
    Scratch(size_t nr, size_t nc) : nrows(nr), ncols(nc) {
        const size_t n = nr * nc;
        for (auto *v : {&mu_ref, &mu_deg, &ref_sq, &deg_sq, &ref_deg, &conv_ref_sq, &conv_deg_sq, &conv_rd, &srs, &rms})
            v->assign(n, 0.0);
        row_crd.assign(nc, 0.0);
        row_sim.assign(nc, 0.0);
    }
    // precomputeRef (src/nsim.zig:318-329).
    void precompute_ref(const double *ref) {
        const size_t n = nrows * ncols;
        conv2d3x3(ref, mu_ref.data(), nrows, ncols);
        for (size_t i = 0; i < n; ++i) ref_sq[i] = ref[i] * ref[i];
        conv2d3x3(ref_sq.data(), conv_ref_sq.data(), nrows, ncols);
        for (size_t i = 0; i < n; ++i) {
            rms[i] = mu_ref[i] * mu_ref[i];
            srs[i] = conv_ref_sq[i] - rms[i];
        }
    }
    // measureSimilarityAt (src/nsim.zig:364-424).
    double similarity_at(const double *ref, const DegPlane &plane, size_t off) {
        const size_t nr = nrows, nc = ncols, w = plane.width;
        for (size_t r = 0; r < nr; ++r)
            for (size_t c = 0; c < nc; ++c) ref_deg[r * nc + c] = ref[r * nc + c] * plane.pad[r * w + off + c];
        double sum = 0.0;
        for (size_t r = 0; r < nr; ++r) {
            const size_t rm = row_above(r), rp = row_below(r, nr);
            kTaps.row(ref_deg.data(), rm * nc, r * nc, rp * nc, nc, row_crd.data());
            const size_t pr = r * w + off, ri = r * nc;
            const size_t edges[2] = {0, nc - 1};
            const size_t ne = std::min(nc, (size_t)2);
            for (size_t e = 0; e < ne; ++e) {
                const size_t c = edges[e];
                const size_t cm = off + (c == 0 ? 0 : c - 1);
                const size_t cp = off + (c + 1 >= nc ? nc - 1 : c + 1);
                const double md = kTaps.at(plane.pad.data(), rm * w, r * w, rp * w, cm, off + c, cp);
                const double cdsq = kTaps.at(plane.sq.data(), rm * w, r * w, rp * w, cm, off + c, cp);
                const double dms = md * md;
                row_sim[c] = sim_cell(mu_ref[ri + c], rms[ri + c], srs[ri + c], md, dms, cdsq - dms, row_crd[c]);
            }
            for (size_t c = 1; c + 1 < nc; ++c)
                row_sim[c] = sim_cell(mu_ref[ri + c], rms[ri + c], srs[ri + c], plane.mu[pr + c], plane.dms[pr + c],
                                      plane.sds[pr + c], row_crd[c]);
            for (size_t c = 0; c < nc; ++c) sum += row_sim[c];
        }
        return sum / (double)(nr * nc);
    }
    // measureSimilarityScalar (src/nsim.zig:332-360), without a cached ref.
    double similarity_scalar(const double *ref, const double *deg) {
        const size_t n = nrows * ncols;
        precompute_ref(ref);
        conv2d3x3(deg, mu_deg.data(), nrows, ncols);
        for (size_t i = 0; i < n; ++i) deg_sq[i] = deg[i] * deg[i];
        for (size_t i = 0; i < n; ++i) ref_deg[i] = ref[i] * deg[i];
        conv2d3x3(deg_sq.data(), conv_deg_sq.data(), nrows, ncols);
        conv2d3x3(ref_deg.data(), conv_rd.data(), nrows, ncols);
        double sum = 0.0;
        for (size_t i = 0; i < n; ++i) {
            const double mr = mu_ref[i], md = mu_deg[i], dms = md * md;
            sum += sim_cell(mr, mr * mr, srs[i], md, dms, conv_deg_sq[i] - dms, conv_rd[i]);
        }
        return sum / (double)n;
    }
    // measurePatchSimilarity (src/nsim.zig:427-510).
    double patch_similarity(const double *ref, const double *deg, double *means, double *stddevs, double *energy) {
        const size_t n = nrows * ncols;
        conv2d3x3(ref, mu_ref.data(), nrows, ncols);
        conv2d3x3(deg, mu_deg.data(), nrows, ncols);
        for (size_t i = 0; i < n; ++i) ref_sq[i] = ref[i] * ref[i];
        for (size_t i = 0; i < n; ++i) deg_sq[i] = deg[i] * deg[i];
        for (size_t i = 0; i < n; ++i) ref_deg[i] = ref[i] * deg[i];
        conv2d3x3(ref_sq.data(), conv_ref_sq.data(), nrows, ncols);
        conv2d3x3(deg_sq.data(), conv_deg_sq.data(), nrows, ncols);
        conv2d3x3(ref_deg.data(), conv_rd.data(), nrows, ncols);
        const double inv_ncols = 1.0 / (double)ncols;
        for (size_t r = 0; r < nrows; ++r) {
            double deg_sum = 0.0;
            for (size_t c = 0; c < ncols; ++c) deg_sum += deg[r * ncols + c];
            energy[r] = deg_sum * inv_ncols;
        }
        for (size_t r = 0; r < nrows; ++r) {
            double sim_sum = 0.0;
            for (size_t c = 0; c < ncols; ++c) {
                const size_t idx = r * ncols + c;
                const double mr = mu_ref[idx], md = mu_deg[idx];
                const double rms_ = mr * mr, dms = md * md, mrd = mr * md;
                const double srs_ = conv_ref_sq[idx] - rms_;
                const double sds = conv_deg_sq[idx] - dms;
                const double srd = conv_rd[idx] - mrd;
                const double intensity = (2.0 * mrd + C1) / (rms_ + dms + C1);
                const double prod = srs_ * sds;
                const double structure_denom = prod < 0.0 ? C3 : std::sqrt(prod) + C3;
                const double structure = (srd + C3) / structure_denom;
                const double sim = intensity * structure;
                sim_sum += sim;
                conv_rd[idx] = sim;
            }
            means[r] = sim_sum * inv_ncols;
        }
        for (size_t r = 0; r < nrows; ++r) {
            if (ncols <= 1) {
                stddevs[r] = 0.0;
                continue;
            }
            const double mean = means[r];
            double ss = 0.0;
            for (size_t c = 0; c < ncols; ++c) {
                const double diff = conv_rd[r * ncols + c] - mean;
                ss += diff * diff;
            }
            stddevs[r] = std::sqrt(ss / ((double)ncols - 1.0));
        }
        double mean_acc = 0.0;
        for (size_t r = 0; r < nrows; ++r) mean_acc += means[r];
        return mean_acc / (double)nrows;
    }
};

// ---------------------------------------------------------------------
// Patches, search plan, DP (src/dp.zig) and VAD (src/vad.zig).
// ---------------------------------------------------------------------

// refPatchIndices (src/dp.zig:47-70).
std::vector<size_t> ref_patch_indices(size_t num_frames, size_t patch_size) {
    const size_t init = patch_size / 2;
    if (num_frames < patch_size + init) throw VqError(E_SIGNAL, "ReferenceSpectrogramTooSmall");
    const size_t max_index = init < num_frames - patch_size ? num_frames - patch_size : init + 1;
    std::vector<size_t> out;
    for (size_t i = init; i < max_index; i += patch_size) out.push_back(i - 1);
    return out;
}

// calcMaxNumPatches (src/dp.zig:73-87).
size_t calc_max_num_patches(const std::vector<size_t> &idx, size_t nf_deg, size_t per_patch) {
    size_t n = idx.size();
    while (n > 0) {
        const size_t last = idx[n - 1];
        if (last < per_patch / 2) break;
        if (last - per_patch / 2 <= nf_deg) break;
        n -= 1;
    }
    return n;
}

// vad.refPatchIndices (src/vad.zig:15-81).
std::vector<size_t> vad_patch_indices(const double *ref, size_t ref_len, size_t num_frames, size_t patch_size,
                                      size_t window_size, double overlap) {
    const double frame_size = (double)window_size * overlap;
    const size_t frame_len = (size_t)frame_size;
    const size_t patch_sample_len = (size_t)((double)patch_size * frame_size);
    const size_t first_patch_idx = patch_size / 2 - 1;
    if (num_frames <= first_patch_idx || frame_len == 0) return {};
    const size_t patch_count = (num_frames - first_patch_idx) / patch_size;
    const size_t total_samples = patch_count * patch_sample_len;
    double max_val = -kInf;
    for (size_t i = 0; i < ref_len; ++i) max_val = std::fmax(max_val, ref[i]);
    const size_t n_chunks = total_samples / frame_len;
    std::vector<uint8_t> active(n_chunks);
    for (size_t c = 0; c < n_chunks; ++c) {
        double square = 0.0;
        for (size_t j = 0; j < frame_len; ++j) {
            const size_t idx = first_patch_idx + c * frame_len + j;
            const double x = idx < ref_len ? ref[idx] / max_val : 0.0;
            const double scaled = std::min(std::max(x * 32768.0, -32768.0), 32767.0);
            const double s = std::trunc(scaled);
            square += s * s;
        }
        const double rms = std::sqrt(square / (double)frame_len);
        active[c] = rms >= 5000.0;
    }
    const size_t silent = 3;
    const size_t vad_len = std::max(n_chunks, silent - 1);
    std::vector<double> vad(vad_len, 0.0);
    for (size_t i = 0; i < silent - 1; ++i) vad[i] = 1.0;
    for (size_t i = silent - 1; i < n_chunks; ++i) {
        bool prev_silent = true;
        for (size_t j = 1; j < silent; ++j)
            if (active[i - j]) {
                prev_silent = false;
                break;
            }
        vad[i] = (!active[i] && prev_silent) ? 0.0 : 1.0;
    }
    std::vector<size_t> out;
    size_t patch_idx = first_patch_idx;
    for (size_t p = 0; p < patch_count; ++p) {
        double with_va = 0.0;
        const size_t lo = p * patch_size;
        for (size_t k = lo; k < lo + patch_size; ++k)
            if (k < vad.size()) with_va += vad[k];
        if (with_va >= 1.0) out.push_back(patch_idx);
        patch_idx += patch_size;
    }
    return out;
}

struct SearchPlan {
    size_t num_patches = 0;
    std::vector<size_t> lo, hi;
    std::vector<double> sims;  // [num_patches][nf_deg]
    size_t nf_deg = 0;
};

// searchPatches + searchWindow + planSearch (src/dp.zig:153-201).
SearchPlan plan_search(const std::vector<size_t> &idx, size_t nf_ref, size_t nf_deg, size_t patch_size, int32_t radius) {
    const size_t num = calc_max_num_patches(idx, nf_deg, patch_size);
    if (num == 0 || nf_deg == 0) throw VqError(E_SIGNAL, "SignalsTooDifferent");
    for (size_t i = 0; i < num; ++i)
        if (idx[i] + patch_size > nf_ref) throw VqError(E_SIGNAL, "SignalsTooDifferent");
    SearchPlan p;
    p.num_patches = num;
    p.nf_deg = nf_deg;
    p.lo.resize(num), p.hi.resize(num);
    p.sims.assign(num * nf_deg, 0.0);
    const int64_t sw = (int64_t)radius * (int64_t)patch_size;
    const int64_t last = (int64_t)nf_deg - 1;
    for (size_t i = 0; i < num; ++i) {
        const int64_t r = (int64_t)idx[i];
        const int64_t lo = std::max<int64_t>(0, r - sw);
        p.lo[i] = (size_t)lo;
        p.hi[i] = (size_t)std::max(lo, std::min(r + sw, last));
    }
    return p;
}

// accel.Cpu.patchSimilarities for one pair (src/accel.zig:126-146).
void patch_similarities(const double *ref_spec, size_t nf_ref, const double *deg_spec, size_t nf_deg, size_t nb,
                        size_t patch, const std::vector<size_t> &ref_idx, SearchPlan &plan, Work *work) {
    Scratch s(nb, patch);
    std::vector<double> ref_patch(nb * patch);
    size_t width = nf_deg;
    for (size_t p = 0; p < plan.num_patches; ++p) width = std::max(width, plan.hi[p] + patch);
    DegPlane plane(deg_spec, nb, nf_deg, width);
    for (size_t p = 0; p < plan.num_patches; ++p) {
        for (size_t b = 0; b < nb; ++b)
            for (size_t c = 0; c < patch; ++c) ref_patch[b * patch + c] = ref_spec[b * nf_ref + ref_idx[p] + c];
        s.precompute_ref(ref_patch.data());
        for (size_t off = plan.lo[p]; off <= plan.hi[p]; ++off)
            plan.sims[p * nf_deg + off] = s.similarity_at(ref_patch.data(), plane, off);
        if (work) work->n_cells += (plan.hi[p] - plan.lo[p] + 1) * nb * patch;
    }
}

struct Match {
    double similarity = 0, ref_start = 0, ref_end = 0, deg_start = 0, deg_end = 0;
    std::vector<double> means, stddevs, energy;
    bool valid = true;
    int64_t deg_offset = -1;
    int64_t realign_lag = 0;
    int64_t realign_frames = -1;
    uint8_t realign_reused = 0;
    bool realign_accepted = false;
};

// DP recurrence and backtrack (src/dp.zig:216-288, 313-352), the per-patch
// NSIM left to the caller: returns (offset, valid) per patch reached.
struct DpOut {
    std::vector<int64_t> offset;
    std::vector<uint8_t> valid;
    std::vector<uint8_t> reached;
};
DpOut dp_backtrack(const SearchPlan &plan) {
    const size_t np = plan.num_patches, cols = plan.nf_deg;
    const size_t NONE = std::numeric_limits<size_t>::max();
    std::vector<double> dp(np * cols, 0.0);
    std::vector<size_t> bt(np * cols, 0);
    for (size_t pi = 0; pi < np; ++pi) {
        const size_t start = plan.lo[pi], end = plan.hi[pi];
        size_t prev_row = 0, prev_lower = 0;
        if (pi > 0) prev_row = (pi - 1) * cols, prev_lower = plan.lo[pi - 1];
        double running_max = -kInf;
        int64_t running_idx = -1;
        if (pi > 0)
            for (size_t i = prev_lower; i < start; ++i) {
                const double val = dp[prev_row + i];
                if (val >= running_max) running_max = val, running_idx = (int64_t)i;
            }
        for (size_t slide = start; slide <= end; ++slide) {
            double similarity = plan.sims[pi * cols + slide];
            int64_t past = -1;
            if (pi > 0) {
                similarity += running_max;
                past = running_idx;
                const double no_move = dp[prev_row + slide];
                if (no_move > similarity) similarity = no_move, past = (int64_t)slide;
                if (no_move >= running_max) running_max = no_move, running_idx = (int64_t)slide;
            }
            dp[pi * cols + slide] = similarity;
            bt[pi * cols + slide] = past < 0 ? NONE : (size_t)past;
        }
    }
    const size_t last = np - 1;
    double max_score = -kInf;
    size_t last_offset = 0;
    for (size_t off = plan.lo[last]; off <= plan.hi[last]; ++off) {
        const double v = dp[last * cols + off];
        if (v > max_score) max_score = v, last_offset = off;
    }
    DpOut out;
    out.offset.assign(np, -1);
    out.valid.assign(np, 1);
    out.reached.assign(np, 0);
    int64_t p_idx = (int64_t)np - 1;
    size_t cur = last_offset;
    while (p_idx >= 0) {
        const size_t i = (size_t)p_idx;
        out.offset[i] = (int64_t)cur;
        out.reached[i] = 1;
        const size_t back = bt[i * cols + cur];
        out.valid[i] = back == cur ? 0 : 1;
        if (back == NONE) break;
        cur = back;
        p_idx -= 1;
    }
    return out;
}

// findOptimalDegPatchesFromSims (src/dp.zig:205-355).
std::vector<Match> find_optimal_deg_patches(const SearchPlan &plan, const double *ref_spec, const std::vector<size_t> &ref_idx,
                                            const double *deg_spec, size_t nb, size_t nf_ref, size_t patch,
                                            double frame_duration, Work *work) {
    const size_t np = plan.num_patches, nf_deg = plan.nf_deg;
    DpOut d = dp_backtrack(plan);
    std::vector<Match> items(np);
    for (auto &m : items) {
        m.means.assign(nb, 0.0);
        m.stddevs.assign(nb, 0.0);
        m.energy.assign(nb, 0.0);
    }
    Scratch s(nb, patch);
    std::vector<double> refp(nb * patch), degp(nb * patch);
    const double patch_duration = frame_duration * (double)patch;
    for (int64_t p = (int64_t)np - 1; p >= 0; --p) {
        const size_t i = (size_t)p;
        if (!d.reached[i]) break;
        const size_t cur = (size_t)d.offset[i];
        const size_t ref_i = ref_idx[i];
        // buildDegradedPatch / buildRefPatch (src/dp.zig:90-132).
        for (size_t b = 0; b < nb; ++b)
            for (size_t c = 0; c < patch; ++c) {
                degp[b * patch + c] = cur + c < nf_deg ? deg_spec[b * nf_deg + cur + c] : 0.0;
                refp[b * patch + c] = ref_spec[b * nf_ref + ref_i + c];
            }
        Match &m = items[i];
        m.similarity = s.patch_similarity(refp.data(), degp.data(), m.means.data(), m.stddevs.data(), m.energy.data());
        if (work) work->n_cells += nb * patch;
        m.deg_offset = (int64_t)cur;
        if (!d.valid[i]) {
            m.deg_start = 0.0;
            m.deg_end = 0.0;
            m.similarity = 0.0;
            std::fill(m.means.begin(), m.means.end(), 0.0);
            m.valid = false;
        } else {
            m.deg_start = (double)cur * frame_duration;
            m.deg_end = m.deg_start + patch_duration;
            m.valid = true;
        }
        m.ref_start = (double)ref_i * frame_duration;
        m.ref_end = m.ref_start + patch_duration;
    }
    return items;
}

// ---------------------------------------------------------------------
// Realignment (src/realign.zig).
// ---------------------------------------------------------------------
struct SliceLayout {
    size_t pad, base, len;
};

// sliceLayout (src/realign.zig:41-51).
SliceLayout slice_layout(size_t signal_len, uint32_t sample_rate, double start_time, double end_time) {
    const double sr_f = (double)sample_rate;
    const int64_t n = (int64_t)signal_len;
    const int64_t start_idx = std::max<int64_t>(0, (int64_t)(start_time * sr_f));
    const int64_t end_idx = std::min<int64_t>(n - 1, (int64_t)(end_time * sr_f));
    const size_t real_len = end_idx > start_idx ? (size_t)(end_idx - start_idx) : 0;
    const double end_diff = end_time * sr_f - (double)signal_len;
    const size_t post_pad = end_diff > 0.0 ? (size_t)end_diff : 0;
    const size_t pre_pad = start_time < 0.0 ? (size_t)(-start_time * sr_f) : 0;
    return {pre_pad + post_pad, real_len > 0 ? (size_t)start_idx : 0, real_len};
}

std::vector<double> slice_view(const double *signal, const SliceLayout &l) {
    std::vector<double> out(l.pad + l.len, 0.0);
    if (l.len) std::memcpy(out.data() + l.pad, signal + l.base, l.len * sizeof(double));
    return out;
}

struct Aligned {
    std::vector<double> deg;
    double lag_seconds = 0;
    int64_t lag_samples = 0;
};

// applyLag (src/realign.zig:91-110).
Aligned apply_lag(size_t ref_len, const double *deg, size_t deg_len, int64_t lag, uint32_t sample_rate) {
    const int64_t half_ref = (int64_t)(ref_len / 2);
    Aligned a;
    const int64_t mag = lag < 0 ? -lag : lag;
    if (lag == 0 || mag > half_ref) {
        a.deg.assign(deg, deg + deg_len);
        return a;
    }
    a.lag_seconds = (double)lag / (double)sample_rate;
    a.lag_samples = lag;
    if (lag < 0) {
        const size_t k = std::min((size_t)(-lag), deg_len);
        a.deg.assign(deg + k, deg + deg_len);
    } else {
        const size_t k = (size_t)lag;
        a.deg.assign(k + deg_len, 0.0);
        std::memcpy(a.deg.data() + k, deg, deg_len * sizeof(double));
    }
    return a;
}

struct Trimmed {
    std::vector<double> ref, deg;
    double lag_seconds = 0;
    size_t ref_off = 0;
    int64_t deg_off = 0;
};

// truncateAligned (src/realign.zig:147-210).
Trimmed truncate_aligned(const double *ref, size_t ref_len, const double *deg, size_t deg_len, int64_t lag,
                         uint32_t sample_rate) {
    Aligned aligned = apply_lag(ref_len, deg, deg_len, lag, sample_rate);
    const size_t dl = aligned.deg.size();
    const double sr_f = (double)sample_rate;
    Trimmed t;
    size_t head = 0;
    if (ref_len > dl) {
        t.ref.assign(ref, ref + dl);
        t.deg = aligned.deg;
    } else if (ref_len < dl) {
        const int64_t ls_i = (int64_t)(aligned.lag_seconds * sr_f);
        if (ls_i > 0) {
            const size_t ls = (size_t)ls_i;
            head = ls;
            t.ref.assign(ref + ls, ref + ref_len);
            const size_t d_take = std::min(ls + t.ref.size(), dl);
            t.deg.assign(aligned.deg.begin() + ls, aligned.deg.begin() + d_take);
        } else {
            t.deg.assign(aligned.deg.begin(), aligned.deg.begin() + ref_len);
            t.ref.assign(ref, ref + ref_len);
        }
    } else {
        t.ref.assign(ref, ref + ref_len);
        t.deg = aligned.deg;
    }
    const size_t min_len = std::min(t.ref.size(), t.deg.size());
    t.ref.resize(min_len);
    t.deg.resize(min_len);
    t.lag_seconds = aligned.lag_seconds;
    t.ref_off = head;
    t.deg_off = (int64_t)head - aligned.lag_samples;
    return t;
}

// lagSamplesBack + trimGeometry (src/realign.zig:223-250).
int64_t lag_samples_back(int64_t lag, uint32_t sample_rate) {
    const double sr_f = (double)sample_rate;
    const double seconds = (double)lag / sr_f;
    return (int64_t)(seconds * sr_f);
}
struct Geometry {
    size_t len, ref_off;
    int64_t deg_off;
    double lag_seconds;
};
Geometry trim_geometry(size_t ref_len, size_t deg_len, int64_t lag, uint32_t sample_rate) {
    const int64_t r = (int64_t)ref_len, d = (int64_t)deg_len;
    const int64_t mag = lag < 0 ? -lag : lag;
    const int64_t shift = (lag == 0 || mag > (int64_t)(ref_len / 2)) ? 0 : lag;
    const int64_t dl = shift < 0 ? d - std::min(-shift, d) : d + shift;
    int64_t head = 0, len = r;
    if (r > dl) {
        len = dl;
    } else if (r < dl && shift > 0) {
        head = std::max<int64_t>(lag_samples_back(shift, sample_rate), 0);
        len = r - head;
    }
    const double sr_f = (double)sample_rate;
    return {(size_t)len, (size_t)head, head - shift, shift == 0 ? 0.0 : (double)shift / sr_f};
}

// RawSpectrograms.reuse (src/realign.zig:262-281).
bool reuse_frames(size_t nb, const double *global, size_t nf_global, const SliceLayout &l, int64_t off, size_t hop,
                  size_t nf_local, double *out) {
    if (off < (int64_t)l.pad) return false;
    const size_t start = l.base + (size_t)off - l.pad;
    if (start % hop != 0) return false;
    const size_t g0 = start / hop;
    if (g0 + nf_local > nf_global) return false;
    for (size_t b = 0; b < nb; ++b) std::memcpy(out + b * nf_local, global + b * nf_global + g0, nf_local * sizeof(double));
    return true;
}

// ---------------------------------------------------------------------
// SVR (src/svr.zig) and the speech exponential map (src/visqol.zig:85-96).
// ---------------------------------------------------------------------
struct SvrModel {
    double gamma = 0.01, rho = 0.0;
    size_t num_features = 0;
    std::vector<double> sv, coeff;

    // Model.predict (src/svr.zig:37-61), f64 kernel.
    double predict(const double *x) const {
        double sum = 0.0;
        for (size_t i = 0; i < coeff.size(); ++i) {
            const double *s = &sv[i * num_features];
            double dist = 0.0;
            for (size_t f = 0; f < num_features; ++f) {
                const double d = s[f] - x[f];
                dist += d * d;
            }
            sum += coeff[i] * std::exp(-gamma * dist);
        }
        return sum - rho;
    }
    double predict_clamped(const double *x) const { return std::min(std::max(predict(x), 1.0), 5.0); }
};

// parseModel (src/svr.zig:80-165).
SvrModel parse_model(const std::string &data) {
    SvrModel m;
    bool saw_sv = false;
    std::vector<std::string> sv_lines;
    size_t max_feat = 0;
    size_t pos = 0;
    auto trim = [](std::string s) {
        size_t a = s.find_first_not_of(" \t");
        size_t b = s.find_last_not_of(" \t");
        return a == std::string::npos ? std::string() : s.substr(a, b - a + 1);
    };
    while (pos <= data.size()) {
        size_t nl = data.find('\n', pos);
        if (nl == std::string::npos) nl = data.size();
        std::string line = data.substr(pos, nl - pos);
        pos = nl + 1;
        if (!line.empty() && line.back() == '\r') line.pop_back();
        if (line.empty()) {
            if (nl == data.size()) break;
            continue;
        }
        if (!saw_sv) {
            if (line == "SV") {
                saw_sv = true;
                continue;
            }
            const size_t sp = line.find(' ');
            if (sp == std::string::npos) continue;
            const std::string key = line.substr(0, sp), val = trim(line.substr(sp + 1));
            char *end = nullptr;
            if (key == "svm_type") {
                if (val != "nu_svr" && val != "epsilon_svr") throw VqError(E_MODEL, "UnsupportedSvmType");
            } else if (key == "kernel_type") {
                if (val != "rbf") throw VqError(E_MODEL, "UnsupportedKernel");
            } else if (key == "gamma") {
                m.gamma = std::strtod(val.c_str(), &end);
                if (end == val.c_str()) throw VqError(E_MODEL, "InvalidModelFile");
            } else if (key == "rho") {
                m.rho = std::strtod(val.c_str(), &end);
                if (end == val.c_str()) throw VqError(E_MODEL, "InvalidModelFile");
            }
            continue;
        }
        sv_lines.push_back(line);
        size_t p = line.find_first_of(" \t");
        while (p != std::string::npos) {
            p = line.find_first_not_of(" \t", p);
            if (p == std::string::npos) break;
            size_t e = line.find_first_of(" \t", p);
            std::string tok = line.substr(p, e == std::string::npos ? std::string::npos : e - p);
            size_t colon = tok.find(':');
            if (colon != std::string::npos) {
                char *end = nullptr;
                unsigned long idx = std::strtoul(tok.substr(0, colon).c_str(), &end, 10);
                if (end && *end == 0 && idx > max_feat) max_feat = idx;
            }
            p = e;
        }
        if (nl == data.size()) break;
    }
    if (sv_lines.empty()) throw VqError(E_MODEL, "NoSupportVectors");
    if (max_feat == 0) throw VqError(E_MODEL, "InvalidModelFile");
    m.num_features = max_feat;
    m.sv.assign(sv_lines.size() * max_feat, 0.0);
    m.coeff.resize(sv_lines.size());
    for (size_t i = 0; i < sv_lines.size(); ++i) {
        const std::string &line = sv_lines[i];
        size_t p = line.find_first_not_of(" \t");
        size_t e = line.find_first_of(" \t", p);
        const std::string c = line.substr(p, e == std::string::npos ? std::string::npos : e - p);
        char *end = nullptr;
        m.coeff[i] = std::strtod(c.c_str(), &end);
        if (end == c.c_str()) throw VqError(E_MODEL, "InvalidModelFile");
        p = e;
        while (p != std::string::npos) {
            p = line.find_first_not_of(" \t", p);
            if (p == std::string::npos) break;
            size_t e2 = line.find_first_of(" \t", p);
            std::string tok = line.substr(p, e2 == std::string::npos ? std::string::npos : e2 - p);
            p = e2;
            size_t colon = tok.find(':');
            if (colon == std::string::npos) continue;
            char *ie = nullptr;
            unsigned long idx = std::strtoul(tok.substr(0, colon).c_str(), &ie, 10);
            if (!ie || *ie != 0) continue;
            const std::string vs = tok.substr(colon + 1);
            char *ve = nullptr;
            double v = std::strtod(vs.c_str(), &ve);
            if (ve == vs.c_str()) continue;
            if (idx == 0 || idx > max_feat) throw VqError(E_MODEL, "InvalidFeatureIndex");
            m.sv[i * max_feat + (idx - 1)] = v;
        }
    }
    return m;
}

std::string default_model_text() { return std::string(vqo_svr_model_start, vqo_svr_model_end - vqo_svr_model_start); }

std::string read_file(const char *path) {
    FILE *f = std::fopen(path, "rb");
    if (!f) throw VqError(-3, "cannot read model file");
    std::string s;
    char buf[65536];
    size_t k;
    while ((k = std::fread(buf, 1, sizeof buf, f)) > 0) s.append(buf, k);
    std::fclose(f);
    return s;
}

// ---------------------------------------------------------------------
// The model (src/visqol.zig).
// ---------------------------------------------------------------------
struct Options {
    bool speech = false;
    int32_t radius = 60;
    bool unscaled_speech = false;
    bool use_lattice = false;
    bool disable_global_alignment = false;
    bool disable_realignment = false;
};

struct ResultData {
    vqo_result c{};
    std::vector<double> fvnsim, fvnsim10, fstdnsim, fvdegenergy, cfb, band_data;
    std::vector<vqo_patch> patches;
};

struct TraceData {
    vqo_trace c{};
    std::vector<int64_t> ref_index, deg_offset, realign_lag, realign_frames;
    std::vector<uint8_t> valid, realign_reused, realign_accepted;
};

class Model {
public:
    Model(const Options &o, const SvrModel *svr) : opt_(o), svr_(svr) {
        nb_ = o.speech ? 21 : 32;
        patch_ = o.speech ? 20 : 30;
        max_freq_ = o.speech ? 8000.0 : -1.0;
    }

    // Pipeline(NB).runBatch for one pair (src/visqol.zig:394-487).
    ResultData *measure(const double *ref, size_t ref_len, const double *deg_in, size_t deg_len, uint32_t sr,
                        TraceData *tr) {
        if (sr == 0) throw VqError(E_INVALID, "InvalidInput");
        ensure_cache(sr);
        Work work;
        // 1: global-alignment lag (src/visqol.zig:425-434).
        int64_t lag = 0;
        if (!opt_.disable_global_alignment && ref_len > 0 && deg_len > 0)
            lag = envelope_lag(ref, ref_len, deg_in, deg_len, &work);
        // 2: prepareSignals (src/visqol.zig:489-517).
        std::vector<double> deg;
        double lag_s = 0.0;
        if (opt_.disable_global_alignment) {
            deg.assign(deg_in, deg_in + deg_len);
        } else {
            Aligned a = apply_lag(ref_len, deg_in, deg_len, lag, sr);
            lag_s = a.lag_seconds;
            deg = std::move(a.deg);
        }
        const double factor = scale_to_match_spl(ref, ref_len, deg.data(), deg.size());
        if (ref_len <= window_ || deg.size() <= window_) throw VqError(E_SIGNAL, "SpectrogramTooShort");
        const size_t nf_ref = num_frames(ref_len, window_, hop_);
        const size_t nf_deg = num_frames(deg.size(), window_, hop_);
        std::vector<double> ref_spec(nb_ * nf_ref), deg_spec(nb_ * nf_deg);
        // 3: spectrograms.
        build_spectrogram(filters_.bands, ref, ref_len, window_, hop_, hann_.data(), ref_spec.data());
        build_spectrogram(filters_.bands, deg.data(), deg.size(), window_, hop_, hann_.data(), deg_spec.data());
        work.n_rms += nb_ * (nf_ref + nf_deg);
        // 4-5: planPair (src/visqol.zig:519-555).
        std::vector<double> ref_raw, deg_raw;
        if (!opt_.disable_realignment) ref_raw = ref_spec, deg_raw = deg_spec;
        prepare_for_comparison(ref_spec.data(), deg_spec.data(), nb_, nf_ref, nf_deg);
        std::vector<size_t> idx = opt_.speech
                                      ? vad_patch_indices(ref, ref_len, nf_ref, patch_, window_, 0.25)
                                      : ref_patch_indices(nf_ref, patch_);
        if (idx.empty()) throw VqError(E_SIGNAL, "NoPatches");
        SearchPlan plan = plan_search(idx, nf_ref, nf_deg, patch_, opt_.radius);
        // 6a: DP similarity matrix.
        patch_similarities(ref_spec.data(), nf_ref, deg_spec.data(), nf_deg, nb_, patch_, idx, plan, &work);
        // 6b: DP, backtrack, per-match NSIM (src/visqol.zig:557-591).
        std::vector<Match> matches = find_optimal_deg_patches(plan, ref_spec.data(), idx, deg_spec.data(), nb_, nf_ref,
                                                              patch_, frame_duration_, &work);
        // 7: realign (src/realign.zig:294-460).
        if (!opt_.disable_realignment)
            realign(matches, ref, ref_len, deg.data(), deg.size(), sr, ref_raw, nf_ref, deg_raw, nf_deg, &work);
        // 8: buildResult.
        ResultData *r = build_result(matches, lag_s);
        if (tr) {
            tr->c.global_lag = lag;
            tr->c.spl_factor = factor;
            tr->c.deg_len = deg.size();
            tr->c.nf_ref = nf_ref;
            tr->c.nf_deg = nf_deg;
            tr->c.num_patches = matches.size();
            for (size_t i = 0; i < matches.size(); ++i) {
                tr->ref_index.push_back((int64_t)idx[i]);
                tr->deg_offset.push_back(matches[i].deg_offset);
                tr->valid.push_back(matches[i].valid ? 1 : 0);
                tr->realign_lag.push_back(matches[i].realign_lag);
                tr->realign_frames.push_back(matches[i].realign_frames);
                tr->realign_reused.push_back(matches[i].realign_reused);
                tr->realign_accepted.push_back(matches[i].realign_accepted ? 1 : 0);
            }
            tr->c.n_rms = work.n_rms;
            tr->c.n_rms_window = window_;
            tr->c.n_cells = work.n_cells;
            tr->c.fft_nlogn = work.fft_nlogn;
        }
        return r;
    }

    size_t nb() const { return nb_; }

private:
    // ensureCache (src/visqol.zig:346-359).
    void ensure_cache(uint32_t sr) {
        if (sr == cached_sr_) return;
        const double sr_f = (double)sr;
        filters_ = make_filters(nb_, sr, 50.0, max_freq_ > 0 ? max_freq_ : sr_f / 2.0);
        window_ = (size_t)std::round(sr_f * 0.08);
        hop_ = (size_t)((double)window_ * 0.25);
        if (hop_ == 0) hop_ = 1;
        hann_.resize(window_);
        hann_window(window_, hann_.data());
        frame_duration_ = (double)hop_ / sr_f;
        cached_sr_ = sr;
    }

    // planRealign + realignCpu + finishRealign (src/realign.zig:294-460).
    void realign(std::vector<Match> &matches, const double *ref, size_t ref_len, const double *deg, size_t deg_len,
                 uint32_t sr, const std::vector<double> &ref_raw, size_t nf_ref, const std::vector<double> &deg_raw,
                 size_t nf_deg, Work *work) {
        for (auto &m : matches) {
            if (!m.valid) continue;
            const SliceLayout rl = slice_layout(ref_len, sr, m.ref_start, m.ref_end);
            const SliceLayout dl = slice_layout(deg_len, sr, m.deg_start, m.deg_end);
            const size_t rlen = rl.pad + rl.len, dlen = dl.pad + dl.len;
            if (rlen < window_ || dlen < window_) continue;
            // realignCpu.
            std::vector<double> ref_audio = slice_view(ref, rl), deg_audio = slice_view(deg, dl);
            const int64_t lag = envelope_lag(ref_audio.data(), rlen, deg_audio.data(), dlen, work);
            m.realign_lag = lag;
            Trimmed t = truncate_aligned(ref_audio.data(), rlen, deg_audio.data(), dlen, lag, sr);
            const size_t nf = num_frames(t.ref.size(), window_, hop_);
            m.realign_frames = (int64_t)nf;
            if (nf == 0) continue;
            std::vector<double> rs(nb_ * nf), ds(nb_ * nf);
            if (reuse_frames(nb_, ref_raw.data(), nf_ref, rl, (int64_t)t.ref_off, hop_, nf, rs.data())) {
                m.realign_reused |= 1;
            } else {
                build_spectrogram(filters_.bands, t.ref.data(), t.ref.size(), window_, hop_, hann_.data(), rs.data());
                work->n_rms += nb_ * nf;
            }
            if (reuse_frames(nb_, deg_raw.data(), nf_deg, dl, t.deg_off, hop_, nf, ds.data())) {
                m.realign_reused |= 2;
            } else {
                build_spectrogram(filters_.bands, t.deg.data(), t.deg.size(), window_, hop_, hann_.data(), ds.data());
                work->n_rms += nb_ * nf;
            }
            // finishRealign.
            const Geometry geo = trim_geometry(rlen, dlen, lag, sr);
            prepare_for_comparison(rs.data(), ds.data(), nb_, nf, nf);
            Scratch s(nb_, nf);
            std::vector<double> means(nb_), stddevs(nb_), energy(nb_);
            const double mean = s.patch_similarity(rs.data(), ds.data(), means.data(), stddevs.data(), energy.data());
            work->n_cells += nb_ * nf;
            if (!(mean < m.similarity)) {
                m.means = means, m.stddevs = stddevs, m.energy = energy;
                m.similarity = mean;
                m.realign_accepted = true;
                const double new_dur = (double)geo.len / (double)sr;
                if (geo.lag_seconds > 0.0)
                    m.ref_start += geo.lag_seconds;
                else
                    m.deg_start -= geo.lag_seconds;
                m.ref_end = m.ref_start + new_dur;
                m.deg_end = m.deg_start + new_dur;
            }
        }
    }

    // QualityMapper.predict (src/visqol.zig:81-98).
    double predict(const std::vector<double> &fvnsim) const {
        if (!opt_.speech) return svr_->predict_clamped(fvnsim.data());
        if (opt_.use_lattice) throw VqError(E_MODEL, "lattice mapper is not restated");
        const double a = -262.847869, b = 0.0154302525, x0 = -361.063949;
        double sum = 0.0;
        for (double x : fvnsim) sum += x;
        const double nsim_mean = sum / (double)fvnsim.size();
        const double mos = a + std::exp(b * (nsim_mean - x0));
        const double scale = !opt_.unscaled_speech ? (double)1.245063f : 1.0;
        return std::min(std::max(mos * scale, 1.0), 5.0);
    }

    // buildResult (src/visqol.zig:595-709).
    ResultData *build_result(const std::vector<Match> &matches, double lag_s) {
        const size_t n = matches.size(), NB = nb_;
        const double n_f = (double)n;
        auto *r = new ResultData();
        r->fvnsim.assign(NB, 0.0);
        r->fvdegenergy.assign(NB, 0.0);
        r->fvnsim10.assign(NB, 0.0);
        r->fstdnsim.assign(NB, 0.0);
        r->cfb = filters_.cf;
        for (const auto &m : matches)
            for (size_t b = 0; b < NB; ++b) {
                r->fvnsim[b] += m.means[b];
                r->fvdegenergy[b] += m.energy[b];
            }
        for (size_t b = 0; b < NB; ++b) {
            r->fvnsim[b] /= n_f;
            r->fvdegenergy[b] /= n_f;
        }
        {
            std::vector<double> sorted(n);
            const size_t k = std::max<size_t>(1, (size_t)std::trunc(n_f * 0.10));
            for (size_t b = 0; b < NB; ++b) {
                for (size_t i = 0; i < n; ++i) sorted[i] = matches[i].means[b];
                std::sort(sorted.begin(), sorted.end());
                double acc = 0.0;
                for (size_t i = 0; i < k; ++i) acc += sorted[i];
                r->fvnsim10[b] = acc / (double)k;
            }
        }
        {
            std::vector<double> contribution(NB, 0.0);
            int64_t total_frame_count = 0;
            for (const auto &m : matches) {
                const double secs = m.ref_end - m.ref_start;
                const int64_t fc_i = (int64_t)std::ceil(secs / frame_duration_);
                total_frame_count += fc_i;
                const double fc = (double)fc_i;
                for (size_t b = 0; b < NB; ++b) {
                    const double dev = m.stddevs[b], mean = m.means[b];
                    contribution[b] += (fc - 1.0) * dev * dev;
                    contribution[b] += fc * mean * mean;
                }
            }
            const double total_f = (double)total_frame_count;
            for (size_t b = 0; b < NB; ++b) {
                const double v = (contribution[b] - r->fvnsim[b] * r->fvnsim[b] * total_f) / (total_f - 1.0);
                r->fstdnsim[b] = v < 0.0 ? 0.0 : std::sqrt(v);
            }
        }
        double sum = 0.0;
        for (double x : r->fvnsim) sum += x;
        const double vnsim = sum / (double)NB;
        double mos = predict(r->fvnsim);
        if (vnsim < 0.15) mos = 1.0;
        r->band_data.assign(n * NB * 3, 0.0);
        r->patches.resize(n);
        for (size_t i = 0; i < n; ++i) {
            double *dst = &r->band_data[i * NB * 3];
            const Match &m = matches[i];
            std::copy(m.means.begin(), m.means.end(), dst);
            std::copy(m.stddevs.begin(), m.stddevs.end(), dst + NB);
            std::copy(m.energy.begin(), m.energy.end(), dst + 2 * NB);
            r->patches[i] = {m.similarity, m.ref_start, m.ref_end, m.deg_start, m.deg_end, dst, dst + NB, dst + 2 * NB};
        }
        r->c.moslqo = mos;
        r->c.vnsim = vnsim;
        r->c.alignment_lag_s = lag_s;
        r->c.num_bands = NB;
        r->c.fvnsim = r->fvnsim.data();
        r->c.fvnsim10 = r->fvnsim10.data();
        r->c.fstdnsim = r->fstdnsim.data();
        r->c.fvdegenergy = r->fvdegenergy.data();
        r->c.center_freq_bands = r->cfb.data();
        r->c.num_patches = n;
        r->c.patch_sims = r->patches.data();
        return r;
    }

    Options opt_;
    const SvrModel *svr_;
    size_t nb_, patch_;
    double max_freq_;
    uint32_t cached_sr_ = 0;
    Filters filters_;
    size_t window_ = 0, hop_ = 0;
    std::vector<double> hann_;
    double frame_duration_ = 0;
};

Options to_options(const vqo_options *o) {
    Options opt;
    if (!o) return opt;
    if (o->mode > 1) throw VqError(E_INVALID, "invalid mode");
    opt.speech = o->mode == 1;
    opt.radius = o->search_window_radius > 0 ? o->search_window_radius : 60;
    opt.unscaled_speech = o->use_unscaled_speech_mos_mapping != 0;
    opt.disable_global_alignment = o->disable_global_alignment != 0;
    opt.disable_realignment = o->disable_realignment != 0;
    opt.use_lattice = o->use_lattice_model != 0;
    return opt;
}

std::unique_ptr<SvrModel> load_svr(const vqo_options *o) {
    std::string text = (o && o->model_path && o->model_path[0]) ? read_file(o->model_path) : default_model_text();
    return std::make_unique<SvrModel>(parse_model(text));
}

ResultData *from_c(vqo_result *r) { return reinterpret_cast<ResultData *>(r); }

}  // namespace

// ---------------------------------------------------------------------
// C API.
// ---------------------------------------------------------------------
extern "C" {

const char *vqo_last_error(void) { return g_last_error.c_str(); }

void vqo_options_default(vqo_options *o) {
    if (!o) return;
    std::memset(o, 0, sizeof *o);
    o->search_window_radius = 60;
    o->use_lattice_model = 1;
    o->precision = 3;
}

int vqo_measure(const vqo_options *o, const double *ref, size_t ref_len, const double *deg, size_t deg_len,
                uint32_t sample_rate, vqo_result **out, vqo_trace **trace) {
    if (!out) return E_INVALID;
    *out = nullptr;
    if (trace) *trace = nullptr;
    try {
        const Options opt = to_options(o);
        std::unique_ptr<SvrModel> svr = load_svr(o);
        Model model(opt, svr.get());
        std::unique_ptr<TraceData> tr(trace ? new TraceData() : nullptr);
        ResultData *r = model.measure(ref, ref_len, deg, deg_len, sample_rate, tr.get());
        static_assert(offsetof(ResultData, c) == 0, "result view first");
        *out = &r->c;
        if (trace) {
            TraceData *t = tr.release();
            t->c.ref_index = t->ref_index.data();
            t->c.deg_offset = t->deg_offset.data();
            t->c.valid = t->valid.data();
            t->c.realign_lag = t->realign_lag.data();
            t->c.realign_frames = t->realign_frames.data();
            t->c.realign_reused = t->realign_reused.data();
            t->c.realign_accepted = t->realign_accepted.data();
            *trace = &t->c;
        }
        return 0;
    } catch (const VqError &e) {
        g_last_error = e.what();
        return e.code;
    } catch (const std::exception &e) {
        g_last_error = e.what();
        return -7;
    }
}

void vqo_result_free(vqo_result *r) { delete from_c(r); }
void vqo_trace_free(vqo_trace *t) { delete reinterpret_cast<TraceData *>(t); }

int vqo_measure_batch(const vqo_options *o, size_t n, const double *const *refs, const size_t *ref_lens,
                      const double *const *degs, const size_t *deg_lens, uint32_t sample_rate, uint32_t num_threads,
                      vqo_result **out, int32_t *status) {
    if (n == 0) return 0;
    Options opt;
    std::unique_ptr<SvrModel> svr;
    try {
        opt = to_options(o);
        svr = load_svr(o);
    } catch (const VqError &e) {
        g_last_error = e.what();
        return e.code;
    }
    unsigned want = num_threads ? num_threads : std::max(1u, std::thread::hardware_concurrency());
    const size_t nt = std::max<size_t>(1, std::min<size_t>(want, n));
    std::atomic<size_t> next{0};
    auto worker = [&]() {
        Model model(opt, svr.get());
        for (;;) {
            const size_t i = next.fetch_add(1);
            if (i >= n) return;
            int rc = 0;
            out[i] = nullptr;
            try {
                ResultData *r = model.measure(refs[i], ref_lens[i], degs[i], deg_lens[i], sample_rate, nullptr);
                out[i] = &r->c;
            } catch (const VqError &e) {
                rc = e.code;
            } catch (const std::exception &) {
                rc = -7;
            }
            if (status) status[i] = rc;
        }
    };
    std::vector<std::thread> threads;
    for (size_t t = 1; t < nt; ++t) threads.emplace_back(worker);
    worker();
    for (auto &t : threads) t.join();
    int first = 0;
    if (status)
        for (size_t i = 0; i < n; ++i)
            if (status[i] != 0) {
                first = status[i];
                break;
            }
    return first;
}

void vqo_uniform_center_freqs(size_t n, double low, double high, double *out) { uniform_center_freqs(n, low, high, out); }

void vqo_filters(size_t nb, uint32_t sample_rate, double low, double high, double *coeffs, double *cf) {
    Filters f = make_filters(nb, sample_rate, low, high);
    for (size_t b = 0; b < nb; ++b) {
        const Band &x = f.bands[b];
        const double v[8] = {x.a0, x.a11, x.a12, x.a13, x.a14, x.b1, x.b2, x.gain};
        std::memcpy(coeffs + 8 * b, v, sizeof v);
        if (cf) cf[b] = f.cf[b];
    }
}

void vqo_hann(size_t size, double *out) { hann_window(size, out); }

static Band band_of(const double *c) { return {c[0], c[1], c[2], c[3], c[4], c[5], c[6], c[7]}; }

void vqo_filter_band(const double *c8, const double *x, size_t n, double *out) {
    // filterBand from a fresh BandState: applyStage x4 (src/gammatone.zig:193-265).
    const Band band = band_of(c8);
    const double gi = 1.0 / band.gain;
    std::vector<double> a(x, x + n), b(n);
    const double n0s[4] = {band.a0 * gi, band.a0, band.a0, band.a0};
    const double n1s[4] = {band.a11 * gi, band.a12, band.a13, band.a14};
    for (int st = 0; st < 4; ++st) {
        double c0 = 0, c1 = 0;
        for (size_t i = 0; i < n; ++i) {
            const double s = a[i];
            const double filtered = n0s[st] * s + c0;
            c0 = n1s[st] * s + c1 - band.b1 * filtered;
            c1 = -(band.b2 * filtered);
            b[i] = filtered;
        }
        std::swap(a, b);
    }
    std::memcpy(out, a.data(), n * sizeof(double));
}

double vqo_filter_band_rms_fresh(const double *c8, const double *x, size_t n) {
    return filter_band_rms_fresh(band_of(c8), x, n);
}

size_t vqo_spectrogram(size_t nb, const double *coeffs, const double *hann, size_t window, size_t hop, const double *x,
                       size_t n, double *out) {
    std::vector<Band> bands(nb);
    for (size_t b = 0; b < nb; ++b) bands[b] = band_of(coeffs + 8 * b);
    return build_spectrogram(bands, x, n, window, hop, hann, out);
}

void vqo_upper_envelope(const double *x, size_t n, double *out) { upper_envelope(x, n, out); }
size_t vqo_fft_size_for(size_t biggest) { return fft_size_for(biggest); }

void vqo_fft_dif(double *buf, size_t n) {
    FftPlan p;
    p.init(n);
    dif_forward(p, reinterpret_cast<Cx *>(buf));
}
void vqo_fft_dit(double *buf, size_t n) {
    FftPlan p;
    p.init(n);
    dit_inverse(p, reinterpret_cast<Cx *>(buf));
}
void vqo_fft_twiddles(size_t n, double *out) {
    FftPlan p;
    p.init(n);
    std::memcpy(out, p.top.data(), p.top.size() * sizeof(Cx));
}
int64_t vqo_best_lag(const double *a, size_t la, const double *b, size_t lb) { return best_lag(a, la, b, lb, nullptr); }
int64_t vqo_envelope_lag(const double *a, size_t la, const double *b, size_t lb) {
    return envelope_lag(a, la, b, lb, nullptr);
}
void vqo_convert_to_db(double *x, size_t n, double floor_db) { convert_to_db(x, n, floor_db); }
void vqo_raise_floor_per_frame(double *ref, double *deg, size_t nb, size_t nfr, size_t nfd, double rel) {
    raise_floor_per_frame(ref, deg, nb, nfr, nfd, rel);
}
void vqo_subtract_joint_minimum(double *ref, size_t rn, double *deg, size_t dn) {
    subtract_joint_minimum(ref, rn, deg, dn);
}
void vqo_prepare_for_comparison(double *ref, double *deg, size_t nb, size_t nfr, size_t nfd) {
    prepare_for_comparison(ref, deg, nb, nfr, nfd);
}
void vqo_conv2d3x3(const double *in, double *out, size_t nrows, size_t ncols) { conv2d3x3(in, out, nrows, ncols); }
double vqo_patch_similarity(const double *ref, const double *deg, size_t nrows, size_t ncols, double *means,
                            double *stddevs, double *deg_energy) {
    Scratch s(nrows, ncols);
    return s.patch_similarity(ref, deg, means, stddevs, deg_energy);
}
double vqo_similarity_scalar(const double *ref, const double *deg, size_t nrows, size_t ncols) {
    Scratch s(nrows, ncols);
    return s.similarity_scalar(ref, deg);
}
void vqo_nsim_table(const double *ref_spec, size_t nf_ref, const double *deg_spec, size_t nf_deg, size_t nb, size_t patch,
                    size_t np, const int64_t *ref_idx, const int64_t *lo, const int64_t *hi, double *out) {
    for (size_t i = 0; i < np; ++i)
        if (lo[i] < 0 || hi[i] < lo[i] || (size_t)hi[i] >= nf_deg || ref_idx[i] < 0 || (size_t)ref_idx[i] + patch > nf_ref)
            return;  // out-of-range windows: nothing written
    SearchPlan plan;
    plan.num_patches = np;
    plan.nf_deg = nf_deg;
    std::vector<size_t> idx(np);
    plan.lo.resize(np), plan.hi.resize(np);
    for (size_t i = 0; i < np; ++i) idx[i] = (size_t)ref_idx[i], plan.lo[i] = (size_t)lo[i], plan.hi[i] = (size_t)hi[i];
    plan.sims.assign(np * nf_deg, 0.0);
    patch_similarities(ref_spec, nf_ref, deg_spec, nf_deg, nb, patch, idx, plan, nullptr);
    std::memcpy(out, plan.sims.data(), plan.sims.size() * sizeof(double));
}
size_t vqo_dp_backtrack(const double *sims, size_t np, size_t nf_deg, const int64_t *lo, const int64_t *hi,
                        int64_t *offset, uint8_t *valid) {
    SearchPlan plan;
    plan.num_patches = np;
    plan.nf_deg = nf_deg;
    plan.lo.resize(np), plan.hi.resize(np);
    for (size_t i = 0; i < np; ++i) plan.lo[i] = (size_t)lo[i], plan.hi[i] = (size_t)hi[i];
    plan.sims.assign(sims, sims + np * nf_deg);
    DpOut d = dp_backtrack(plan);
    size_t reached = 0;
    for (size_t i = 0; i < np; ++i) {
        offset[i] = d.offset[i];
        valid[i] = d.valid[i];
        reached += d.reached[i];
    }
    return reached;
}
int vqo_ref_patch_indices(size_t nf, size_t patch, int64_t *out, size_t *count) {
    try {
        std::vector<size_t> v = ref_patch_indices(nf, patch);
        for (size_t i = 0; i < v.size(); ++i) out[i] = (int64_t)v[i];
        *count = v.size();
        return 0;
    } catch (const VqError &e) {
        *count = 0;
        return e.code;
    }
}
int vqo_vad_patch_indices(const double *ref, size_t n, size_t nf, size_t patch, size_t window, double overlap,
                          int64_t *out, size_t *count) {
    std::vector<size_t> v = vad_patch_indices(ref, n, nf, patch, window, overlap);
    for (size_t i = 0; i < v.size(); ++i) out[i] = (int64_t)v[i];
    *count = v.size();
    return 0;
}
size_t vqo_calc_max_num_patches(const int64_t *idx, size_t n, size_t nf_deg, size_t patch) {
    std::vector<size_t> v(idx, idx + n);
    return calc_max_num_patches(v, nf_deg, patch);
}
void vqo_slice_layout(size_t len, uint32_t sr, double t0, double t1, int64_t *pad, int64_t *base, int64_t *n) {
    SliceLayout l = slice_layout(len, sr, t0, t1);
    *pad = (int64_t)l.pad, *base = (int64_t)l.base, *n = (int64_t)l.len;
}
void vqo_trim_geometry(size_t ref_len, size_t deg_len, int64_t lag, uint32_t sr, int64_t *len, int64_t *ref_off,
                       int64_t *deg_off, double *lag_seconds) {
    Geometry g = trim_geometry(ref_len, deg_len, lag, sr);
    *len = (int64_t)g.len, *ref_off = (int64_t)g.ref_off, *deg_off = g.deg_off, *lag_seconds = g.lag_seconds;
}
size_t vqo_truncate_aligned(const double *ref, size_t ref_len, const double *deg, size_t deg_len, int64_t lag,
                            uint32_t sr, double *ref_out, double *deg_out) {
    Trimmed t = truncate_aligned(ref, ref_len, deg, deg_len, lag, sr);
    std::memcpy(ref_out, t.ref.data(), t.ref.size() * sizeof(double));
    std::memcpy(deg_out, t.deg.data(), t.deg.size() * sizeof(double));
    return t.ref.size();
}
double vqo_spl(const double *x, size_t n) { return sound_pressure_level(x, n); }
double vqo_pow(double x, double y) { return zig_pow(x, y); }
int vqo_svr_predict_text(const char *text, size_t len, const double *x, size_t n, double *y) {
    try {
        SvrModel m = parse_model(std::string(text, len));
        if (n != m.num_features) return E_INVALID;
        *y = m.predict(x);
        return 0;
    } catch (const VqError &e) {
        g_last_error = e.what();
        return e.code;
    }
}
int vqo_svr_predict(const char *model_path, const double *x, size_t n, double *y) {
    try {
        std::string t = (model_path && model_path[0]) ? read_file(model_path) : default_model_text();
        return vqo_svr_predict_text(t.data(), t.size(), x, n, y);
    } catch (const VqError &e) {
        g_last_error = e.what();
        return e.code;
    }
}

}  // extern "C"
