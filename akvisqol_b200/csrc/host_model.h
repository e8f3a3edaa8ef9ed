// Host-side parts of the ViSQOL model: filter design, planning of the
// data-dependent steps between device stages, the SPL factor, and the MOS
// mapping. Each restates the reference function it cites; all run in f64
// with glibc transcendentals and no FMA contraction, as the reference's Zig
// CPU code on Linux.
#pragma once

#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <memory>
#include <string>
#include <vector>

#include "device.cuh"

namespace vqb {

// Error with a visqol.h code.
struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

constexpr int kInvalid = -1, kOom = -2, kIo = -3, kModel = -4, kSignal = -5, kBackend = -6, kInternal = -7;

namespace host {

// Zig std.math.pow for f64 (the Go math.Pow method): exp(yf*log(x)) for the
// fractional part of y, repeated squaring of frexp(x) for the integral part.
double zig_pow(double x, double y);

struct Filterbank {
    size_t nb = 0;
    std::vector<double> coeffs;   // nb x {a0,a11,a12,a13,a14,b1,b2,gain}, ascending
    std::vector<double> cf;       // centre frequencies, ascending
    std::vector<BandCoeffs> run;  // filterBandRmsFresh's derived coefficients
};

// Filters.init (reference src/gammatone.zig:41-70) with ERB spacing from
// src/dsp/erb.zig:20-52.
Filterbank make_filterbank(size_t nb, uint32_t sample_rate, double low, double high);
// Derived per-band coefficients (reference src/gammatone.zig:269-277).
BandCoeffs band_coeffs(const double *c8);

// hannWindow (reference src/gammatone.zig:309-316).
std::vector<double> hann(size_t size);

// FFT twiddles W_n^k for k < n/2 as (-2*pi*k)/n (reference src/dsp/fft.zig:55-61).
std::vector<double2> twiddles(size_t n);

size_t num_frames(size_t len, size_t window, size_t hop);
size_t fft_size_for(size_t biggest);

// ensureCache's analysis geometry (reference src/visqol.zig:346-359).
struct Geometry {
    size_t window, hop;
    double frame_duration;
};
Geometry analysis_geometry(uint32_t sample_rate);

// refPatchIndices (reference src/dp.zig:47-70).
std::vector<int64_t> ref_patch_indices(size_t nf, size_t patch);
// vad.refPatchIndices (reference src/vad.zig:15-81).
std::vector<int64_t> vad_patch_indices(const double *ref, size_t len, size_t nf, size_t patch, size_t window,
                                       double overlap);
// calcMaxNumPatches (reference src/dp.zig:73-87).
size_t max_num_patches(const std::vector<int64_t> &idx, size_t nf_deg, size_t patch);

// planSearch (reference src/dp.zig:153-201): patches kept and their
// inclusive degraded-offset windows.
struct Search {
    size_t np = 0;
    std::vector<int64_t> lo, hi;
};
Search plan_search(const std::vector<int64_t> &idx, size_t nf_ref, size_t nf_deg, size_t patch, int32_t radius);

// sliceLayout (reference src/realign.zig:41-51).
struct Slice {
    int64_t pad, base, len;
};
Slice slice_layout(size_t signal_len, uint32_t sample_rate, double t0, double t1);

// trimGeometry (reference src/realign.zig:223-250).
struct Trim {
    int64_t len, ref_off, deg_off;
    double lag_seconds;
};
Trim trim_geometry(int64_t ref_len, int64_t deg_len, int64_t lag, uint32_t sample_rate);

// RawSpectrograms.reuse's test (reference src/realign.zig:262-281): the
// first global frame to copy, or -1 when the frames are off the grid.
int64_t reuse_frame(const Slice &l, int64_t off, size_t hop, size_t nf_local, size_t nf_global);

// Aligned degraded geometry of applyLag (reference src/realign.zig:91-110):
// aligned[i] = deg[i + skip] with `lead` zeros first.
struct Aligned {
    int64_t lead, skip, len;
    double lag_seconds;
};
Aligned apply_lag_geometry(size_t ref_len, size_t deg_len, int64_t lag, uint32_t sample_rate);

// soundPressureLevel / scaleToMatchSpl's factor from energies
// (reference src/audio.zig:132-158); 1 when either SPL is not finite.
double spl_of_energy(double energy, size_t len);
double spl_factor(double ref_energy, size_t ref_len, double deg_energy, size_t deg_len);

// libsvm nu-SVR RBF model (reference src/svr.zig).
struct Svr {
    double gamma = 0.01, rho = 0.0;
    size_t nf = 0;
    std::vector<double> sv, coeff;
    double predict(const double *x) const;
};
Svr parse_svr(const std::string &text);
const std::string &default_svr_text();

// One matched patch as buildResult consumes it.
struct Match {
    double similarity = 0, ref_start = 0, ref_end = 0, deg_start = 0, deg_end = 0;
    std::vector<double> means, stddevs, energy;
    bool valid = true;
};

struct ResultBox;  // defined in capi.cpp

struct Scores {
    double moslqo = 0, vnsim = 0, lag_s = 0;
    std::vector<double> fvnsim, fvnsim10, fstdnsim, fvdegenergy, cf;
    std::vector<Match> patches;
};

// buildResult (reference src/visqol.zig:595-709) with QualityMapper.predict
// (src/visqol.zig:81-98): SVR in audio mode, the exponential fit in speech.
// Speech-mode TF-Lattice mapping (reference src/lattice.zig:14-71). The
// model bytes are parsed once; predict is const and thread-safe.
class LatticeMapper {
public:
    LatticeMapper(const std::string &model_bytes, size_t nb);
    ~LatticeMapper();
    double predict(const double *fvnsim, const double *fvnsim10, const double *fstdnsim,
                   const double *fvdegenergy) const;

private:
    struct Impl;
    std::unique_ptr<Impl> impl_;
};
const std::string &default_lattice_bytes();

// lattice: the speech-mode mapping when set (else the exponential fit).
Scores build_scores(std::vector<Match> matches, size_t nb, double frame_duration, const Svr *svr, bool speech,
                    bool unscaled_speech, const std::vector<double> &cf, double lag_s,
                    const LatticeMapper *lattice = nullptr);

// decodeWavAsMono (reference src/audio.zig:48-129).
std::vector<double> decode_wav(const std::string &bytes, uint32_t *sample_rate);
std::string read_file(const std::string &path);

// A batch cut into at most `chunks` runs of consecutive pairs by size (a
// pair's samples or bytes, `sizes`), for the lanes' chunk queues: the first
// `lanes` chunks at front/100 of the average size, so that every lane starts
// soon, the rest of equal size (front 0 or >= 100, or no more chunks than
// lanes: equal sizes throughout). Returns the bounds 0 = b0 < b1 < ... = n,
// every chunk holding at least one pair (fewer chunks where single pairs
// span several targets); {0} for an empty batch.
std::vector<size_t> chunk_bounds(const std::vector<size_t> &sizes, size_t chunks, size_t lanes, size_t front);

}  // namespace host
}  // namespace vqb
