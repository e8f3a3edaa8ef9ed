// Speech-mode TF-Lattice MOS mapping (reference src/lattice.zig:14-71, the
// upstream TFLiteQualityMapper): one f32 scalar input per (feature, band),
// named fvnsim<b>, fvnsim10_<b>, fstdnsim<b>, fvdegenergy<b>, plus tau = 0.5;
// the f32 "predictions" output widened to f64 without clamping.
#include <string>

#include "host_model.h"
#include "tflite.h"

#define VQB_STR2(x) #x
#define VQB_STR(x) VQB_STR2(x)

// The bundled lattice model, embedded at build time.
__asm__(".section .rodata\n"
        ".balign 16\n"
        "vqb_lattice_model_begin:\n"
        ".incbin \"" VQB_STR(VQB_LATTICE_PATH) "\"\n"
        "vqb_lattice_model_finish:\n"
        ".byte 0\n"
        ".previous\n");
extern "C" const char vqb_lattice_model_begin[];
extern "C" const char vqb_lattice_model_finish[];

namespace vqb {
namespace host {

const std::string &default_lattice_bytes() {
    static const std::string bytes(vqb_lattice_model_begin, vqb_lattice_model_finish - vqb_lattice_model_begin);
    return bytes;
}

struct LatticeMapper::Impl {
    tfl::Model model;
    size_t nb;
    std::vector<int> feature;  // feature-major: fvnsim, fvnsim10_, fstdnsim, fvdegenergy
    int tau, out;
    Impl(const std::string &bytes, size_t nbands) : model(bytes), nb(nbands) {
        static const char *kNames[4] = {"fvnsim", "fvnsim10_", "fstdnsim", "fvdegenergy"};
        for (const char *f : kNames)
            for (size_t b = 0; b < nb; ++b) {
                const int t = model.input(std::string(f) + std::to_string(b));
                if (t < 0) throw Error(kModel, std::string("MissingInput: ") + f + std::to_string(b));
                feature.push_back(t);
            }
        tau = model.input("tau");
        out = model.output("predictions");
        if (tau < 0 || out < 0) throw Error(kModel, "MissingInput: tau or predictions");
    }
};

LatticeMapper::LatticeMapper(const std::string &bytes, size_t nb) : impl_(std::make_unique<Impl>(bytes, nb)) {}
LatticeMapper::~LatticeMapper() = default;

double LatticeMapper::predict(const double *fvnsim, const double *fvnsim10, const double *fstdnsim,
                              const double *fvdegenergy) const {
    const size_t nb = impl_->nb;
    const double *feats[4] = {fvnsim, fvnsim10, fstdnsim, fvdegenergy};
    std::vector<std::pair<int, tfl::Value>> feeds;
    feeds.reserve(4 * nb + 1);
    auto scalar = [](float v) {
        tfl::Value x;
        x.shape = tfl::Shape::of({1});
        x.f.assign(1, v);
        return x;
    };
    for (int f = 0; f < 4; ++f)
        for (size_t b = 0; b < nb; ++b) feeds.emplace_back(impl_->feature[f * nb + b], scalar((float)feats[f][b]));
    feeds.emplace_back(impl_->tau, scalar(0.5f));
    thread_local tfl::Model::Workspace ws;
    const tfl::Value &y = impl_->model.run(feeds, impl_->out, ws);
    if (y.type != tfl::DType::F32 || y.f.empty()) throw Error(kModel, "ShapeMismatch: predictions");
    return (double)y.f[0];
}

}  // namespace host
}  // namespace vqb
