// Host half of the gradient of MOS with respect to the degraded signal
// (reference backend.Engine.measureBatchGrad, src/backend.zig:101-109; its
// GPU flow src/gpu/pipeline.zig:842-1143). The discrete choices of the
// forward pass stay fixed: lags, patch matches, realignment decisions, and
// which cells the spectrogram floors and the joint minimum select. Each
// function here is the reverse of one forward step, in f64:
//
//   MOS mapping -> buildResult -> per-patch band statistics (NSIM)
//     -> prepared spectrograms -> raw (RMS) spectrograms
//
// The gammatone filterbank's reverse (RMS spectrogram -> samples) runs on
// the device (k_grad.cu); the SPL scaling and the lag shift are undone on
// the host by the engine.
#pragma once

#include <cstddef>
#include <vector>

#include "host_model.h"

namespace vqb {
namespace host {

// d MOS / d (one match's band means, standard deviations, energies).
struct MatchGrad {
    std::vector<double> dmeans, dstddevs, denergy;
};

// The MOS of build_scores and its gradient with respect to every match's
// band statistics (out, one per match; zero where the mapping is clamped or
// vnsim < 0.15). SVR and the exponential fit analytically (reference
// src/svr.zig:37-67, src/visqol.zig:81-98); the lattice mapper by central
// differences over its four feature vectors, as the reference does.
double scores_grad(const std::vector<Match> &matches, size_t nb, double frame_duration, const Svr *svr, bool speech,
                   bool unscaled_speech, const LatticeMapper *lattice, std::vector<MatchGrad> &out);

// measurePatchSimilarity's reverse (reference src/nsim.zig:427-510): ref and
// deg are nb x ncols prepared cells (row-major); the gradients with respect
// to the patch's band means, standard deviations and deg energies are
// accumulated into dref and ddeg (nb x ncols).
void patch_similarity_grad(const double *ref, const double *deg, size_t nb, size_t ncols, const double *dmeans,
                           const double *dstddevs, const double *denergy, double *dref, double *ddeg);

// prepareForComparison's reverse (reference src/spectrogram.zig:69-80): from
// the raw (RMS) spectrograms (nb x nfr, nb x nfd) and the gradients with
// respect to the prepared cells, the gradient with respect to the raw
// degraded cells (accumulated into g_deg_raw). The dB floor at -45, the
// per-frame floors at the column maximum - 45 dB and the joint minimum are
// replayed to find the cells each selects; a floored cell passes its
// gradient to the cell that set its floor, and every cell's gradient flows
// (negated) to the joint minimum's cell. Reference cells are constants.
void prepare_grad(const double *ref_raw, const double *deg_raw, size_t nb, size_t nfr, size_t nfd,
                  const double *g_ref, const double *g_deg, double *g_deg_raw);

// prepareForComparison itself on copies (the forward values the reverse
// needs): prepared ref (nb x nfr) and deg (nb x nfd).
void prepare_forward(const double *ref_raw, const double *deg_raw, size_t nb, size_t nfr, size_t nfd,
                     std::vector<double> &ref, std::vector<double> &deg);

}  // namespace host
}  // namespace vqb
