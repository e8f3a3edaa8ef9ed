// Pieces of the C ABI layer shared by capi.cpp and server.cpp.
#pragma once

#include <memory>
#include <string>

#include "../../include/visqol.h"
#include "engine.h"
#include "host_model.h"

namespace vqb {

// A heap-boxed visqol_result owning its arrays (freed by visqol_result_free).
visqol_result *box_result(host::Scores &&s);

// Checks visqol_options and turns them into engine options and the SVR
// model (audio mode); returns VISQOL_OK or an error code with *message.
// In speech mode with use_lattice_model, *lattice gets the TF-Lattice
// mapper (model_path's .tflite file, or the bundled model).
int engine_options(const visqol_options &o, Options *opt, std::shared_ptr<const host::Svr> *svr,
                   std::shared_ptr<const host::LatticeMapper> *lattice, std::string *message);

// The device of new contexts and servers (VISQOL_CUDA_DEVICE, default 0),
// or an error code with *message.
int context_device(int *device, std::string *message);

// Number of lanes asked for by VISQOL_GPU_LANES (1-8, default fallback).
int env_lanes(int fallback);

// Whether host-input batches overlap their uploads with scoring
// (Engine::measure_batch_streamed); VISQOL_STREAMED_UPLOADS=0 turns it off.
bool env_streamed_uploads();

}  // namespace vqb
