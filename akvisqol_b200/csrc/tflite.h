// A small TFLite flatbuffer interpreter for the speech-mode lattice MOS model
// (the reference's src/tflite.zig covers the same op set). Host-side f32:
// the model maps 4 x 21 per-band features to one MOS per pair.
#pragma once

#include <cstdint>
#include <string>
#include <utility>
#include <vector>

namespace vqb {
namespace tfl {

enum class DType : uint8_t { F32, I32, Bool };

constexpr int kMaxRank = 6;

struct Shape {
    int rank = 0;
    int64_t dim[kMaxRank] = {};
    int64_t count() const;
    static Shape of(std::initializer_list<int64_t> dims);
};

// A tensor value: data in the vector that matches `type`.
struct Value {
    DType type = DType::F32;
    Shape shape;
    std::vector<float> f;
    std::vector<int32_t> i;
    std::vector<uint8_t> b;
};

// Loads a .tflite flatbuffer (first subgraph) and runs it on the CPU. Custom
// ops and builtin ops outside the supported set fail at load. Weights are
// copied; the bytes need not outlive the model. run() is const and
// thread-safe.
class Model {
public:
    explicit Model(const std::string &bytes);
    int input(const std::string &name) const;   // tensor index, -1 if absent
    int output(const std::string &name) const;  // tensor index, -1 if absent
    // Per-thread scratch reused across runs (tensor storage keeps its
    // capacity, so a warm run allocates nothing).
    struct Workspace {
        std::vector<Value> live;
        std::vector<uint8_t> have;
    };
    Value run(const std::vector<std::pair<int, Value>> &feeds, int out) const;
    const Value &run(const std::vector<std::pair<int, Value>> &feeds, int out, Workspace &ws) const;

    struct Op {
        int kind = 0;
        std::vector<int> in, out;
        int act = 0;
        int axis = 0;
        bool adj_x = false, adj_y = false, keep_num_dims = false;
        bool has_new_shape = false;
        std::vector<int32_t> new_shape;
    };

private:
    std::vector<int> dtype_;             // per tensor: DType as int, -1 unsupported
    std::vector<int> const_of_;          // per tensor: index into consts_, -1 if not constant
    std::vector<Value> consts_;
    std::vector<Op> ops_;
    std::vector<std::pair<std::string, int>> inputs_, outputs_;
};

}  // namespace tfl
}  // namespace vqb
