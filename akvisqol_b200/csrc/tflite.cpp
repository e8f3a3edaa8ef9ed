// TFLite flatbuffer interpreter (tflite.h). The op semantics follow the
// TFLite builtin kernels as the reference restates them
// (src/tflite.zig:464-800): numpy-style broadcasting for element-wise ops,
// dot products as sequential f32 FMAs from zero, f32 -> i32 casts that
// truncate toward zero, concatenation and split along one axis.
#include "tflite.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>

#include "host_model.h"

namespace vqb {
namespace tfl {

namespace {

[[noreturn]] void bad(const std::string &what) { throw Error(kModel, "InvalidModel: " + what); }
[[noreturn]] void unsupported(const std::string &what) { throw Error(kModel, "UnsupportedOp: " + what); }

// ---- flatbuffer reading, every offset bounds-checked ----------------------
struct Buf {
    const uint8_t *p;
    size_t n;
    template <class T>
    T at(size_t pos) const {
        if (pos > n || n - pos < sizeof(T)) bad("offset out of range");
        T v;
        std::memcpy(&v, p + pos, sizeof(T));
        return v;
    }
};

struct Vec {
    const Buf *buf = nullptr;
    size_t start = 0, len = 0;
    bool present = false;
    template <class T>
    T item(size_t i) const { return buf->at<T>(start + sizeof(T) * i); }
};

struct Tab {
    const Buf *buf = nullptr;
    size_t pos = 0;
    // Absolute position of field id, or 0 when absent.
    size_t field(int id) const {
        const int64_t vt = (int64_t)pos - (int64_t)buf->at<int32_t>(pos);
        if (vt < 0) bad("vtable before buffer");
        const uint16_t vt_size = buf->at<uint16_t>((size_t)vt);
        const size_t slot = 4 + 2 * (size_t)id;
        if (slot + 2 > vt_size) return 0;
        const uint16_t off = buf->at<uint16_t>((size_t)vt + slot);
        return off ? pos + off : 0;
    }
    template <class T>
    T get(int id, T dflt) const {
        const size_t f = field(id);
        return f ? buf->at<T>(f) : dflt;
    }
    Tab table(int id) const {
        const size_t f = field(id);
        if (!f) return Tab{};
        return Tab{buf, f + buf->at<uint32_t>(f)};
    }
    Vec vec(int id) const {
        const size_t f = field(id);
        if (!f) return Vec{};
        const size_t v = f + buf->at<uint32_t>(f);
        const size_t len = buf->at<uint32_t>(v);
        return Vec{buf, v + 4, len, true};
    }
    std::string str(int id) const {
        const Vec v = vec(id);
        if (!v.present) return {};
        if (v.start > buf->n || buf->n - v.start < v.len) bad("string out of range");
        return std::string(reinterpret_cast<const char *>(buf->p + v.start), v.len);
    }
    bool ok() const { return buf != nullptr; }
};

Tab table_at(const Vec &v, size_t i) {
    const size_t slot = v.start + 4 * i;
    return Tab{v.buf, slot + v.buf->at<uint32_t>(slot)};
}

// builtin operator codes used by the lattice model
enum Kind : int {
    kAdd = 0, kConcat = 2, kFullyConnected = 9, kMul = 18, kRelu = 19, kRelu6 = 21, kReshape = 22, kSub = 41,
    kSplit = 49, kCast = 53, kMaximum = 55, kMinimum = 57, kExpandDims = 70, kEqual = 71, kShapeOp = 77,
    kFill = 94, kAbs = 101, kBatchMatmul = 126,
};

bool supported(int k) {
    switch (k) {
        case kAdd: case kConcat: case kFullyConnected: case kMul: case kRelu: case kRelu6: case kReshape:
        case kSub: case kSplit: case kCast: case kMaximum: case kMinimum: case kExpandDims: case kEqual:
        case kShapeOp: case kFill: case kAbs: case kBatchMatmul:
            return true;
        default:
            return false;
    }
}

int dtype_of(int8_t t) {
    switch (t) {
        case 0: return (int)DType::F32;
        case 2: return (int)DType::I32;
        case 6: return (int)DType::Bool;
        default: return -1;
    }
}

float activate(int act, float x) {
    switch (act) {
        case 1: return std::fmax(x, 0.0f);
        case 2: return std::fmax(-1.0f, std::fmin(x, 1.0f));
        case 3: return std::fmax(0.0f, std::fmin(x, 6.0f));
        default: return x;
    }
}

// ---- broadcasting -----------------------------------------------------------
Shape broadcast_shape(const Shape &x, const Shape &y) {
    Shape o;
    o.rank = std::max(x.rank, y.rank);
    for (int k = 0; k < o.rank; ++k) {
        const int64_t dx = k + x.rank >= o.rank ? x.dim[k + x.rank - o.rank] : 1;
        const int64_t dy = k + y.rank >= o.rank ? y.dim[k + y.rank - o.rank] : 1;
        if (dx != dy && dx != 1 && dy != 1) throw Error(kModel, "ShapeMismatch: broadcast");
        o.dim[k] = dx == 1 ? dy : dx;
    }
    return o;
}

// Element offsets of x and y for every element of the broadcast shape o,
// in row-major order of o.
template <class F>
void for_broadcast(const Shape &o, const Shape &x, const Shape &y, F &&fn) {
    int64_t sx[kMaxRank] = {}, sy[kMaxRank] = {};
    auto strides = [&](const Shape &s, int64_t *st) {
        int64_t acc = 1;
        for (int k = s.rank - 1; k >= 0; --k) {
            st[k + o.rank - s.rank] = s.dim[k] == 1 ? 0 : acc;
            acc *= s.dim[k];
        }
    };
    strides(x, sx);
    strides(y, sy);
    int64_t idx[kMaxRank] = {};
    int64_t ix = 0, iy = 0;
    const int64_t n = o.count();
    for (int64_t i = 0; i < n; ++i) {
        fn(i, ix, iy);
        for (int k = o.rank - 1; k >= 0; --k) {
            ++idx[k];
            ix += sx[k];
            iy += sy[k];
            if (idx[k] < o.dim[k]) break;
            ix -= sx[k] * o.dim[k];
            iy -= sy[k] * o.dim[k];
            idx[k] = 0;
        }
    }
}

const std::vector<float> &floats(const Value &v) {
    if (v.type != DType::F32) throw Error(kModel, "UnsupportedType: expected f32");
    return v.f;
}
const std::vector<int32_t> &ints(const Value &v) {
    if (v.type != DType::I32) throw Error(kModel, "UnsupportedType: expected i32");
    return v.i;
}
int32_t scalar_axis(const Value &v) {
    const auto &d = ints(v);
    if (d.size() != 1) throw Error(kModel, "ShapeMismatch: axis");
    return d[0];
}
int norm_axis(int axis, int rank) {
    const int ax = axis < 0 ? axis + rank : axis;
    if (ax < 0 || ax >= rank) throw Error(kModel, "ShapeMismatch: axis");
    return ax;
}

float dot(const float *x, const float *w, int64_t n) {
    float acc = 0.0f;
    for (int64_t k = 0; k < n; ++k) acc = std::fmaf(x[k], w[k], acc);
    return acc;
}

}  // namespace

int64_t Shape::count() const {
    int64_t n = 1;
    for (int k = 0; k < rank; ++k) n *= dim[k];
    return n;
}

Shape Shape::of(std::initializer_list<int64_t> dims) {
    Shape s;
    for (int64_t d : dims) {
        if (s.rank == kMaxRank) throw Error(kModel, "UnsupportedType: rank");
        s.dim[s.rank++] = d;
    }
    return s;
}

Model::Model(const std::string &bytes) {
    const Buf buf{reinterpret_cast<const uint8_t *>(bytes.data()), bytes.size()};
    const Tab root{&buf, buf.at<uint32_t>(0)};
    const Vec codes = root.vec(1), subgraphs = root.vec(2), buffers = root.vec(4);
    if (!codes.present || !subgraphs.present || !buffers.present || subgraphs.len < 1) bad("missing tables");
    const Tab g = table_at(subgraphs, 0);

    std::vector<int> kinds(codes.len);
    for (size_t i = 0; i < codes.len; ++i) {
        const Tab c = table_at(codes, i);
        if (c.field(1)) unsupported("custom operator");
        kinds[i] = std::max<int>(c.get<int8_t>(0, 0), c.get<int32_t>(3, 0));
    }

    const Vec tensors = g.vec(0);
    if (!tensors.present) bad("no tensors");
    const size_t nt = tensors.len;
    std::vector<std::string> names(nt);
    dtype_.assign(nt, -1);
    const_of_.assign(nt, -1);
    for (size_t t = 0; t < nt; ++t) {
        const Tab tt = table_at(tensors, t);
        names[t] = tt.str(3);
        dtype_[t] = dtype_of(tt.get<int8_t>(1, 0));
        const uint32_t bi = tt.get<uint32_t>(2, 0);
        if (bi == 0 || bi >= buffers.len) continue;
        const Tab b = table_at(buffers, bi);
        const uint8_t *data = nullptr;
        size_t size = 0;
        const Vec dv = b.vec(0);
        if (dv.present && dv.len) {
            if (dv.start > buf.n || buf.n - dv.start < dv.len) bad("buffer out of range");
            data = buf.p + dv.start;
            size = dv.len;
        } else {
            // weights stored after the flatbuffer (models over 2 GB)
            const uint64_t off = b.get<uint64_t>(1, 0), sz = b.get<uint64_t>(2, 0);
            if (off > 1 && sz > 0) {
                if (off > buf.n || buf.n - off < sz) bad("external buffer out of range");
                data = buf.p + off;
                size = sz;
            }
        }
        if (!size) continue;
        Value v;
        const Vec sv = tt.vec(0);
        if (sv.len > (size_t)kMaxRank) throw Error(kModel, "UnsupportedType: rank");
        v.shape.rank = (int)sv.len;
        for (size_t d = 0; d < sv.len; ++d) {
            const int32_t x = sv.item<int32_t>(d);
            if (x < 0) bad("negative dimension");
            v.shape.dim[d] = x;
        }
        const int64_t n = v.shape.count();
        if (dtype_[t] < 0) throw Error(kModel, "UnsupportedType: tensor type");
        v.type = (DType)dtype_[t];
        if (v.type == DType::F32) {
            if (size != (size_t)n * 4) bad("f32 buffer size");
            v.f.resize(n);
            std::memcpy(v.f.data(), data, size);
        } else if (v.type == DType::I32) {
            if (size != (size_t)n * 4) bad("i32 buffer size");
            v.i.resize(n);
            std::memcpy(v.i.data(), data, size);
        } else {
            if (size != (size_t)n) bad("bool buffer size");
            v.b.resize(n);
            for (int64_t k = 0; k < n; ++k) v.b[k] = data[k] != 0;
        }
        const_of_[t] = (int)consts_.size();
        consts_.push_back(std::move(v));
    }

    auto tensor_list = [&](const Vec &v) {
        std::vector<int> out;
        if (!v.present) return out;
        for (size_t k = 0; k < v.len; ++k) {
            const int32_t x = v.item<int32_t>(k);
            if (x >= (int64_t)nt) bad("tensor index");
            out.push_back(x);
        }
        return out;
    };
    auto act_of = [](int8_t code) {
        if (code < 0 || code > 3) unsupported("fused activation " + std::to_string(code));
        return (int)code;
    };
    const Vec opsv = g.vec(3);
    if (!opsv.present) bad("no operators");
    ops_.resize(opsv.len);
    for (size_t i = 0; i < opsv.len; ++i) {
        const Tab t = table_at(opsv, i);
        const uint32_t ci = t.get<uint32_t>(0, 0);
        if (ci >= kinds.size()) bad("opcode index");
        Op &op = ops_[i];
        op.kind = kinds[ci];
        if (!supported(op.kind)) unsupported("builtin " + std::to_string(op.kind));
        op.in = tensor_list(t.vec(1));
        op.out = tensor_list(t.vec(2));
        if (op.out.empty()) bad("operator without outputs");
        for (int o : op.out)
            if (o < 0) bad("negative output");
        const Tab o = t.table(4);
        if (!o.ok()) continue;
        switch (op.kind) {
            case kAdd: case kSub: case kMul:
                op.act = act_of(o.get<int8_t>(0, 0));
                break;
            case kConcat:
                op.axis = o.get<int32_t>(0, 0);
                op.act = act_of(o.get<int8_t>(1, 0));
                break;
            case kFullyConnected:
                op.act = act_of(o.get<int8_t>(0, 0));
                if (o.get<int8_t>(1, 0) != 0) unsupported("shuffled fully-connected weights");
                op.keep_num_dims = o.get<uint8_t>(2, 0) != 0;
                break;
            case kBatchMatmul:
                op.adj_x = o.get<uint8_t>(0, 0) != 0;
                op.adj_y = o.get<uint8_t>(1, 0) != 0;
                break;
            case kReshape: {
                const Vec ns = o.vec(0);
                if (ns.present) {
                    op.has_new_shape = true;
                    for (size_t k = 0; k < ns.len; ++k) op.new_shape.push_back(ns.item<int32_t>(k));
                }
                break;
            }
            default:
                break;
        }
    }

    // Named inputs and outputs: the "predict" signature (or the only one),
    // else the subgraph's own, under their tensor names.
    const Vec sigs = root.vec(7);
    if (sigs.present) {
        for (size_t i = 0; i < sigs.len; ++i) {
            const Tab s = table_at(sigs, i);
            if (s.str(2) != "predict" && sigs.len > 1) continue;
            if (s.get<uint32_t>(4, 0) != 0) unsupported("signature on another subgraph");
            auto maps = [&](const Vec &v, std::vector<std::pair<std::string, int>> &dst) {
                if (!v.present) return;
                for (size_t k = 0; k < v.len; ++k) {
                    const Tab m = table_at(v, k);
                    const uint32_t ti = m.get<uint32_t>(1, 0);
                    if (ti >= nt) bad("signature tensor index");
                    dst.emplace_back(m.str(0), (int)ti);
                }
            };
            maps(s.vec(0), inputs_);
            maps(s.vec(1), outputs_);
            break;
        }
    }
    if (inputs_.empty()) {
        for (int t : tensor_list(g.vec(1))) inputs_.emplace_back(names.at(t), t);
        for (int t : tensor_list(g.vec(2))) outputs_.emplace_back(names.at(t), t);
    }
}

int Model::input(const std::string &name) const {
    for (const auto &p : inputs_)
        if (p.first == name) return p.second;
    return -1;
}

int Model::output(const std::string &name) const {
    for (const auto &p : outputs_)
        if (p.first == name) return p.second;
    return -1;
}

Value Model::run(const std::vector<std::pair<int, Value>> &feeds, int out) const {
    Workspace ws;
    return run(feeds, out, ws);
}

const Value &Model::run(const std::vector<std::pair<int, Value>> &feeds, int out, Workspace &ws) const {
    const size_t nt = dtype_.size();
    std::vector<Value> &live = ws.live;
    std::vector<uint8_t> &have = ws.have;
    live.resize(nt);
    have.assign(nt, 0);
    for (const auto &f : feeds) {
        if (f.first < 0 || (size_t)f.first >= nt) bad("feed tensor index");
        live[f.first] = f.second;
        have[f.first] = 1;
    }
    auto get = [&](const Op &op, size_t k) -> const Value & {
        if (k >= op.in.size() || op.in[k] < 0) bad("missing operand");
        const int t = op.in[k];
        if (have[t]) return live[t];
        if (const_of_[t] >= 0) return consts_[const_of_[t]];
        bad("operand not computed");
    };
    auto opt = [&](const Op &op, size_t k) -> const Value * {
        if (k >= op.in.size() || op.in[k] < 0) return nullptr;
        return &get(op, k);
    };

    for (const Op &op : ops_) {
        const int o0 = op.out[0];
        for (int o : op.out)
            for (int t : op.in)
                if (o == t) bad("operator writes its own input");
        Value &r = live[o0];
        r.type = DType::F32;
        r.shape = Shape{};
        switch (op.kind) {
            case kAdd: case kSub: case kMul: case kMinimum: case kMaximum: {
                const Value &x = get(op, 0), &y = get(op, 1);
                const auto &xs = floats(x), &ys = floats(y);
                r.shape = broadcast_shape(x.shape, y.shape);
                r.f.resize(r.shape.count());
                const int kind = op.kind, act = op.act;
                for_broadcast(r.shape, x.shape, y.shape, [&](int64_t i, int64_t ix, int64_t iy) {
                    const float p = xs[ix], q = ys[iy];
                    float v;
                    switch (kind) {
                        case kAdd: v = p + q; break;
                        case kSub: v = p - q; break;
                        case kMul: v = p * q; break;
                        case kMinimum: v = std::fmin(p, q); break;
                        default: v = std::fmax(p, q); break;
                    }
                    r.f[i] = activate(act, v);
                });
                break;
            }
            case kEqual: {
                const Value &x = get(op, 0), &y = get(op, 1);
                if (x.type != y.type || x.type == DType::Bool) throw Error(kModel, "UnsupportedType: equal");
                r.type = DType::Bool;
                r.shape = broadcast_shape(x.shape, y.shape);
                r.b.resize(r.shape.count());
                for_broadcast(r.shape, x.shape, y.shape, [&](int64_t i, int64_t ix, int64_t iy) {
                    r.b[i] = x.type == DType::F32 ? x.f[ix] == y.f[iy] : x.i[ix] == y.i[iy];
                });
                break;
            }
            case kRelu: case kRelu6: case kAbs: {
                const Value &x = get(op, 0);
                const auto &xs = floats(x);
                r.shape = x.shape;
                r.f.resize(xs.size());
                for (size_t k = 0; k < xs.size(); ++k)
                    r.f[k] = op.kind == kAbs ? std::fabs(xs[k]) : activate(op.kind == kRelu ? 1 : 3, xs[k]);
                break;
            }
            case kCast: {
                const Value &x = get(op, 0);
                if (dtype_[o0] < 0) throw Error(kModel, "UnsupportedType: cast target");
                r.type = (DType)dtype_[o0];
                r.shape = x.shape;
                const int64_t n = x.shape.count();
                auto src = [&](int64_t k) -> double {
                    return x.type == DType::F32 ? (double)x.f[k] : x.type == DType::I32 ? (double)x.i[k] : (double)x.b[k];
                };
                if (r.type == DType::F32) {
                    r.f.resize(n);
                    for (int64_t k = 0; k < n; ++k)
                        r.f[k] = x.type == DType::F32 ? x.f[k] : x.type == DType::I32 ? (float)x.i[k] : (x.b[k] ? 1.f : 0.f);
                } else if (r.type == DType::I32) {
                    r.i.resize(n);
                    for (int64_t k = 0; k < n; ++k) {
                        // toward zero, saturating (TFLite's static_cast on representable values)
                        const double v = std::trunc(src(k));
                        r.i[k] = v >= 2147483647.0 ? std::numeric_limits<int32_t>::max()
                                 : v <= -2147483648.0 ? std::numeric_limits<int32_t>::min()
                                 : std::isnan(v) ? 0 : (int32_t)v;
                    }
                } else {
                    r.b.resize(n);
                    for (int64_t k = 0; k < n; ++k) r.b[k] = src(k) != 0.0;
                }
                break;
            }
            case kConcat: {
                const Value &first = get(op, 0);
                const int ax = norm_axis(op.axis, first.shape.rank);
                r.shape = first.shape;
                r.shape.dim[ax] = 0;
                for (size_t k = 0; k < op.in.size(); ++k) {
                    const Value &v = get(op, k);
                    if (v.shape.rank != r.shape.rank) throw Error(kModel, "ShapeMismatch: concat rank");
                    for (int d = 0; d < r.shape.rank; ++d)
                        if (d != ax && v.shape.dim[d] != first.shape.dim[d]) throw Error(kModel, "ShapeMismatch: concat");
                    r.shape.dim[ax] += v.shape.dim[ax];
                }
                int64_t outer = 1, inner = 1;
                for (int d = 0; d < ax; ++d) outer *= r.shape.dim[d];
                for (int d = ax + 1; d < r.shape.rank; ++d) inner *= r.shape.dim[d];
                r.f.clear();
                r.f.reserve(r.shape.count());
                for (int64_t o = 0; o < outer; ++o)
                    for (size_t k = 0; k < op.in.size(); ++k) {
                        const Value &v = get(op, k);
                        const auto &xs = floats(v);
                        const int64_t chunk = v.shape.dim[ax] * inner;
                        for (int64_t e = 0; e < chunk; ++e) r.f.push_back(activate(op.act, xs[o * chunk + e]));
                    }
                break;
            }
            case kFullyConnected: {
                const Value &x = get(op, 0), &w = get(op, 1);
                const Value *bias = opt(op, 2);
                const auto &xs = floats(x), &ws = floats(w);
                if (w.shape.rank != 2) throw Error(kModel, "ShapeMismatch: fully-connected weights");
                const int64_t n_out = w.shape.dim[0], n_in = w.shape.dim[1];
                if (n_in == 0 || (int64_t)xs.size() % n_in) throw Error(kModel, "ShapeMismatch: fully-connected");
                const int64_t batch = (int64_t)xs.size() / n_in;
                if (bias && (int64_t)floats(*bias).size() != n_out) throw Error(kModel, "ShapeMismatch: bias");
                r.f.resize(batch * n_out);
                for (int64_t row = 0; row < batch; ++row)
                    for (int64_t o = 0; o < n_out; ++o) {
                        float y = dot(xs.data() + row * n_in, ws.data() + o * n_in, n_in);
                        if (bias) y += bias->f[o];
                        r.f[row * n_out + o] = activate(op.act, y);
                    }
                if (op.keep_num_dims) {
                    r.shape = x.shape;
                    r.shape.dim[r.shape.rank - 1] = n_out;
                } else {
                    r.shape = Shape::of({batch, n_out});
                }
                break;
            }
            case kBatchMatmul: {
                const Value &x = get(op, 0), &y = get(op, 1);
                const auto &xs = floats(x), &ys = floats(y);
                const int xr = x.shape.rank, yr = y.shape.rank;
                if (xr < 2 || yr < 2) throw Error(kModel, "ShapeMismatch: batch matmul rank");
                const int64_t m = op.adj_x ? x.shape.dim[xr - 1] : x.shape.dim[xr - 2];
                const int64_t k = op.adj_x ? x.shape.dim[xr - 2] : x.shape.dim[xr - 1];
                const int64_t k2 = op.adj_y ? y.shape.dim[yr - 1] : y.shape.dim[yr - 2];
                const int64_t n = op.adj_y ? y.shape.dim[yr - 2] : y.shape.dim[yr - 1];
                if (k != k2) throw Error(kModel, "ShapeMismatch: batch matmul");
                Shape xb, yb;
                xb.rank = xr - 2;
                yb.rank = yr - 2;
                for (int d = 0; d < xb.rank; ++d) xb.dim[d] = x.shape.dim[d];
                for (int d = 0; d < yb.rank; ++d) yb.dim[d] = y.shape.dim[d];
                const Shape ob = broadcast_shape(xb, yb);
                r.f.resize(ob.count() * m * n);
                for_broadcast(ob, xb, yb, [&](int64_t bi, int64_t bx, int64_t by) {
                    const float *xm = xs.data() + bx * m * k, *ym = ys.data() + by * k * n;
                    float *om = r.f.data() + bi * m * n;
                    // Each output accumulates over l in order from zero; the
                    // outputs of a row advance together (vectorised over j).
                    for (int64_t i = 0; i < m; ++i) {
                        float *acc = om + i * n;
                        for (int64_t j = 0; j < n; ++j) acc[j] = 0.0f;
                        for (int64_t l = 0; l < k; ++l) {
                            const float p = op.adj_x ? xm[l * m + i] : xm[i * k + l];
                            if (!op.adj_y) {
                                const float *q = ym + l * n;
                                for (int64_t j = 0; j < n; ++j) acc[j] = std::fmaf(p, q[j], acc[j]);
                            } else {
                                for (int64_t j = 0; j < n; ++j) acc[j] = std::fmaf(p, ym[j * k + l], acc[j]);
                            }
                        }
                    }
                });
                if (ob.rank + 2 > kMaxRank) throw Error(kModel, "UnsupportedType: rank");
                r.shape = ob;
                r.shape.dim[r.shape.rank++] = m;
                r.shape.dim[r.shape.rank++] = n;
                break;
            }
            case kReshape: {
                const Value &x = get(op, 0);
                const Value *sv = opt(op, 1);
                if (!sv && !op.has_new_shape) bad("reshape without a shape");
                const std::vector<int32_t> spec = sv ? ints(*sv) : op.new_shape;
                if (spec.size() > (size_t)kMaxRank) throw Error(kModel, "UnsupportedType: rank");
                const int64_t total = x.shape.count();
                r = x;
                r.shape = Shape{};
                r.shape.rank = (int)spec.size();
                int64_t known = 1;
                int infer = -1;
                for (size_t d = 0; d < spec.size(); ++d) {
                    if (spec[d] == -1) {
                        if (infer >= 0) throw Error(kModel, "ShapeMismatch: reshape");
                        infer = (int)d;
                    } else if (spec[d] < 0) {
                        throw Error(kModel, "ShapeMismatch: reshape");
                    } else {
                        r.shape.dim[d] = spec[d];
                        known *= spec[d];
                    }
                }
                if (infer >= 0) {
                    if (known == 0 || total % known) throw Error(kModel, "ShapeMismatch: reshape");
                    r.shape.dim[infer] = total / known;
                }
                if (r.shape.count() != total) throw Error(kModel, "ShapeMismatch: reshape");
                break;
            }
            case kExpandDims: {
                const Value &x = get(op, 0);
                const int axis = scalar_axis(get(op, 1));
                const int rank = x.shape.rank;
                const int ax = axis < 0 ? axis + rank + 1 : axis;
                if (ax < 0 || ax > rank || rank >= kMaxRank) throw Error(kModel, "ShapeMismatch: expand_dims");
                r = x;
                r.shape.rank = rank + 1;
                for (int d = rank; d > ax; --d) r.shape.dim[d] = x.shape.dim[d - 1];
                r.shape.dim[ax] = 1;
                break;
            }
            case kShapeOp: {
                const Value &x = get(op, 0);
                r.type = DType::I32;
                r.shape = Shape::of({x.shape.rank});
                r.i.clear();
                for (int d = 0; d < x.shape.rank; ++d) r.i.push_back((int32_t)x.shape.dim[d]);
                break;
            }
            case kFill: {
                const auto &dims = ints(get(op, 0));
                const Value &v = get(op, 1);
                if (dims.size() > (size_t)kMaxRank) throw Error(kModel, "UnsupportedType: rank");
                r.type = v.type;
                r.shape.rank = (int)dims.size();
                for (size_t d = 0; d < dims.size(); ++d) {
                    if (dims[d] < 0) throw Error(kModel, "ShapeMismatch: fill");
                    r.shape.dim[d] = dims[d];
                }
                const int64_t n = r.shape.count();
                const size_t have_n = v.type == DType::F32 ? v.f.size() : v.type == DType::I32 ? v.i.size() : v.b.size();
                if (have_n != 1) throw Error(kModel, "ShapeMismatch: fill value");
                if (v.type == DType::F32) r.f.assign(n, v.f[0]);
                if (v.type == DType::I32) r.i.assign(n, v.i[0]);
                if (v.type == DType::Bool) r.b.assign(n, v.b[0]);
                break;
            }
            case kSplit: {
                const int axis = scalar_axis(get(op, 0));
                const Value &x = get(op, 1);
                const auto &xs = floats(x);
                const int ax = norm_axis(axis, x.shape.rank);
                const int64_t parts = (int64_t)op.out.size();
                if (x.shape.dim[ax] % parts) throw Error(kModel, "ShapeMismatch: split");
                Shape s = x.shape;
                s.dim[ax] /= parts;
                int64_t outer = 1, inner = 1;
                for (int d = 0; d < ax; ++d) outer *= x.shape.dim[d];
                for (int d = ax + 1; d < x.shape.rank; ++d) inner *= x.shape.dim[d];
                const int64_t chunk = s.dim[ax] * inner;
                for (int64_t p = 0; p < parts; ++p) {
                    Value &v = live[op.out[p]];
                    v.type = DType::F32;
                    v.shape = s;
                    v.f.resize(outer * chunk);
                    for (int64_t o = 0; o < outer; ++o)
                        std::copy(xs.begin() + (o * parts + p) * chunk, xs.begin() + (o * parts + p + 1) * chunk,
                                  v.f.begin() + o * chunk);
                    have[op.out[p]] = 1;
                }
                continue;
            }
            default:
                unsupported("builtin " + std::to_string(op.kind));
        }
        have[o0] = 1;
    }
    if (out < 0 || (size_t)out >= nt || !have[out]) bad("output not computed");
    return live[out];
}

}  // namespace tfl
}  // namespace vqb
