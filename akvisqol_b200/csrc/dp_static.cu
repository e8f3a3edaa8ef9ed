// visqol_b200_dp_static: the patch-alignment DP and backtrack of
// visqol_b200_dp (reference src/dp.zig:216-352), with every device buffer
// carved from one fixed array that the library image reserves at module
// load. The call allocates no device memory.
//
// Who needs it: a caller whose process already hands all free HBM to a
// caching allocator (a serving process that reserved its memory up front,
// or a framework that owns the device), where a cudaMalloc can fail at call
// time; and a caller sharing the device with long-running streams, where
// cudaFree blocks until the whole device is idle. Both can call this entry
// point instead: its memory was reserved when the module was loaded.
//
// Limits: np * nf_deg <= kMaxCells (262,144) and np <= kMaxPatches (2048).
// A 10 s 48 kHz audio pair is 16 patches x 497 frames = 7,952 cells; the
// limit covers audio-mode pairs up to about 55 s. Larger tables are
// rejected with VISQOL_E_INVALID_ARGUMENT before any device work.
//
// Setup: the first call on a device, with that device current, resolves the
// array's device address (cudaGetSymbolAddress) and caches it per device.
// That first call must come before any stream capture the caller makes.
//
// Sharing: every call on a device uses the same array. Calls that overlap in
// time on one device (two host threads, say) race on it and must be
// serialised by the caller. Nothing in the array needs to start at zero:
// the DP kernel clears its dp and backtrack tables on entry, and the
// offsets and flags are written in full by the backtrack.
#include <mutex>

#include "../../include/visqol_b200.h"
#include "engine.h"
#include "kernels.h"

namespace {

constexpr size_t kMaxCells = size_t{1} << 18;  // np * nf_deg
constexpr size_t kMaxPatches = 2048;
constexpr size_t kMaxDevices = 64;

constexpr size_t align256(size_t n) { return (n + 255) & ~size_t{255}; }

// Byte offsets of the buffers inside the array.
constexpr size_t kJobAt = 0;
constexpr size_t kLoAt = align256(kJobAt + sizeof(vqb::DpJob));
constexpr size_t kHiAt = kLoAt + align256(kMaxPatches * sizeof(int64_t));
constexpr size_t kOffAt = kHiAt + align256(kMaxPatches * sizeof(int64_t));
constexpr size_t kValidAt = kOffAt + align256(kMaxPatches * sizeof(int64_t));
constexpr size_t kSimsAt = kValidAt + align256(kMaxPatches);
constexpr size_t kDpAt = kSimsAt + kMaxCells * sizeof(double);
constexpr size_t kBtAt = kDpAt + kMaxCells * sizeof(double);
constexpr size_t kScratchBytes = kBtAt + kMaxCells * sizeof(int64_t);  // ~6.05 MiB

static __device__ __align__(256) unsigned char g_dp_scratch[kScratchBytes];

std::mutex g_setup_mu;
unsigned char *g_scratch_ptr[kMaxDevices] = {};

int fail(int code, const char *m) {
    vqb::set_last_error(m);
    return code;
}

// Device address of g_dp_scratch on the current device, resolved once.
int scratch_for_current_device(unsigned char **out) {
    int dev = 0;
    cudaError_t rc = cudaGetDevice(&dev);
    if (rc != cudaSuccess) return fail(VISQOL_E_BACKEND, cudaGetErrorString(rc));
    if (dev < 0 || (size_t)dev >= kMaxDevices) return fail(VISQOL_E_BACKEND, "dp_static: device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_setup_mu);
    if (!g_scratch_ptr[dev]) {
        void *p = nullptr;
        rc = cudaGetSymbolAddress(&p, g_dp_scratch);
        if (rc != cudaSuccess || !p) return fail(VISQOL_E_BACKEND, cudaGetErrorString(rc));
        g_scratch_ptr[dev] = static_cast<unsigned char *>(p);
    }
    *out = g_scratch_ptr[dev];
    return VISQOL_OK;
}

int check(cudaError_t rc) {
    return rc == cudaSuccess ? VISQOL_OK : fail(VISQOL_E_BACKEND, cudaGetErrorString(rc));
}

}  // namespace

extern "C" int visqol_b200_dp_static(const double *sims, size_t np, size_t nf_deg, const int64_t *lo,
                                     const int64_t *hi, int64_t *offset, uint8_t *valid, size_t *reached) {
    if (!sims || !lo || !hi || !offset || !valid || np == 0 || nf_deg == 0)
        return fail(VISQOL_E_INVALID_ARGUMENT, "invalid argument");
    if (np > kMaxPatches || np > kMaxCells / nf_deg)
        return fail(VISQOL_E_INVALID_ARGUMENT,
                    "dp_static: table exceeds the static scratch (np <= 2048 and np * nf_deg <= 262144)");
    for (size_t p = 0; p < np; ++p)
        if (lo[p] < 0 || hi[p] < lo[p] || (size_t)hi[p] >= nf_deg || (p && lo[p] < lo[p - 1]))
            return fail(VISQOL_E_INVALID_ARGUMENT, "window out of range");

    unsigned char *base = nullptr;
    if (int rc = scratch_for_current_device(&base)) return rc;
    auto *d_job = reinterpret_cast<vqb::DpJob *>(base + kJobAt);
    auto *d_lo = reinterpret_cast<int64_t *>(base + kLoAt);
    auto *d_hi = reinterpret_cast<int64_t *>(base + kHiAt);
    auto *d_off = reinterpret_cast<int64_t *>(base + kOffAt);
    auto *d_valid = reinterpret_cast<uint8_t *>(base + kValidAt);
    auto *d_sims = reinterpret_cast<double *>(base + kSimsAt);
    auto *d_dp = reinterpret_cast<double *>(base + kDpAt);
    auto *d_bt = reinterpret_cast<int64_t *>(base + kBtAt);

    const cudaStream_t s = cudaStreamPerThread;
    const vqb::DpJob job{d_sims, d_lo, d_hi, (int32_t)np, (int64_t)nf_deg, d_dp, d_bt, d_off, d_valid};
    int rc = check(cudaMemcpyAsync(d_sims, sims, np * nf_deg * sizeof(double), cudaMemcpyHostToDevice, s));
    if (!rc) rc = check(cudaMemcpyAsync(d_lo, lo, np * sizeof(int64_t), cudaMemcpyHostToDevice, s));
    if (!rc) rc = check(cudaMemcpyAsync(d_hi, hi, np * sizeof(int64_t), cudaMemcpyHostToDevice, s));
    if (!rc) rc = check(cudaMemcpyAsync(d_job, &job, sizeof(job), cudaMemcpyHostToDevice, s));
    if (rc) return rc;
    vqb::launch_dp(d_job, 1, s);
    rc = check(cudaGetLastError());
    if (!rc) rc = check(cudaMemcpyAsync(offset, d_off, np * sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    if (!rc) rc = check(cudaMemcpyAsync(valid, d_valid, np, cudaMemcpyDeviceToHost, s));
    if (!rc) rc = check(cudaStreamSynchronize(s));
    if (rc) return rc;
    size_t r = 0;
    for (size_t p = 0; p < np; ++p) r += offset[p] >= 0;
    if (reached) *reached = r;
    return VISQOL_OK;
}
