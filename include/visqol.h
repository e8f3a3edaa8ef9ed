/* ViSQOL C ABI, served by akvisqol_b200's libvisqol.so (backend CUDA on a
 * B200, sm_100a).
 *
 * This is the drop-in boundary: the declarations, types, enum values and
 * error codes are those of the reference's C ABI (jdek/akvisqol
 * src/include/visqol.h:1-129, implemented by src/capi.zig:119-456), so its
 * Python package (src/python/visqol/_native.py:83-134, via VISQOL_LIBRARY),
 * its C++ compat layer and any Zig host that links libvisqol load this
 * library unchanged. Each declaration cites the reference line it replaces.
 *
 * Calls return VISQOL_OK (0) or a negative code; visqol_last_error() holds
 * the calling thread's last message. One visqol_ctx is used by one thread
 * at a time; visqol_measure_batch batches all pairs on the GPU.
 *
 * Backends: this library serves VISQOL_BACKEND_CUDA only. Asking it for
 * CPU, Metal or Vulkan fails with VISQOL_E_BACKEND, and there is no CPU
 * fallback. visqol_options_default selects CUDA.
 */
#ifndef VISQOL_H
#define VISQOL_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VISQOL_ABI_VERSION 1

/* Error codes (reference visqol.h:20-29). */
enum {
    VISQOL_OK = 0,
    VISQOL_E_INVALID_ARGUMENT = -1,
    VISQOL_E_OUT_OF_MEMORY = -2,
    VISQOL_E_IO = -3,
    VISQOL_E_MODEL = -4,
    VISQOL_E_SIGNAL = -5,
    VISQOL_E_BACKEND = -6,
    VISQOL_E_INTERNAL = -7,
};

/* Modes (reference visqol.h:31). */
enum { VISQOL_MODE_AUDIO = 0, VISQOL_MODE_SPEECH = 1 };

/* Backends (reference visqol.h:33-38). */
enum {
    VISQOL_BACKEND_CPU = 0,
    VISQOL_BACKEND_METAL = 1,
    VISQOL_BACKEND_CUDA = 2,
    VISQOL_BACKEND_VULKAN = 3,
};

/* Precision forms (reference visqol.h:40-43). EXACT: f64, the reference
 * CPU model's scores to 1e-12 with identical lags. FAST: f32 with
 * compensated low bands. AUTO: EXACT. */
enum {
    VISQOL_PRECISION_EXACT = 0,
    VISQOL_PRECISION_FAST = 1,
    VISQOL_PRECISION_BALANCED = 2,
    VISQOL_PRECISION_AUTO = 3
};

/* Options (reference visqol.h:45-57). */
typedef struct {
    uint32_t mode;
    int32_t search_window_radius;        /* <= 0 means 60 */
    uint8_t use_unscaled_speech_mos_mapping;
    uint8_t disable_global_alignment;
    uint8_t disable_realignment;
    uint8_t use_lattice_model;
    const char *model_path;              /* NULL or "": the bundled SVR model */
    uint32_t backend;
    uint32_t precision;
} visqol_options;

/* One matched patch (reference visqol.h:59-68). */
typedef struct {
    double similarity;
    double ref_patch_start_time;
    double ref_patch_end_time;
    double deg_patch_start_time;
    double deg_patch_end_time;
    const double *freq_band_means;       /* num_bands values each */
    const double *freq_band_stddevs;
    const double *freq_band_deg_energy;
} visqol_patch;

/* Scores of one pair (reference visqol.h:70-82). */
typedef struct {
    double moslqo;
    double vnsim;
    double alignment_lag_s;
    size_t num_bands;
    const double *fvnsim;
    const double *fvnsim10;
    const double *fstdnsim;
    const double *fvdegenergy;
    const double *center_freq_bands;
    size_t num_patches;
    const visqol_patch *patch_sims;
} visqol_result;

typedef struct visqol_ctx visqol_ctx;

/* reference visqol.h:86-90 */
uint32_t visqol_abi_version(void);
const char *visqol_version(void);
const char *visqol_last_error(void);
uint32_t visqol_available_backends(void);

/* reference visqol.h:92 */
void visqol_options_default(visqol_options *opts);

/* reference visqol.h:94-95 */
int visqol_create(const visqol_options *opts, visqol_ctx **out);
void visqol_destroy(visqol_ctx *ctx);

/* reference visqol.h:97-102 */
int visqol_measure(visqol_ctx *ctx,
                   const double *ref, size_t ref_len,
                   const double *deg, size_t deg_len,
                   uint32_t sample_rate,
                   visqol_result **out);

/* reference visqol.h:104-106 */
int visqol_measure_files(visqol_ctx *ctx, const char *ref_path,
                         const char *deg_path, visqol_result **out);

/* reference visqol.h:108-114. num_threads is accepted for compatibility;
 * the pairs are batched on the GPU, host planning uses up to that many
 * threads (0: all cores). */
int visqol_measure_batch(visqol_ctx *ctx, size_t n,
                         const double *const *refs, const size_t *ref_lens,
                         const double *const *degs, const size_t *deg_lens,
                         uint32_t sample_rate, uint32_t num_threads,
                         visqol_result **out, int32_t *status);

/* reference visqol.h:116-121 */
int visqol_measure_files_batch(visqol_ctx *ctx, size_t n,
                               const char *const *ref_paths,
                               const char *const *deg_paths,
                               uint32_t num_threads,
                               visqol_result **out, int32_t *status);

/* reference visqol.h:123 */
void visqol_result_free(visqol_result *result);

#ifdef __cplusplus
}
#endif

#endif /* VISQOL_H */
