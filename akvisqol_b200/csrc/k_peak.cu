// Arithmetic-pipe peaks of this GPU, for roofline fractions: independent
// multiply/add chains that keep every SM's FP64 (or FP32) pipe busy.
// kind 0: f64 multiply and add as separate instructions (the exact form's
//         arithmetic; one flop per instruction);
// kind 1: f64 fused multiply-add (two flops per instruction);
// kind 2: f32 fused multiply-add.
#include <cuda_runtime.h>

#include "../../include/visqol_b200.h"
#include "engine.h"
#include "kernels.h"

namespace {

constexpr int kChains = 8;
constexpr int kIters = 4096;

template <int KIND>
__global__ void __launch_bounds__(256) peak_kernel(float *sink, float seed) {
    if (KIND == 2) {
        float x[kChains];
#pragma unroll
        for (int c = 0; c < kChains; ++c) x[c] = seed + threadIdx.x * 1e-7f + c;
        const float m = 0.9999999f, a = 1e-7f;
        for (int i = 0; i < kIters; ++i) {
#pragma unroll
            for (int c = 0; c < kChains; ++c) x[c] = fmaf(x[c], m, a);
        }
        float s = 0;
#pragma unroll
        for (int c = 0; c < kChains; ++c) s += x[c];
        if (s == 12345.0f) sink[0] = s;
    } else {
        double x[kChains];
#pragma unroll
        for (int c = 0; c < kChains; ++c) x[c] = (double)seed + threadIdx.x * 1e-9 + c;
        const double m = 0.999999999, a = 1e-9;
        for (int i = 0; i < kIters; ++i) {
#pragma unroll
            for (int c = 0; c < kChains; ++c) {
                if (KIND == 1)
                    x[c] = fma(x[c], m, a);
                else
                    x[c] = __dadd_rn(__dmul_rn(x[c], m), a);
            }
        }
        double s = 0;
#pragma unroll
        for (int c = 0; c < kChains; ++c) s += x[c];
        if (s == 12345.0) sink[0] = (float)s;
    }
}

}  // namespace

extern "C" int visqol_b200_peak(int kind, double *tflops) {
    if (!tflops || kind < 0 || kind > 2) return VISQOL_E_INVALID_ARGUMENT;
    try {
        int dev = 0, sms = 0;
        VQB_CUDA(cudaGetDevice(&dev));
        VQB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        float *sink = nullptr;
        VQB_CUDA(cudaMalloc(&sink, sizeof(float)));
        cudaEvent_t a, b;
        VQB_CUDA(cudaEventCreate(&a));
        VQB_CUDA(cudaEventCreate(&b));
        const int blocks = sms * 8, threads = 256;
        double best = 0;
        for (int rep = 0; rep < 4; ++rep) {
            VQB_CUDA(cudaEventRecord(a));
            if (kind == 0) peak_kernel<0><<<blocks, threads>>>(sink, 1.0f);
            if (kind == 1) peak_kernel<1><<<blocks, threads>>>(sink, 1.0f);
            if (kind == 2) peak_kernel<2><<<blocks, threads>>>(sink, 1.0f);
            VQB_CUDA(cudaEventRecord(b));
            VQB_CUDA(cudaEventSynchronize(b));
            float ms = 0;
            VQB_CUDA(cudaEventElapsedTime(&ms, a, b));
            const double flops = (double)blocks * threads * kChains * kIters * 2.0;
            if (rep > 0) best = std::max(best, flops / (ms * 1e-3) / 1e12);
        }
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        cudaFree(sink);
        *tflops = best;
        return VISQOL_OK;
    } catch (const vqb::Error &e) {
        vqb::set_last_error(e.what());
        return e.code;
    }
}
