// FP64 peak microbenchmarks: the denominators of the FP64 sigma kernels' roofline fractions.
//
// Two kernels, each timed alone with CUDA events on a private stream and no setting changed:
// * k_peak_dfma: 8 independent FMA chains per thread, 4 CTAs of 256 threads per SM (CUDA-core
//   FP64 pipe);
// * k_peak_dmma: 8 independent mma.sync m8n8k4 f64 accumulators per warp (FP64 tensor cores).
// The chains' results are written only under a condition that never holds for these inputs but
// that the compiler cannot prove, so no work is removed.
#include "fcib_internal.h"

namespace fcib {

__global__ void __launch_bounds__(256) k_peak_dfma(double* out, int iters, double seed) {
    double a[8];
#pragma unroll
    for (int j = 0; j < 8; j++) a[j] = seed * (threadIdx.x + 1) + j;
    const double m = 1.0 - 1e-12, c = 1e-9;
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int j = 0; j < 8; j++) a[j] = fma(a[j], m, c);
    }
    double s = 0.0;
#pragma unroll
    for (int j = 0; j < 8; j++) s += a[j];
    if (s == -1.0) out[0] = s;
}

__global__ void __launch_bounds__(256) k_peak_dmma(double* out, int iters, double seed) {
    double d[8][2];
#pragma unroll
    for (int j = 0; j < 8; j++) d[j][0] = d[j][1] = 0.0;
    const double a = seed * (threadIdx.x & 31), b = 1e-3 * seed;
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int j = 0; j < 8; j++)
            asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                : "+d"(d[j][0]), "+d"(d[j][1])
                : "d"(a), "d"(b));
    }
    double s = 0.0;
#pragma unroll
    for (int j = 0; j < 8; j++) s += d[j][0] + d[j][1];
    if (s == -1.0) out[0] = s;
}

}  // namespace fcib

// FP64 throughput of this GPU in TFLOP/s: dfma = CUDA-core FMA chains, dmma = FP64 tensor-core
// MMAs (2 flops per multiply-add).  Best of three timed launches each, after one warm-up launch.
// No counterpart in the reference (measurement only).
extern "C" int fcib_fp64_peak(int device, double* dfma_tflops, double* dmma_tflops) {
    using namespace fcib;
    try {
        FCIB_CUDA(cudaSetDevice(device));
        int sms = 0;
        FCIB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
        cudaStream_t st;
        FCIB_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        cudaEvent_t e0, e1;
        FCIB_CUDA(cudaEventCreate(&e0));
        FCIB_CUDA(cudaEventCreate(&e1));
        double* out = nullptr;
        const int grid = 4 * sms, threads = 256, iters = 1 << 16;
        auto best = [&](auto kern, double flop_per_iter_per_thread) {
            float bestms = 1e30f;
            for (int r = 0; r < 4; r++) {
                FCIB_CUDA(cudaEventRecord(e0, st));
                kern<<<grid, threads, 0, st>>>(out, iters, 1e-7);
                FCIB_KCHECK();
                FCIB_CUDA(cudaEventRecord(e1, st));
                FCIB_CUDA(cudaEventSynchronize(e1));
                float ms = 0.f;
                FCIB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
                if (r > 0) bestms = std::min(bestms, ms);
            }
            return flop_per_iter_per_thread * iters * (double)grid * threads / (bestms * 1e-3) / 1e12;
        };
        // DFMA: 8 FMAs (16 flops) per thread per iteration.  DMMA: 8 MMAs of 8x8x4 per warp per
        // iteration, 256 multiply-adds each: 8 * 512 / 32 = 128 flops per thread per iteration.
        const double f = best(k_peak_dfma, 16.0);
        const double m = best(k_peak_dmma, 128.0);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        cudaStreamDestroy(st);
        if (dfma_tflops) *dfma_tflops = f;
        if (dmma_tflops) *dmma_tflops = m;
        return FCIB_OK;
    } catch (const Error& e) {
        set_error(e.msg);
        return e.code;
    }
}
