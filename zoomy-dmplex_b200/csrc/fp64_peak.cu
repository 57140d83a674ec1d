// Measured FP64 arithmetic rate of a GPU (zsme_fp64_fma_peak).
//
// The step's face and finalize kernels are bound by FP64 arithmetic rather
// than by HBM, so their roofline needs the device's FP64 rate.  This entry
// point measures it instead of taking a data-sheet figure: every thread runs
// eight independent chains of fused multiply-adds (x = x * a + b, a < 1, so
// the values stay bounded), 256 threads per block and four blocks per SM,
// which gives each scheduler enough independent instructions to keep the
// FP64 pipe busy through its latency.  One FMA counts as two flops; the
// best of several launches, timed with CUDA events, is reported.
//
// The step's own kernels are compiled without FMA contraction (bit-identical
// rounding with the CPU restatement), so they issue one add or one multiply
// per FP64 instruction: their attainable rate is half of this figure.
#include <cuda_runtime.h>

#include <string>

#include "prepared_mesh.h"
#include "zsme.h"

namespace {

constexpr int kChains = 8;
constexpr int kThreads = 256;
constexpr int kBlocksPerSM = 4;
constexpr int kIters = 16384;
constexpr int kRuns = 5;

__global__ void __launch_bounds__(kThreads) fma_chains_kernel(double* sink, int iters, double a, double b) {
    double x[kChains];
#pragma unroll
    for (int k = 0; k < kChains; ++k) x[k] = 1e-3 * (threadIdx.x + k);
#pragma unroll 4
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < kChains; ++k) x[k] = __fma_rn(x[k], a, b);
    }
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < kChains; ++k) s += x[k];
    if (s < 0.0) sink[blockIdx.x] = s;   // never true (all terms positive); keeps the chains live
}

int cuda_fail(const char* what, cudaError_t e) {
    return zsme::set_error(ZSME_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

}  // namespace

extern "C" int zsme_fp64_fma_peak(int device, double* tflops) {
    if (!tflops) return zsme::set_error(ZSME_ERR_ARG, "null argument");
    int prev = 0;
    cudaError_t e = cudaGetDevice(&prev);
    if (e != cudaSuccess) return cuda_fail("cudaGetDevice", e);
    if ((e = cudaSetDevice(device)) != cudaSuccess) return cuda_fail("cudaSetDevice", e);
    int sms = 0;
    double* sink = nullptr;
    cudaStream_t s = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    double best = 0.0;
    int rc = ZSME_OK;
    do {
        if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device)) != cudaSuccess) {
            rc = cuda_fail("cudaDeviceGetAttribute", e);
            break;
        }
        const int blocks = sms * kBlocksPerSM;
        if ((e = cudaMalloc(&sink, sizeof(double) * blocks)) != cudaSuccess ||
            (e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking)) != cudaSuccess ||
            (e = cudaEventCreate(&e0)) != cudaSuccess || (e = cudaEventCreate(&e1)) != cudaSuccess) {
            rc = cuda_fail("setup", e);
            break;
        }
        const double flops = 2.0 * kChains * (double)kIters * kThreads * blocks;
        for (int r = 0; r <= kRuns; ++r) {   // run 0 warms up
            cudaEventRecord(e0, s);
            fma_chains_kernel<<<blocks, kThreads, 0, s>>>(sink, kIters, 0.999999, 1e-6);
            cudaEventRecord(e1, s);
            if ((e = cudaEventSynchronize(e1)) != cudaSuccess) {
                rc = cuda_fail("fma_chains_kernel", e);
                break;
            }
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, e0, e1);
            if (r > 0 && ms > 0.0f && flops / (ms * 1e9) > best) best = flops / (ms * 1e9);
        }
    } while (false);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (s) cudaStreamDestroy(s);
    if (sink) cudaFree(sink);
    cudaSetDevice(prev);
    if (rc == ZSME_OK) *tflops = best;
    return rc;
}
