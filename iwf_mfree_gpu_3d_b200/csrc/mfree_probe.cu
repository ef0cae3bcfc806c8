// mfree_probe.cu -- measurement helper: sustained FP32 FMA throughput of the
// device, the denominator of the pair kernel's roofline (the pair loop is
// bound by the FP32 pipe, not by HBM or tensor cores).
#include "mfree_kernels.cuh"

namespace mfree {

// 8 independent FMA chains per thread, ITER iterations: 2*8*ITER flops/thread
template <int ITER>
__global__ void __launch_bounds__(256) k_fma_probe(float *out, float a, float b) {
    float x0 = threadIdx.x * 1e-7f, x1 = x0 + 1e-7f, x2 = x0 + 2e-7f, x3 = x0 + 3e-7f;
    float x4 = x0 + 4e-7f, x5 = x0 + 5e-7f, x6 = x0 + 6e-7f, x7 = x0 + 7e-7f;
#pragma unroll 16
    for (int k = 0; k < ITER; k++) {
        x0 = fmaf(x0, a, b); x1 = fmaf(x1, a, b); x2 = fmaf(x2, a, b); x3 = fmaf(x3, a, b);
        x4 = fmaf(x4, a, b); x5 = fmaf(x5, a, b); x6 = fmaf(x6, a, b); x7 = fmaf(x7, a, b);
    }
    const float s = ((x0 + x1) + (x2 + x3)) + ((x4 + x5) + (x6 + x7));
    if (s == 1234.5678f) out[blockIdx.x] = s;  // keeps the chains alive
}

double fp32_peak_probe(int num_sms) {
    constexpr int ITER = 4096;
    float *d = nullptr;
    if (cudaMalloc(&d, 4096 * sizeof(float)) != cudaSuccess) return -1.0;
    const int blocks = num_sms * 8;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    k_fma_probe<ITER><<<blocks, 256>>>(d, 0.999999f, 1e-7f);  // warm up (clocks)
    float best = 1e30f;
    for (int r = 0; r < 5; r++) {
        cudaEventRecord(e0);
        for (int k = 0; k < 8; k++) k_fma_probe<ITER><<<blocks, 256>>>(d, 0.999999f, 1e-7f);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        best = ms < best ? ms : best;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(d);
    const double flops = 8.0 * double(blocks) * 256.0 * 2.0 * 8.0 * ITER;
    return flops / (double(best) * 1e-3) / 1e12;
}

}  // namespace mfree
