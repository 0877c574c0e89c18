// FP64 pipe throughput probe, used only by bench.py to measure the roofline denominator of the exact engine
// (its work is FP64 add/mul/fma instructions, not tensor-core contractions). Each thread runs independent
// chains of DADD / DMUL / DFMA on registers; one instruction counts as one operation.
#include <cuda_runtime.h>

namespace {

template <int KIND>
__global__ void __launch_bounds__(256) k_fp64(double* out, int iters, double seed) {
    double a[8];
#pragma unroll
    for (int i = 0; i < 8; i++) a[i] = seed + threadIdx.x * 1e-9 + i * 1e-7;
    const double b = 1.0000000001, c = 1e-12;
    for (int it = 0; it < iters; it++) {
#pragma unroll
        for (int i = 0; i < 8; i++) {
            if (KIND == 0) a[i] = __fma_rn(a[i], b, c);
            else if (KIND == 1) a[i] = __dadd_rn(a[i], c);
            else a[i] = __dmul_rn(a[i], b);
        }
    }
    double s = 0;
#pragma unroll
    for (int i = 0; i < 8; i++) s += a[i];
    if (s == 12345.678) out[0] = s;  // keeps the chains live
}

}  // namespace

// Measures FP64 instructions per second (one DFMA, DADD or DMUL counts once) for kind 0 fma, 1 add, 2 mul.
// Returns 0 on success.
extern "C" int kbsrc_probe_fp64(int kind, double* ops_per_second) {
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev))
        return -1;
    double* out = nullptr;
    if (cudaMalloc(&out, 8) != cudaSuccess) return -1;
    const int iters = 20000, blocks = sms * 8, threads = 256;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    auto launch = [&] {
        if (kind == 0) k_fp64<0><<<blocks, threads>>>(out, iters, 1.0);
        else if (kind == 1) k_fp64<1><<<blocks, threads>>>(out, iters, 1.0);
        else k_fp64<2><<<blocks, threads>>>(out, iters, 1.0);
    };
    launch();  // warm-up
    cudaEventRecord(e0);
    for (int r = 0; r < 5; r++) launch();
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    if (cudaGetLastError() != cudaSuccess || ms <= 0) return -1;
    *ops_per_second = 5.0 * blocks * threads * (double)iters * 8 / (ms * 1e-3);
    return 0;
}
