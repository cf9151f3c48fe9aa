// A measurement entry point: the FP64 fused multiply-add throughput of this GPU, for the
// roofline denominator of the f64 kernels (independent chains of DFMA on every SM).
#include <cuda_runtime.h>

#include "../../include/pacuda_b200.h"

namespace {
__global__ void __launch_bounds__(512) dfma_chains(double *sink, uint32_t iterations, double a, double b) {
    double x0 = threadIdx.x * 1e-3, x1 = x0 + 1, x2 = x0 + 2, x3 = x0 + 3, x4 = x0 + 4, x5 = x0 + 5, x6 = x0 + 6,
           x7 = x0 + 7;
    for (uint32_t i = 0; i < iterations; i++) {
        x0 = __fma_rn(x0, a, b); x1 = __fma_rn(x1, a, b); x2 = __fma_rn(x2, a, b); x3 = __fma_rn(x3, a, b);
        x4 = __fma_rn(x4, a, b); x5 = __fma_rn(x5, a, b); x6 = __fma_rn(x6, a, b); x7 = __fma_rn(x7, a, b);
    }
    double s = ((x0 + x1) + (x2 + x3)) + ((x4 + x5) + (x6 + x7));
    if (s == 123.456) sink[blockIdx.x] = s;  // keeps the chains live
}
}  // namespace

extern "C" int pacuda_b200_measure_fp64(double *sink, uint32_t iterations, uint32_t *blocks, uint32_t *threads,
                                        void *stream) {
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    *blocks = 4 * sms;
    *threads = 512;
    dfma_chains<<<*blocks, *threads, 0, (cudaStream_t)stream>>>(sink, iterations, 0.999999, 1e-7);
    return cudaGetLastError() == cudaSuccess ? PACMAN_RECURRENCE_OK : PACMAN_RECURRENCE_DEVICE_ERROR;
}
