// Diagnostics used by the benchmark: a measured INT32 issue peak for the
// roofline denominator of the integer filter kernels.
#include <cuda_runtime.h>
#include <stdint.h>
#include "../../include/ccs.h"

namespace {

// Eight independent add / xor chains: every iteration issues 16 single-cycle
// integer ALU instructions per thread (IADD3 / LOP3), no memory traffic.
__global__ void __launch_bounds__(256) int_peak_kernel(uint32_t* out, uint32_t iters, uint32_t seed) {
    uint32_t a[8];
#pragma unroll
    for (int j = 0; j < 8; j++) a[j] = seed * (threadIdx.x + 1 + j) + blockIdx.x + j;
    for (uint32_t i = 0; i < iters; i++) {
#pragma unroll
        for (int j = 0; j < 8; j++) a[j] = a[j] + a[(j + 1) & 7] + 0x9E3779B9u;
#pragma unroll
        for (int j = 0; j < 8; j++) a[j] = a[j] ^ a[(j + 3) & 7] ^ 0x7F4A7C15u;
    }
    uint32_t r = 0;
#pragma unroll
    for (int j = 0; j < 8; j++) r ^= a[j];
    if (r == seed) out[0] = r;   // practically never taken; keeps the chains live
}

// Eight independent multiply-add chains: lo and hi halves of 32x32-bit
// products (IMAD / IMAD.HI), the building block of the Montgomery products.
__global__ void __launch_bounds__(256) imad_peak_kernel(uint32_t* out, uint32_t iters, uint32_t seed) {
    uint32_t a[8];
#pragma unroll
    for (int j = 0; j < 8; j++) a[j] = seed * (threadIdx.x + 3 + j) + blockIdx.x + j;
    const uint32_t m = seed | 1u;
    for (uint32_t i = 0; i < iters; i++) {
#pragma unroll
        for (int j = 0; j < 8; j++) a[j] = a[j] * m + a[(j + 1) & 7];
#pragma unroll
        for (int j = 0; j < 8; j++) a[j] = __umulhi(a[j], m) + a[(j + 5) & 7];
    }
    uint32_t r = 0;
#pragma unroll
    for (int j = 0; j < 8; j++) r ^= a[j];
    if (r == seed) out[0] = r;
}

}  // namespace

extern "C" ccs_status ccs_measure_imad_peak(int device, double* tops) {
    if (!tops) return CCS_ERR_INVALID;
    if (cudaSetDevice(device) != cudaSuccess) return CCS_ERR_CUDA;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return CCS_ERR_CUDA;
    uint32_t* out = nullptr;
    if (cudaMalloc(&out, 4) != cudaSuccess) return CCS_ERR_NOMEM;
    const int blocks = prop.multiProcessorCount * 8;
    const uint32_t iters = 1u << 15;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    imad_peak_kernel<<<blocks, 256>>>(out, 512, 777);
    cudaEventRecord(e0);
    imad_peak_kernel<<<blocks, 256>>>(out, iters, 777);
    cudaEventRecord(e1);
    cudaError_t e = cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    if (e != cudaSuccess || ms <= 0) return CCS_ERR_CUDA;
    // 16 multiply instructions per iteration per thread
    *tops = (double)blocks * 256.0 * iters * 16.0 / (ms * 1e-3) / 1e12;
    return CCS_OK;
}

extern "C" ccs_status ccs_measure_int32_peak(int device, double* tops) {
    if (!tops) return CCS_ERR_INVALID;
    if (cudaSetDevice(device) != cudaSuccess) return CCS_ERR_CUDA;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return CCS_ERR_CUDA;
    uint32_t* out = nullptr;
    if (cudaMalloc(&out, 4) != cudaSuccess) return CCS_ERR_NOMEM;
    const int blocks = prop.multiProcessorCount * 8;
    const uint32_t iters = 1u << 16;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    int_peak_kernel<<<blocks, 256>>>(out, 1024, 12345);          // warm-up
    cudaEventRecord(e0);
    int_peak_kernel<<<blocks, 256>>>(out, iters, 12345);
    cudaEventRecord(e1);
    cudaError_t e = cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    if (e != cudaSuccess || ms <= 0) return CCS_ERR_CUDA;
    double ops = (double)blocks * 256.0 * iters * 16.0;
    *tops = ops / (ms * 1e-3) / 1e12;
    return CCS_OK;
}
