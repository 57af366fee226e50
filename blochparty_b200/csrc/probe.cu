// Roofline denominator: the FP32 FMA throughput of the device, measured with independent FFMA chains.
// Each thread runs 8 independent dependency chains of `iters` fused multiply-adds (2 flops each); the grid
// is 4 CTAs of 256 threads per SM. The host times it with CUDA events and divides the flops by the time.
// bp_ffma2_peak does the same with the paired form (__ffma2_rn: two FMAs per instruction on a float2), which
// shows whether paired FMAs raise the FP32 rate or only save issue slots.
#include <cuda_runtime.h>

#include "../../include/blochparty_b200.h"

__global__ void __launch_bounds__(256) bp_ffma_peak_kernel(float* out, int iters, float a, float b) {
    float x0 = threadIdx.x * 1e-7f, x1 = x0 + 1e-7f, x2 = x0 + 2e-7f, x3 = x0 + 3e-7f;
    float x4 = x0 + 4e-7f, x5 = x0 + 5e-7f, x6 = x0 + 6e-7f, x7 = x0 + 7e-7f;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            x0 = fmaf(x0, a, b), x1 = fmaf(x1, a, b), x2 = fmaf(x2, a, b), x3 = fmaf(x3, a, b);
            x4 = fmaf(x4, a, b), x5 = fmaf(x5, a, b), x6 = fmaf(x6, a, b), x7 = fmaf(x7, a, b);
        }
    }
    const float s = ((x0 + x1) + (x2 + x3)) + ((x4 + x5) + (x6 + x7));
    if (s == 1234.5f) out[blockIdx.x * blockDim.x + threadIdx.x] = s;  // keeps the chains live
}

extern "C" int bp_ffma_peak(float* out, int iters, int64_t* flops, void* stream) {
    if (!out || !flops || iters < 1) return BP_E_ARG;
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int grid = 4 * sms, threads = 256;
    bp_ffma_peak_kernel<<<grid, threads, 0, static_cast<cudaStream_t>(stream)>>>(out, iters, 0.999999f, 1e-7f);
    *flops = (int64_t)grid * threads * iters * 16 * 8 * 2;
    return cudaGetLastError() == cudaSuccess ? BP_OK : BP_E_LAUNCH;
}

__global__ void __launch_bounds__(256) bp_ffma2_peak_kernel(float* out, int iters, float a, float b) {
    const float t = threadIdx.x * 1e-7f;
    float2 x0 = make_float2(t, t + 1e-7f), x1 = make_float2(t + 2e-7f, t + 3e-7f);
    float2 x2 = make_float2(t + 4e-7f, t + 5e-7f), x3 = make_float2(t + 6e-7f, t + 7e-7f);
    const float2 a2 = make_float2(a, a), b2 = make_float2(b, b);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            x0 = __ffma2_rn(x0, a2, b2), x1 = __ffma2_rn(x1, a2, b2);
            x2 = __ffma2_rn(x2, a2, b2), x3 = __ffma2_rn(x3, a2, b2);
        }
    }
    const float s = ((x0.x + x0.y) + (x1.x + x1.y)) + ((x2.x + x2.y) + (x3.x + x3.y));
    if (s == 1234.5f) out[blockIdx.x * blockDim.x + threadIdx.x] = s;  // keeps the chains live
}

extern "C" int bp_ffma2_peak(float* out, int iters, int64_t* flops, void* stream) {
    if (!out || !flops || iters < 1) return BP_E_ARG;
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int grid = 4 * sms, threads = 256;
    bp_ffma2_peak_kernel<<<grid, threads, 0, static_cast<cudaStream_t>(stream)>>>(out, iters, 0.999999f, 1e-7f);
    *flops = (int64_t)grid * threads * iters * 16 * 8 * 2;
    return cudaGetLastError() == cudaSuccess ? BP_OK : BP_E_LAUNCH;
}
