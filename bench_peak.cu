// FP32 throughput probe for bench.py (not part of the encoder library): each thread
// runs independent chains of dependent FMAs.  It measures the roofline denominator of
// the FP32-bound search kernels (the recorded peaks of this GPU give HBM and bf16
// figures but no FP32 one).  Built into bench_peak.so by __graft_entry__.build():
//   nvcc -gencode arch=compute_100a,code=sm_100a -O3 -shared -Xcompiler -fPIC bench_peak.cu -o bench_peak.so
#include <cuda_runtime.h>

namespace {

__global__ void k_fma_chain(float* out, int iters, float a, float b) {
    float x0 = threadIdx.x * 1e-7f, x1 = x0 + 1.0f, x2 = x0 + 2.0f, x3 = x0 + 3.0f;
    float x4 = x0 + 4.0f, x5 = x0 + 5.0f, x6 = x0 + 6.0f, x7 = x0 + 7.0f;
    for (int i = 0; i < iters; i++) {
        x0 = __fmaf_rn(x0, a, b); x1 = __fmaf_rn(x1, a, b); x2 = __fmaf_rn(x2, a, b); x3 = __fmaf_rn(x3, a, b);
        x4 = __fmaf_rn(x4, a, b); x5 = __fmaf_rn(x5, a, b); x6 = __fmaf_rn(x6, a, b); x7 = __fmaf_rn(x7, a, b);
    }
    const float s = ((x0 + x1) + (x2 + x3)) + ((x4 + x5) + (x6 + x7));
    if (s == 123.456f) out[blockIdx.x] = s;  // keeps the chains live
}

}  // namespace

// TFLOP/s of dependent-FMA chains on `device` (an FMA counts 2 ops); 0 on success.
extern "C" int bench_fp32_peak(int device, double* tflops) {
    if (!tflops) return 1;
    if (cudaSetDevice(device) != cudaSuccess) return 2;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return 2;
    float* out = nullptr;
    const int blocks = prop.multiProcessorCount * 8, threads = 256, iters = 1 << 14;
    if (cudaMalloc((void**)&out, blocks * sizeof(float)) != cudaSuccess) return 3;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0); cudaEventCreate(&e1);
    k_fma_chain<<<blocks, threads>>>(out, 256, 0.999999f, 1e-7f);  // warm-up
    float best = 1e30f;
    for (int r = 0; r < 5; r++) {
        cudaEventRecord(e0);
        k_fma_chain<<<blocks, threads>>>(out, iters, 0.999999f, 1e-7f);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best) best = ms;
    }
    const cudaError_t err = cudaGetLastError();
    cudaEventDestroy(e0); cudaEventDestroy(e1); cudaFree(out);
    if (err != cudaSuccess) return 2;
    const double flops = 2.0 * 8.0 * (double)iters * blocks * threads;
    *tflops = flops / (best * 1e-3) / 1e12;
    return 0;
}
