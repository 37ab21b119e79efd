// Selects a device for the duration of a C-ABI call and restores the caller's
// current device when the call returns, so the library never changes a host
// thread's device behind its back.
#pragma once
#include <cuda_runtime.h>

namespace astcb200 {

struct DeviceGuard {
    int prev = -1;
    int dev = -1;
    cudaError_t err = cudaSuccess;
    explicit DeviceGuard(int device) : dev(device) {
        if (cudaGetDevice(&prev) != cudaSuccess) { prev = -1; cudaGetLastError(); }
        if (prev != device) err = cudaSetDevice(device);
    }
    ~DeviceGuard() {
        if (prev >= 0 && prev != dev) cudaSetDevice(prev);
    }
    DeviceGuard(const DeviceGuard&) = delete;
    DeviceGuard& operator=(const DeviceGuard&) = delete;
};

}  // namespace astcb200

// Selects ctx->device until the enclosing scope ends; returns from the caller on failure.
#define ASTCB200_DEVICE_SCOPE(ctx)                                                         \
    ::astcb200::DeviceGuard device_scope_((ctx)->device);                                  \
    if (device_scope_.err != cudaSuccess) return ::astcb200::cuda_fail((ctx), device_scope_.err, "cudaSetDevice")
