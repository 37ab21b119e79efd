// Training kernels of the proposal network (FP32 throughout, deterministic:
// every output element is summed by one thread in a fixed order).
//
//   k_gemm      C = A . B (+ bias) (ReLU), A and B addressed by arbitrary row and
//               column strides, so forward (X W^T), input gradient (dY W) and
//               weight gradient (dY^T X) are the same kernel; 64x64 tiles,
//               16-deep K slices staged in shared memory, 4x4 outputs a thread.
//   k_xent      softmax cross-entropy of the partition head (all valid
//               partitionings and the single-partition class) plus that of the
//               block-mode head of the label's partition count; writes dZ
//               (already divided by the batch) and the two losses per row.
//   k_relu_bwd, k_colsum (bias gradients), k_adam.
#include <cuda_runtime.h>
#include <stdint.h>

#include "astcb200.h"
#include "mlp.h"

namespace astcb200 {
namespace {

constexpr int kBM = 64, kBN = 64, kBK = 16;

__global__ void __launch_bounds__(256) k_gemm(const float* __restrict__ A, const float* __restrict__ B, float* __restrict__ C,
                                              int M, int N, int K, long long sa_i, long long sa_l, long long sb_l, long long sb_j,
                                              const float* __restrict__ bias, int relu, int accumulate) {
    __shared__ float As[kBK][kBM + 4];
    __shared__ float Bs[kBK][kBN + 4];
    const int tid = threadIdx.x, tx = tid % 16, ty = tid / 16;
    const int i0 = blockIdx.y * kBM, j0 = blockIdx.x * kBN;
    float acc[4][4] = {};
    for (int l0 = 0; l0 < K; l0 += kBK) {
        for (int e = tid; e < kBK * kBM; e += 256) {
            const int l = e / kBM, i = e % kBM;
            const int gi = i0 + i, gl = l0 + l;
            As[l][i] = (gi < M && gl < K) ? A[gi * sa_i + gl * sa_l] : 0.0f;
        }
        for (int e = tid; e < kBK * kBN; e += 256) {
            const int l = e / kBN, j = e % kBN;
            const int gj = j0 + j, gl = l0 + l;
            Bs[l][j] = (gj < N && gl < K) ? B[gl * sb_l + gj * sb_j] : 0.0f;
        }
        __syncthreads();
#pragma unroll
        for (int l = 0; l < kBK; l++) {
            float a[4], b[4];
#pragma unroll
            for (int r = 0; r < 4; r++) a[r] = As[l][ty * 4 + r];
#pragma unroll
            for (int c = 0; c < 4; c++) b[c] = Bs[l][tx * 4 + c];
#pragma unroll
            for (int r = 0; r < 4; r++)
#pragma unroll
                for (int c = 0; c < 4; c++) acc[r][c] = fmaf(a[r], b[c], acc[r][c]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int r = 0; r < 4; r++) {
        const int gi = i0 + ty * 4 + r;
        if (gi >= M) continue;
#pragma unroll
        for (int c = 0; c < 4; c++) {
            const int gj = j0 + tx * 4 + c;
            if (gj >= N) continue;
            float v = acc[r][c];
            if (accumulate) v += C[(size_t)gi * N + gj];
            if (bias) v += bias[gj];
            if (relu) v = fmaxf(v, 0.0f);
            C[(size_t)gi * N + gj] = v;
        }
    }
}

struct XentShape {
    int nout, nbm, head_stride, batch;
    mlp::Shape cls;  // class plan (p1, part_base, head_base)
};
__device__ __forceinline__ float wmax(float v) {
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xFFFFFFFFu, v, o));
    return v;
}
__device__ __forceinline__ float wsum(float v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
    return v;
}

__global__ void __launch_bounds__(128) k_xent(const float* __restrict__ Z, const int* __restrict__ part_label,
                                               const int* __restrict__ bm_label, XentShape s, float* __restrict__ dZ,
                                               float* __restrict__ loss) {
    const int lane = threadIdx.x & 31;
    const int b = blockIdx.x * 4 + (threadIdx.x >> 5);
    if (b >= s.batch) return;
    const float* z = Z + (size_t)b * s.nout;
    float* g = dZ + (size_t)b * s.nout;
    const float inv_b = 1.0f / (float)s.batch;
    const int pl = part_label[b], bl = bm_label[b];
    // partition head
    float mx = -3.0e38f;
    const int p1 = s.cls.p1, hb = s.cls.head_base;
    for (int c = lane; c <= p1; c += 32) mx = fmaxf(mx, z[c]);
    mx = wmax(mx);
    float se = 0.0f;
    for (int c = lane; c <= p1; c += 32) se += expf(z[c] - mx);
    se = wsum(se);
    for (int c = lane; c < hb; c += 32) {
        float v = 0.0f;
        if (c <= p1) v = (expf(z[c] - mx) / se - (c == pl ? 1.0f : 0.0f)) * inv_b;
        g[c] = v;
    }
    // block-mode head of the label's partition count
    const int head = mlp::head_of_class(s.cls, pl);
    const int h0 = hb + head * s.head_stride;
    float hm = -3.0e38f;
    for (int c = lane; c < s.nbm; c += 32) hm = fmaxf(hm, z[h0 + c]);
    hm = wmax(hm);
    float hs = 0.0f;
    for (int c = lane; c < s.nbm; c += 32) hs += expf(z[h0 + c] - hm);
    hs = wsum(hs);
    for (int c = hb + lane; c < s.nout; c += 32) {
        float v = 0.0f;
        const int k = c - h0;
        if (k >= 0 && k < s.nbm) v = (expf(z[c] - hm) / hs - (k == bl ? 1.0f : 0.0f)) * inv_b;
        g[c] = v;
    }
    if (lane == 0) {
        loss[2 * b] = logf(se) + mx - z[pl];
        loss[2 * b + 1] = logf(hs) + hm - z[h0 + bl];
    }
}

__global__ void k_relu_bwd(float* __restrict__ dh, const float* __restrict__ h, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        if (!(h[i] > 0.0f)) dh[i] = 0.0f;
}

__global__ void k_colsum(const float* __restrict__ dy, float* __restrict__ db, int rows, int cols) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= cols) return;
    float s = 0.0f;
    for (int r = 0; r < rows; r++) s += dy[(size_t)r * cols + j];
    db[j] = s;
}

__global__ void k_adam(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v, size_t n,
                       float lr, float b1, float b2, float eps, float c1, float c2) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.0f - b1) * gi;
        const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
}

int launch_status() { return cudaGetLastError() == cudaSuccess ? ASTCB200_OK : ASTCB200_CUDA_ERROR; }

}  // namespace
}  // namespace astcb200

using namespace astcb200;

extern "C" {

int astcb200_train_gemm(const float* A, const float* B, float* C, int M, int N, int K, int64_t sa_i, int64_t sa_l, int64_t sb_l,
                        int64_t sb_j, const float* bias, int relu, int accumulate, void* stream) {
    if (!A || !B || !C || M <= 0 || N <= 0 || K <= 0) return ASTCB200_BAD_ARG;
    const dim3 grid((N + kBN - 1) / kBN, (M + kBM - 1) / kBM);
    k_gemm<<<grid, 256, 0, (cudaStream_t)stream>>>(A, B, C, M, N, K, sa_i, sa_l, sb_l, sb_j, bias, relu, accumulate);
    return launch_status();
}

int astcb200_train_xent(const float* Z, uint32_t nout, const int32_t* part_label, const int32_t* bm_label, uint32_t batch,
                        uint32_t nbm, uint32_t head_stride, const uint32_t* sel3, float* dZ, float* loss_rows, void* stream) {
    if (!Z || !part_label || !bm_label || !sel3 || !dZ || !loss_rows || batch == 0) return ASTCB200_BAD_ARG;
    XentShape s;
    s.cls = mlp::shape_for(0, (int)nbm, sel3);
    if (nbm > head_stride || nout < (uint32_t)s.cls.head_base + 4 * head_stride) return ASTCB200_BAD_ARG;
    s.nout = (int)nout; s.nbm = (int)nbm; s.head_stride = (int)head_stride; s.batch = (int)batch;
    k_xent<<<(batch + 3) / 4, 128, 0, (cudaStream_t)stream>>>(Z, part_label, bm_label, s, dZ, loss_rows);
    return launch_status();
}

int astcb200_train_relu_backward(float* dH, const float* H, size_t n, void* stream) {
    if (!dH || !H) return ASTCB200_BAD_ARG;
    k_relu_bwd<<<1184, 256, 0, (cudaStream_t)stream>>>(dH, H, n);
    return launch_status();
}

int astcb200_train_colsum(const float* dY, float* db, uint32_t rows, uint32_t cols, void* stream) {
    if (!dY || !db) return ASTCB200_BAD_ARG;
    k_colsum<<<(cols + 127) / 128, 128, 0, (cudaStream_t)stream>>>(dY, db, (int)rows, (int)cols);
    return launch_status();
}

int astcb200_train_adam(float* w, const float* g, float* m, float* v, size_t n, float lr, float beta1, float beta2, float eps,
                        uint32_t step, void* stream) {
    if (!w || !g || !m || !v || step == 0) return ASTCB200_BAD_ARG;
    const float c1 = 1.0f - powf(beta1, (float)step), c2 = 1.0f - powf(beta2, (float)step);
    k_adam<<<1184, 256, 0, (cudaStream_t)stream>>>(w, g, m, v, n, lr, beta1, beta2, eps, c1, c2);
    return launch_status();
}

}  // extern "C"
