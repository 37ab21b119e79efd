// Learned proposal: network inference on the tcgen05 tensor cores and the
// selection of partitionings, block modes and routes from its logits.
//
// k_mlp_logits: one CTA of 8 warps per 128 blocks (two threads per block row,
// each taking half of a row's accumulator columns).  The block texels are
// staged in shared memory as bf16 in the tensor core's K-major core-matrix
// layout; each layer is a chain of tcgen05.mma (M=128, K=16 per instruction,
// A and B from shared memory, FP32 accumulators in tensor memory) issued by
// one thread.  Weights arrive by bulk copies (cp.async.bulk, completion on an
// mbarrier) already laid out on the host in the same core-matrix order.  The
// two hidden layers' epilogues (bias, ReLU, bf16) read the accumulators with
// tcgen05.ld and write the next layer's A operand in place; layer 3 runs in
// 64-column chunks with double-buffered weights and accumulators, so the
// epilogue of chunk j overlaps the MMAs of chunk j+1 and the copy of chunk
// j+2.  The layer-3 epilogue adds the bias, stages each row's 64 FP32 logits
// in shared memory and writes the row with one 256-byte bulk copy to global
// memory (instead of 64 strided stores per thread); CTAs start the chunk
// sequence at different chunks so that they do not all fetch the same weights
// from L2 at once.  Every wait on an mbarrier is bounded (error_flag[1] polls, 0 = 2^24);
// a CTA that gives up sets error_flag[0], waits (bounded by 2^24 polls) for its own copies
// and MMAs in flight, frees its tensor memory and returns.
//
// k_select: one warp per block turns the logits into the proposal search's
// inputs: a softmax over the partition classes, the best partitionings (in
// probability order, until the proposed mass reaches the coverage), the best
// block modes of each partition count as bit masks, and the route: blocks
// whose best-kmax mass is below the threshold take the full search.
#include <cuda_bf16.h>

#include "mlp.h"

namespace astcb200 {
namespace mlp {
namespace {

constexpr uint32_t kOffA = 0;                 // 64 KB: X, then H1, then H2 (128 rows x up to 256 bf16)
constexpr uint32_t kOffW = 65536;             // 128 KB: W1 | W2 | two W3 chunks of 32 KB
constexpr uint32_t kW3Buf = kChunkN * 256 * 2;               // one W3 chunk (bf16)
constexpr uint32_t kStageStride = kChunkN + 4;                // floats per staged logit row (padded)
constexpr uint32_t kStageBuf = kTileRows * kStageStride * 4;  // one staged chunk of logits
constexpr uint32_t kOffStage = kOffW + 2 * kW3Buf;            // two staging buffers (free after layer 2)
constexpr uint32_t kOffBar = kOffStage + 2 * kStageBuf;       // mbarriers and flags
static_assert(kOffBar == 200704 && kOffBar + 1024 + 1024 <= (uint32_t)kMlpSmemBytes, "shared memory plan");
constexpr uint32_t kTmemCols = 512;
constexpr uint32_t kWaitLimit = 1u << 24;     // polls of an mbarrier before a CTA gives up
constexpr uint32_t kCopyPiece = 32768;        // bytes per bulk copy instruction

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ bool mbar_test_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Waits for the phase of parity `parity` to complete, at most `limit` polls.  Limits below
// 2^16 (set by tests of the give-up path) poll with the non-blocking test_wait, so that a
// wait for work still in flight gives up at once; larger ones use try_wait, which may
// suspend the thread until the phase completes.
__device__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint32_t limit = kWaitLimit) {
    if (limit < (1u << 16)) {
        for (uint32_t i = 0; i < limit; i++)
            if (mbar_test_wait(bar, parity)) return true;
        return false;
    }
    for (uint32_t i = 0; i < limit; i++)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
// One thread: expect `bytes` on bar and copy them in pieces.
__device__ void load_weights(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    mbar_expect_tx(bar, bytes);
    for (uint32_t o = 0; o < bytes; o += kCopyPiece)
        bulk_load(static_cast<uint8_t*>(dst) + o, static_cast<const uint8_t*>(src) + o, min(kCopyPiece, bytes - o), bar);
}

__device__ __forceinline__ void tc_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void async_proxy_fence() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Shared-memory matrix descriptor: no swizzle, K-major core matrices; lbo =
// bytes between K-adjacent core matrices, sbo = bytes between M/N-adjacent
// ones; descriptor version 1 (bits 46-47), base offset 0.
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);
}
// Instruction descriptor of kind::f16: bf16 A and B (K-major), FP32 accumulator.
__host__ __device__ constexpr uint32_t instr_desc(int m, int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}
static_assert(instr_desc(128, 256) == 0x08400490u, "instruction descriptor layout");

__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc)
        : "memory");
}
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// 32 consecutive FP32 columns of the calling thread's tensor-memory lane.
__device__ __forceinline__ void tmem_load32(uint32_t taddr, float* v) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
          "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
          "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ uint32_t bf16_bits(float f) {
    return (uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(f));
}
__device__ __forceinline__ uint4 pack8(const float* v) {
    return make_uint4(bf16_bits(v[0]) | (bf16_bits(v[1]) << 16), bf16_bits(v[2]) | (bf16_bits(v[3]) << 16),
                      bf16_bits(v[4]) | (bf16_bits(v[5]) << 16), bf16_bits(v[6]) | (bf16_bits(v[7]) << 16));
}

// Hidden-layer epilogue: accumulator columns [col0 + c0, col0 + c0 + 128) of this thread's
// row (c0: its half of the 256) -> bias, ReLU, bf16 -> the A operand (128 rows x 256) of the
// next layer.
__device__ void hidden_epilogue(uint32_t tmem_row, uint32_t col0, int c0, const float* __restrict__ bias, uint8_t* sA, int m) {
    for (int c = c0; c < c0 + 128; c += 32) {
        float v[32];
        tmem_load32(tmem_row + col0 + c, v);
#pragma unroll
        for (int q = 0; q < 4; q++) {
            float h[8];
#pragma unroll
            for (int i = 0; i < 8; i++) h[i] = fmaxf(v[q * 8 + i] + __ldg(bias + c + q * 8 + i), 0.0f);
            *reinterpret_cast<uint4*>(sA + core_index(m, c + q * 8, kTileRows) * 2) = pack8(h);
        }
    }
}

constexpr int kMlpThreads = 2 * kTileRows;  // two threads per row, each taking half of the columns

__global__ void __launch_bounds__(kMlpThreads, 1)
    k_mlp_logits(const __grid_constant__ KernelArgs a, const __grid_constant__ Net net, float* __restrict__ logits, int* error_flag) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* sm = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint8_t* sA = sm + kOffA;
    uint8_t* sW = sm + kOffW;
    uint64_t* bw = reinterpret_cast<uint64_t*>(sm + kOffBar);       // [2] weight buffers
    uint64_t* bm = bw + 2;                                           // [3] MMA completion: layers 1-2, layer-3 buffers
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bw + 5);
    int* abort_flag = reinterpret_cast<int*>(bw + 6);
    const int tid = threadIdx.x, warp = tid >> 5;
    // this thread's row (block) in the tile and tensor-memory lane; warps w and w + 4 share
    // the lanes of quarter w and split the columns (half)
    const int m = tid % kTileRows, half = tid / kTileRows;
    const int lb = blockIdx.x * kTileRows + m;
    const Shape& S = net.s;
    const int nchunks = S.nout / kChunkN;
    // CTAs walk the layer-3 chunks from different starting points, so that at any moment they
    // read different parts of the weights from L2 instead of all the same chunk
    const int j0 = blockIdx.x % nchunks;
    auto chunk_of = [&](int j) { const int c = j0 + j; return c < nchunks ? c : c - nchunks; };
    const uint32_t wl = error_flag[1] ? (uint32_t)error_flag[1] : kWaitLimit;  // polls per wait

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)), "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        for (int i = 0; i < 5; i++) mbar_init(&bw[i], 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc_before();
    __syncthreads();
    tc_after();
    const uint32_t tmem = *tmem_slot;
    const uint32_t tmem_row = tmem + ((uint32_t)((warp & 3) * 32) << 16);

    // thread 0's bookkeeping of weight copies and MMA commits in flight: a phase counts as
    // done only once a wait saw it complete, so the drain after a give-up waits for the rest
    uint32_t w_issued[2] = {0, 0}, w_done[2] = {0, 0};
    uint32_t m_issued[3] = {0, 0, 0}, m_done[3] = {0, 0, 0};  // only the waits of all threads advance m_done
    bool ok = true, failed = false;  // failed: the same in every thread (set only at uniform exits)

    if (tid == 0) { load_weights(sW, net.w1, 256u * S.k0p * 2, &bw[0]); w_issued[0]++; }

    // stage the block's texels (RGBA8 / 255 -> bf16), zero rows past the chunk
    {
        const int blk = lb < a.nblocks ? chunk_block(a, lb) : -1;
        const int T = a.L.T;
        BlockSrc src{};
        if (blk >= 0) src = block_src(a, blk);
        for (int j = half; j < S.k0p / 8; j += 2) {
            float v[8];
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int t = 2 * j + h;
                uchar4 p = make_uchar4(0, 0, 0, 0);
                if (blk >= 0 && t < T) p = src_rgba8(src, a.L.bx, t);
                v[4 * h + 0] = (float)p.x / 255.0f; v[4 * h + 1] = (float)p.y / 255.0f;
                v[4 * h + 2] = (float)p.z / 255.0f; v[4 * h + 3] = (float)p.w / 255.0f;
            }
            *reinterpret_cast<uint4*>(sA + core_index(m, 8 * j, kTileRows) * 2) = pack8(v);
        }
    }
    async_proxy_fence();
    tc_before();
    __syncthreads();

    const uint32_t a_base = smem_u32(sA), w_base = smem_u32(sW);
    constexpr uint32_t kLboA = (kTileRows / 8) * 128, kLboW256 = (256 / 8) * 128, kLboW3 = (kChunkN / 8) * 128;
    auto issue_chunk = [&](int jj) -> bool {  // thread 0: chunk jj's MMAs once its weights have landed
        const int bb = jj & 1;
        if (!mbar_wait(&bw[bb], w_done[bb] & 1, wl)) return false;
        w_done[bb]++;
        for (int kk = 0; kk < 16; kk++)
            mma_bf16(tmem + bb * kChunkN, smem_desc(a_base + kk * 2 * kLboA, kLboA, 128),
                     smem_desc(w_base + bb * kW3Buf + kk * 2 * kLboW3, kLboW3, 128), instr_desc(128, kChunkN), kk > 0);
        mma_commit(&bm[1 + bb]);
        m_issued[1 + bb]++;
        return true;
    };

    // ---- layer 1: X (128 x k0p) . W1^T -> tensor memory columns [0, 256)
    if (tid == 0) {
        tc_after();
        if (!mbar_wait(&bw[0], w_done[0] & 1, wl)) *abort_flag = 1;
        else {
            w_done[0]++;
            for (int kk = 0; kk < S.k0p / 16; kk++)
                mma_bf16(tmem, smem_desc(a_base + kk * 2 * kLboA, kLboA, 128), smem_desc(w_base + kk * 2 * kLboW256, kLboW256, 128),
                         instr_desc(128, 256), kk > 0);
            mma_commit(&bm[0]);
            m_issued[0]++;
        }
    }
    __syncthreads();
    if (*abort_flag) { failed = true; goto cleanup; }
    ok = mbar_wait(&bm[0], m_done[0] & 1, wl);
    if (ok) m_done[0]++;
    if (__syncthreads_or(!ok)) { failed = true; goto cleanup; }
    tc_after();
    if (tid == 0) { load_weights(sW, net.w2, 256u * 256u * 2, &bw[0]); w_issued[0]++; }
    hidden_epilogue(tmem_row, 0, half * 128, net.b1, sA, m);
    async_proxy_fence();
    tc_before();
    __syncthreads();

    // ---- layer 2: H1 (128 x 256) . W2^T -> columns [256, 512)
    if (tid == 0) {
        tc_after();
        if (!mbar_wait(&bw[0], w_done[0] & 1, wl)) *abort_flag = 1;
        else {
            w_done[0]++;
            for (int kk = 0; kk < 16; kk++)
                mma_bf16(tmem + 256, smem_desc(a_base + kk * 2 * kLboA, kLboA, 128),
                         smem_desc(w_base + kk * 2 * kLboW256, kLboW256, 128), instr_desc(128, 256), kk > 0);
            mma_commit(&bm[0]);
            m_issued[0]++;
        }
    }
    __syncthreads();
    if (*abort_flag) { failed = true; goto cleanup; }
    ok = mbar_wait(&bm[0], m_done[0] & 1, wl);
    if (ok) m_done[0]++;
    if (__syncthreads_or(!ok)) { failed = true; goto cleanup; }
    tc_after();
    if (tid == 0) {
        for (int j = 0; j < 2 && j < nchunks; j++) {
            load_weights(sW + j * kW3Buf, net.w3 + (size_t)chunk_of(j) * kChunkN * 256, kW3Buf, &bw[j]);
            w_issued[j]++;
        }
    }
    hidden_epilogue(tmem_row, 256, half * 128, net.b2, sA, m);
    async_proxy_fence();
    tc_before();
    __syncthreads();

    // ---- layer 3: H2 (128 x 256) . W3^T in chunks of 64 columns, accumulators alternating
    // between tensor-memory columns [0, 64) and [64, 128).  Chunk 0's MMAs are issued here;
    // chunk j + 1's right after chunk j's have completed, into the accumulator buffer chunk
    // j - 1's epilogue read before the previous staging barrier, so that they run while chunk
    // j's epilogue reads its own.  Two barriers per chunk.
    if (tid == 0) {
        tc_after();
        if (!issue_chunk(0)) *abort_flag = 1;
    }
    __syncthreads();
    if (*abort_flag) { failed = true; goto cleanup; }
    for (int j = 0; j < nchunks; j++) {
        const int b = j & 1;
        // this thread's 32 biases of the chunk, loaded before the wait so that it hides them
        float bv[32];
        {
            const float4* bias4 = reinterpret_cast<const float4*>(net.b3 + chunk_of(j) * kChunkN + half * 32);
#pragma unroll
            for (int q = 0; q < 8; q++) {
                const float4 t = __ldg(bias4 + q);
                bv[4 * q] = t.x; bv[4 * q + 1] = t.y; bv[4 * q + 2] = t.z; bv[4 * q + 3] = t.w;
            }
        }
        ok = mbar_wait(&bm[1 + b], m_done[1 + b] & 1, wl);  // chunk j was issued before this iteration
        if (ok) m_done[1 + b]++;
        if (__syncthreads_or(!ok)) { failed = true; goto cleanup; }
        tc_after();
        if (tid == 0) {
            if (j + 2 < nchunks) {  // chunk j's MMAs are done with its weight buffer
                load_weights(sW + b * kW3Buf, net.w3 + (size_t)chunk_of(j + 2) * kChunkN * 256, kW3Buf, &bw[b]);
                w_issued[b]++;
            }
            if (j + 1 < nchunks && !issue_chunk(j + 1)) *abort_flag = 1;  // seen after the staging barrier
        }
        // the row's 64 logits go to padded shared memory (32 from each of its two threads),
        // then to global memory as one contiguous 256-byte bulk copy issued by the row's first
        // thread (a warp's direct stores would touch 32 rows)
        const bool store = lb < a.nblocks;
        float* st = reinterpret_cast<float*>(sm + kOffStage + b * kStageBuf) + m * kStageStride;
        {
            const int c = half * 32;
            float v[32];
            tmem_load32(tmem_row + b * kChunkN + c, v);
#pragma unroll
            for (int q = 0; q < 8; q++)
                reinterpret_cast<float4*>(st + c)[q] = make_float4(v[4 * q] + bv[4 * q], v[4 * q + 1] + bv[4 * q + 1],
                                                                   v[4 * q + 2] + bv[4 * q + 2], v[4 * q + 3] + bv[4 * q + 3]);
        }
        async_proxy_fence();
        tc_before();
        __syncthreads();  // the row is staged; every read of this accumulator buffer is done
        if (*abort_flag) { failed = true; goto cleanup; }
        if (half == 0) {
            if (store) {
                float* out = logits + (size_t)lb * S.nout + chunk_of(j) * kChunkN;
                asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(out), "r"(smem_u32(st)),
                             "r"(kChunkN * 4)
                             : "memory");
                asm volatile("cp.async.bulk.commit_group;" ::: "memory");
            }
            // the other buffer, written next, must have been read by its copy (chunk j - 1);
            // the barriers of the next iteration order this before those writes
            asm volatile("cp.async.bulk.wait_group.read 1;" ::: "memory");
        }
    }

cleanup:
    asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");  // this thread's logit rows are written
    __syncthreads();
    if (failed) {
        // give up: record it, then let our own copies and MMAs drain (bounded) before the
        // shared and tensor memory are released
        if (tid == 0) {
            atomicExch(error_flag, 1);  // error_flag[0]
            for (int b = 0; b < 2; b++)
                while (w_done[b] < w_issued[b]) { mbar_wait(&bw[b], w_done[b] & 1); w_done[b]++; }
            for (int b = 0; b < 3; b++)
                for (uint32_t i = m_done[b]; i < m_issued[b]; i++) mbar_wait(&bm[b], i & 1);
        }
        __syncthreads();
    }
    tc_after();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
}

// ------------------------------------------------------------ selection

__device__ __forceinline__ float warp_max(float v) {
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xFFFFFFFFu, v, o));
    return v;
}
__device__ __forceinline__ float warp_sum(float v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
    return v;
}

// Monotone map of a finite float to an unsigned key (larger value, larger key).
__device__ __forceinline__ uint32_t okey(float v) {
    const uint32_t u = __float_as_uint(v);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float okey_value(uint32_t k) {
    return __uint_as_float((k & 0x80000000u) ? (k ^ 0x80000000u) : ~k);
}

// K: length of each lane's list of its best partition classes (>= kmax), so one pass over
// the logits finds them; the warp then merges the lanes' lists with two redux steps per pick.
template <int K>
__global__ void __launch_bounds__(128) k_select(const __grid_constant__ KernelArgs a, const __grid_constant__ Shape S,
                                                 const float* __restrict__ logits, const __grid_constant__ Select sel,
                                                 const __grid_constant__ Routes r) {
    constexpr uint32_t kFull = 0xFFFFFFFFu;
    const int lane = threadIdx.x & 31;
    const int lb = blockIdx.x * 4 + (threadIdx.x >> 5);
    if (lb >= a.nblocks) return;
    const int blk = chunk_block(a, lb);
    if (blk < 0) return;
    const float* z = logits + (size_t)lb * S.nout;
    // First pass: the softmax maximum and each lane's best partitioning logit.  The kmax-th
    // largest of the 32 lane maxima bounds the kmax-th largest logit from below (those lanes'
    // maxima are kmax distinct logits at least that large), so only logits at or above it
    // can be among the kmax best.
    float mx = -3.0e38f, lm = -3.0e38f;
    for (int c = lane; c <= S.p1; c += 32) {
        const float v = z[c];
        mx = fmaxf(mx, v);
        if (c < S.p1) lm = fmaxf(lm, v);
    }
    mx = warp_max(mx);
    float theta = 3.0e38f;
    if (sel.kmax >= 1) {
        int rank = 0;  // lanes ahead of this one in (maximum descending, lane ascending) order
        for (int j = 0; j < 32; j++) {
            const float o = __shfl_sync(kFull, lm, j);
            rank += (o > lm || (o == lm && j < lane)) ? 1 : 0;
        }
        const uint32_t at = __ballot_sync(kFull, rank == sel.kmax - 1);
        theta = __shfl_sync(kFull, lm, __ffs(at) - 1);
    }
    // Second pass: the softmax sum (in the same order as ever) and this lane's K best
    // partitionings among those at or above the bound (value desc, index asc).
    float lv[K];
    int lc[K];
#pragma unroll
    for (int k = 0; k < K; k++) { lv[k] = -3.0e38f; lc[k] = 0x7FFFFFFF; }
    float se = 0.0f;
    for (int c = lane; c <= S.p1; c += 32) {
        const float v = z[c];
        se += __expf(v - mx);
        if (c < S.p1 && v >= theta && v > lv[K - 1]) {  // a lane sees its classes in increasing order
            lv[K - 1] = v; lc[K - 1] = c;
#pragma unroll
            for (int k = K - 1; k > 0; k--)
                if (lv[k] > lv[k - 1]) {
                    const float tv = lv[k]; lv[k] = lv[k - 1]; lv[k - 1] = tv;
                    const int tc = lc[k]; lc[k] = lc[k - 1]; lc[k - 1] = tc;
                }
        }
    }
    se = warp_sum(se);
    const float p1 = __expf(z[S.p1] - mx) / se;
    // the kmax best partitionings, merged from the lanes' lists
    uint16_t picks[kMaxProposals];
    float mass[kMaxProposals];
    int n = 0;
    float acc = p1;
    for (int k = 0; k < sel.kmax; k++) {
        const uint32_t key = lc[0] == 0x7FFFFFFF ? 0u : okey(lv[0]);
        const uint32_t best = __reduce_max_sync(kFull, key);
        if (best == 0u) break;
        const uint32_t ci = __reduce_min_sync(kFull, key == best ? (uint32_t)lc[0] : 0xFFFFFFFFu);
        if ((uint32_t)lc[0] == ci) {  // the winning lane drops it from its list
#pragma unroll
            for (int j = 0; j < K - 1; j++) { lv[j] = lv[j + 1]; lc[j] = lc[j + 1]; }
            lv[K - 1] = -3.0e38f; lc[K - 1] = 0x7FFFFFFF;
        }
        picks[n] = (uint16_t)pick_of_class(S, (int)ci);
        acc += __expf(okey_value(best) - mx) / se;
        mass[n] = acc;
        n++;
    }
    const bool confident = acc >= sel.threshold;
    if (r.confidence && lane == 0) r.confidence[lb] = acc;
    int pos = 0;
    if (lane == 0) pos = atomicAdd(&r.counts[confident ? 0 : 1], 1);
    pos = __shfl_sync(kFull, pos, 0);
    if (!confident) {
        if (lane == 0) { r.full[pos] = blk; r.full_err[pos] = 3e38f; }
        return;
    }
    // propose the shortest best-first prefix whose mass reaches the coverage
    int used = n;
    for (int k = 0; k < n; k++)
        if (mass[k] >= sel.coverage) { used = k + 1; break; }
    if (p1 >= sel.coverage) used = 0;
    const bool skip_p1 = used > 0 && p1 < sel.p1_floor;
    uint32_t heads = skip_p1 ? 0u : 1u;  // block-mode heads the front will read: P = 1 and the proposed counts
    for (int k = 0; k < used; k++) heads |= 2u << (picks[k] >> 10);
    if (lane == 0) {
        r.pruned[pos] = blk;
        PropPicks& pp = r.prop[pos];
        pp.n = (uint16_t)used;
        pp.flags = skip_p1 ? 1 : 0;
        for (int k = 0; k < kMaxProposals; k++) pp.v[k] = k < used ? picks[k] : 0;
        // the work list: slot 0 (P = 1) and one slot per proposed partitioning, by P
        if (!skip_p1) r.pb_list[atomicAdd(&r.counts[2], 1)] = (uint32_t)pos << 5;
        for (int k = 0; k < used; k++) {
            const int p = 1 + (picks[k] >> 10);  // list of P = 2 + (v >> 10)
            r.pb_list[(size_t)p * r.pb_stride + atomicAdd(&r.counts[2 + p], 1)] = ((uint32_t)pos << 5) | (uint32_t)(k + 1);
        }
    }
    // block-mode masks: the kbm best modes of each needed head; lane l holds modes l + 32u.
    // When kbm covers every mode, each needed head's mask is every mode (the ranking would
    // pick them all).
    uint64_t* mk = r.masks + (size_t)pos * 4 * kMaskWords;
    if (sel.kbm >= S.nbm) {
        if (lane < 4 * kMaskWords) {
            const int p = lane / kMaskWords, w = lane % kMaskWords;
            const int lo = w * 64;
            const uint64_t all = S.nbm - lo >= 64 ? ~0ull : S.nbm > lo ? ((1ull << (S.nbm - lo)) - 1) : 0ull;
            mk[lane] = ((heads >> p) & 1) ? all : 0ull;
        }
        return;
    }
    for (int p = 0; p < 4; p++) {
        if (!((heads >> p) & 1)) continue;
        const float* h = z + S.head_base + p * S.nbm_pad;
        float hv[2 * kMaskWords];
        uint32_t picked = 0;
#pragma unroll
        for (int u = 0; u < 2 * kMaskWords; u++) {
            const int c = lane + 32 * u;
            hv[u] = c < S.nbm ? h[c] : 0.0f;
            if (c >= S.nbm) picked |= 1u << u;  // absent: never offered
        }
        // The kbm best modes by (value descending, index ascending), one pick per round.  When
        // kbm is above half the modes, the rounds pick the others instead, worst first (value
        // ascending, index descending): the same set in fewer rounds.
        const int kk = sel.kbm < S.nbm ? sel.kbm : S.nbm;
        const bool worst = 2 * kk > S.nbm;
        const int rounds = worst ? S.nbm - kk : kk;
        for (int k = 0; k < rounds; k++) {
            uint32_t key = 0;
            int mine = -1;
            float mv = 0.0f;
#pragma unroll
            for (int u = 0; u < 2 * kMaskWords; u++)
                if (!((picked >> u) & 1) && (mine < 0 || (worst ? hv[u] <= mv : hv[u] > mv))) { mine = u; mv = hv[u]; }
            if (mine >= 0) key = worst ? ~okey(mv) : okey(mv);
            const uint32_t best = __reduce_max_sync(kFull, key);
            if (best == 0u) break;
            const uint32_t idx = (uint32_t)(lane + 32 * mine);
            const uint32_t ci = worst ? __reduce_max_sync(kFull, key == best ? idx : 0u)
                                      : __reduce_min_sync(kFull, key == best ? idx : 0xFFFFFFFFu);
            if (mine >= 0 && idx == ci) picked |= 1u << mine;
        }
        uint64_t word = 0;
#pragma unroll
        for (int u = 0; u < 2 * kMaskWords; u++) {
            const bool valid = lane + 32 * u < S.nbm;
            const uint32_t chosen = __ballot_sync(kFull, valid && (((picked >> u) & 1) != 0) != worst);
            if (lane == (u >> 1)) word |= (uint64_t)chosen << (32 * (u & 1));
        }
        if (lane < kMaskWords) mk[p * kMaskWords + lane] = word;
    }
}

}  // namespace

cudaError_t configure_mlp() {
    return cudaFuncSetAttribute(k_mlp_logits, cudaFuncAttributeMaxDynamicSharedMemorySize, kMlpSmemBytes);
}

cudaError_t launch_mlp_logits(const KernelArgs& a, const Net& net, float* logits, int* error_flag, cudaStream_t s) {
    const int grid = (a.nblocks + kTileRows - 1) / kTileRows;
    k_mlp_logits<<<grid, kMlpThreads, kMlpSmemBytes, s>>>(a, net, logits, error_flag);
    return cudaGetLastError();
}

cudaError_t launch_select(const KernelArgs& a, const Net& net, const float* logits, const Select& sel, const Routes& r,
                          cudaStream_t s) {
    const int grid = (a.nblocks + 3) / 4;
    if (sel.kmax <= 4) k_select<4><<<grid, 128, 0, s>>>(a, net.s, logits, sel, r);
    else if (sel.kmax <= 8) k_select<8><<<grid, 128, 0, s>>>(a, net.s, logits, sel, r);
    else k_select<16><<<grid, 128, 0, s>>>(a, net.s, logits, sel, r);
    return cudaGetLastError();
}

}  // namespace mlp
}  // namespace astcb200
