// C-ABI of the encoder (include/astcb200.h): context, device buffers, the
// chunked launch sequence and the .astc writer.
//
// Launch sequence per chunk of blocks, all on the context's stream:
//   k_partition_search -> k_front -> k_refine -> k_select_pack
// The per-chunk intermediates (partition picks, 13 partitioned-block records
// and 104 candidate snapshots per block) stay in device memory and are reused
// by every chunk; only the RGBA8 input and the 16-byte blocks cross PCIe.
#include <chrono>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "ctx.h"

using namespace astcb200;

namespace astcb200 {

int cuda_fail(astcb200_ctx* c, cudaError_t e, const char* what) {
    if (c) c->err = std::string(what) + ": " + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? ASTCB200_OOM : ASTCB200_CUDA_ERROR;
}

// Bounded host wait on stream s (astcb200_config.timeout_ms).
int wait_stream(astcb200_ctx* ctx, cudaStream_t s) {
    if (ctx->cfg.timeout_ms == 0) {
        CK(cudaStreamSynchronize(s), "cudaStreamSynchronize");
        return ASTCB200_OK;
    }
    const auto t0 = std::chrono::steady_clock::now();
    for (;;) {
        cudaError_t e = cudaStreamQuery(s);
        if (e == cudaSuccess) return ASTCB200_OK;
        if (e != cudaErrorNotReady) return cuda_fail(ctx, e, "cudaStreamQuery");
        const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        if (ms > ctx->cfg.timeout_ms) { ctx->err = "device work did not finish within timeout_ms"; return ASTCB200_TIMEOUT; }
        std::this_thread::sleep_for(std::chrono::microseconds(200));
    }
}

int HostResults::reserve(astcb200_ctx* ctx) {
    size_t need = 0;
    for (Item& it : items) {
        cudaPointerAttributes at{};
        it.pinned = cudaPointerGetAttributes(&at, it.dst) == cudaSuccess && at.type == cudaMemoryTypeHost;
        cudaGetLastError();  // an unregistered pointer is not an error here
        if (!it.pinned) { it.off = need; need += (it.bytes + 255) & ~(size_t)255; }
    }
    if (need > ctx->stage_cap) {
        // an earlier call that timed out may still be copying into the old buffer
        CK(cudaStreamSynchronize(ctx->stream), "cudaStreamSynchronize");
        if (ctx->h_stage) cudaFreeHost(ctx->h_stage);
        ctx->h_stage = nullptr;
        ctx->stage_cap = 0;
        CK(cudaHostAlloc((void**)&ctx->h_stage, need, cudaHostAllocDefault), "cudaHostAlloc staging");
        ctx->stage_cap = need;
    }
    return ASTCB200_OK;
}

int HostResults::queue(astcb200_ctx* ctx, cudaStream_t s) {
    for (const Item& it : items)
        CK(cudaMemcpyAsync(it.pinned ? it.dst : (void*)(ctx->h_stage + it.off), it.src, it.bytes, cudaMemcpyDeviceToHost, s),
           "D2H results");
    return ASTCB200_OK;
}

void HostResults::finish(astcb200_ctx* ctx) const {
    for (const Item& it : items)
        if (!it.pinned) std::memcpy(it.dst, ctx->h_stage + it.off, it.bytes);
}

// Tables of footprint bx x by on the context's device, built and uploaded on first use.
int get_tables(astcb200_ctx* ctx, int bx, int by, const FootTables** out) {
    for (const FootTables* f : ctx->feet)
        if (f->bx == bx && f->by == by) { *out = f; return ASTCB200_OK; }
    std::vector<uint8_t> blob;
    FootTables* f = new FootTables();
    f->bx = bx; f->by = by;
    if (!build_tables(bx, by, f->L, blob)) { delete f; return ASTCB200_INVALID_FOOTPRINT; }
    cudaError_t e = cudaMalloc((void**)&f->d, blob.size());
    if (e == cudaSuccess) e = cudaMemcpy(f->d, blob.data(), blob.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = configure_kernels(f->L);
    if (e != cudaSuccess) { cudaFree(f->d); delete f; return cuda_fail(ctx, e, "upload tables"); }
    ctx->feet.push_back(f);
    *out = f;
    return ASTCB200_OK;
}

int ensure_scratch(astcb200_ctx* ctx, Scratch& sc, size_t blocks, int slots) {
    int rc;
    if ((rc = ensure_buf(ctx, sc.picks, sc.cap_picks, blocks * sizeof(PartPicks), "cudaMalloc picks"))) return rc;
    if ((rc = ensure_buf(ctx, sc.pbrec, sc.cap_rec, blocks * slots * sizeof(PBRec), "cudaMalloc records"))) return rc;
    return ensure_buf(ctx, sc.snaps, sc.cap_snap, blocks * slots * kNumCand * sizeof(Snap), "cudaMalloc snapshots");
}

void free_scratch(Scratch& sc) {
    cudaFree(sc.picks); cudaFree(sc.pbrec); cudaFree(sc.snaps);
    cudaFree(sc.logits); cudaFree(sc.lists); cudaFree(sc.prop); cudaFree(sc.masks); cudaFree(sc.pbl); cudaFree(sc.full_err); cudaFree(sc.tail);
    sc = Scratch();
}

}  // namespace astcb200

namespace {

int run_search(astcb200_ctx* ctx, const uint8_t* d_img, uint8_t* d_out, uint32_t* d_sym, cudaStream_t s, uint32_t* launches) {
    KernelArgs a;
    std::memset(&a, 0, sizeof(a));
    a.img = d_img;
    a.width = (int)ctx->width; a.height = (int)ctx->height; a.nbx = (int)ctx->nbx; a.nby = (int)ctx->nby;
    a.out_blocks = d_out; a.symbolic = d_sym;
    const bool timing = (ctx->cfg.flags & ASTCB200_FLAG_STAGE_TIMING) != 0;
    const int nchunks = (int)((ctx->nblocks + ctx->chunk - 1) / ctx->chunk);
    int rc = ensure_chunk_scratch(ctx, ctx->scratch, std::min<size_t>(ctx->chunk, ctx->nblocks), ctx->cur);
    if (rc) return rc;
    if ((rc = begin_routes(ctx, nchunks, s))) return rc;
    constexpr int E = kStageIntervals + 1;
    if (timing) {
        if (!ctx->d_work) CK(cudaMalloc((void**)&ctx->d_work, kWorkCounters * sizeof(unsigned long long)), "cudaMalloc work counters");
        CK(cudaMemsetAsync(ctx->d_work, 0, kWorkCounters * sizeof(unsigned long long), s), "reset work counters");
        a.work = ctx->d_work;
        while ((int)ctx->stage_ev.size() < E * nchunks) {
            cudaEvent_t e;
            CK(cudaEventCreate(&e), "cudaEventCreate");
            ctx->stage_ev.push_back(e);
        }
        ctx->stage_kind.assign((size_t)kStageIntervals * nchunks, -1);
        ctx->stage_chunks = nchunks;
    }
    uint32_t n = 0;
    int c = 0;
    for (uint32_t first = 0; first < ctx->nblocks; first += ctx->chunk, c++) {
        a.block_first = (int)first;
        a.nblocks = (int)std::min<uint32_t>(ctx->chunk, ctx->nblocks - first);
        if ((rc = enqueue_chunk(ctx, a, ctx->cur, ctx->scratch, s, timing ? &ctx->stage_ev[(size_t)E * c] : nullptr,
                                timing ? &ctx->stage_kind[(size_t)kStageIntervals * c] : nullptr, &n,
                                (uint64_t)ctx->width * ctx->height < (uint64_t)mlp::kMinProposalTexels)))
            return rc;
    }
    if (launches) *launches = n;
    return ASTCB200_OK;
}

}  // namespace

extern "C" {

const char* astcb200_status_string(int s) {
    switch (s) {
        case ASTCB200_OK: return "ok";
        case ASTCB200_INVALID_FOOTPRINT: return "invalid block footprint";
        case ASTCB200_BAD_ARG: return "bad argument";
        case ASTCB200_OOM: return "out of memory";
        case ASTCB200_CUDA_ERROR: return "CUDA error";
        case ASTCB200_TIMEOUT: return "timeout";
        case ASTCB200_NO_IMAGE: return "no image configured";
        case ASTCB200_IO_ERROR: return "file write failed";
        case ASTCB200_TOO_LARGE: return "request exceeds the no-allocation scratch (at most 2048 blocks per call)";
        default: return "unknown status";
    }
}

const char* astcb200_last_error(const astcb200_ctx* ctx) { return ctx ? ctx->err.c_str() : ""; }

int astcb200_create(astcb200_ctx** out, int device_ordinal, const astcb200_config* cfg) {
    if (!out) return ASTCB200_BAD_ARG;
    *out = nullptr;
    astcb200_ctx* ctx = new (std::nothrow) astcb200_ctx();
    if (!ctx) return ASTCB200_OOM;
    if (cfg && cfg->struct_size) {
        std::memcpy(&ctx->cfg, cfg, std::min<size_t>(cfg->struct_size, sizeof(astcb200_config)));
    }
    ctx->chunk = ctx->cfg.chunk_blocks ? ctx->cfg.chunk_blocks : 65536;
    ctx->device = device_ordinal;
    int rc = ASTCB200_OK;
    DeviceGuard dg(device_ordinal);
    cudaError_t e = dg.err;
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&ctx->ev0);
    if (e == cudaSuccess) e = cudaEventCreate(&ctx->ev1);
    if (e != cudaSuccess) { rc = cuda_fail(ctx, e, "create"); astcb200_destroy(ctx); return rc; }
    *out = ctx;
    return ASTCB200_OK;
}

int astcb200_destroy(astcb200_ctx* ctx) {
    if (!ctx) return ASTCB200_BAD_ARG;
    DeviceGuard dg(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    release_batches(ctx);
    free_scratch(ctx->scratch);
    for (FootTables* f : ctx->feet) { cudaFree(f->d); delete f; }
    for (NetDev* nd : ctx->nets) { cudaFree(nd->mem); delete nd; }
    cudaFree(ctx->d_counts); cudaFree(ctx->d_mlp_error); cudaFree(ctx->d_work);
    cudaFree(ctx->d_img); cudaFree(ctx->d_out); cudaFree(ctx->d_sym);
    if (ctx->h_stage) cudaFreeHost(ctx->h_stage);
    if (ctx->ev0) cudaEventDestroy(ctx->ev0);
    if (ctx->ev1) cudaEventDestroy(ctx->ev1);
    for (cudaEvent_t e : ctx->stage_ev) cudaEventDestroy(e);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return ASTCB200_OK;
}

int astcb200_set_image(astcb200_ctx* ctx, uint32_t width, uint32_t height, uint8_t block_x, uint8_t block_y) {
    if (!ctx || width == 0 || height == 0) return ASTCB200_BAD_ARG;
    if (!valid_footprint(block_x, block_y)) return ASTCB200_INVALID_FOOTPRINT;
    const uint64_t nbx = (width + block_x - 1) / block_x, nby = (height + block_y - 1) / block_y;
    if (nbx * nby > 0x7FFFFFFFull) return ASTCB200_BAD_ARG;
    ASTCB200_DEVICE_SCOPE(ctx);
    const FootTables* ft = nullptr;
    int rc = get_tables(ctx, block_x, block_y, &ft);
    if (rc) return rc;
    ctx->cur = ft;
    ctx->width = width; ctx->height = height; ctx->bx = block_x; ctx->by = block_y;
    ctx->nbx = (uint32_t)nbx; ctx->nby = (uint32_t)nby; ctx->nblocks = (uint32_t)(nbx * nby);
    ctx->have_image = true;
    return ASTCB200_OK;
}

int astcb200_set_timeout(astcb200_ctx* ctx, uint32_t timeout_ms) {
    if (!ctx) return ASTCB200_BAD_ARG;
    ctx->cfg.timeout_ms = timeout_ms;
    return ASTCB200_OK;
}

int astcb200_blocks(const astcb200_ctx* ctx, uint32_t* bxo, uint32_t* byo) {
    if (!ctx || !bxo || !byo) return ASTCB200_BAD_ARG;
    if (!ctx->have_image) return ASTCB200_NO_IMAGE;
    *bxo = ctx->nbx; *byo = ctx->nby;
    return ASTCB200_OK;
}

int astcb200_encode_device(astcb200_ctx* ctx, const uint8_t* d_rgba8, uint8_t* d_out, void* stream) {
    if (!ctx || !d_rgba8 || !d_out) return ASTCB200_BAD_ARG;
    if (!ctx->have_image) return ASTCB200_NO_IMAGE;
    if (((uintptr_t)d_rgba8 & 3) || ((uintptr_t)d_out & 15)) return ASTCB200_BAD_ARG;
    ASTCB200_DEVICE_SCOPE(ctx);
    cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
    return run_search(ctx, d_rgba8, d_out, nullptr, s, nullptr);
}

static int encode_host(astcb200_ctx* ctx, const uint8_t* rgba8, uint8_t* out_blocks, uint32_t* symbolic, astcb200_stats* stats) {
    const auto t0 = std::chrono::steady_clock::now();
    ASTCB200_DEVICE_SCOPE(ctx);
    const size_t in_bytes = (size_t)ctx->width * ctx->height * 4, out_bytes = (size_t)ctx->nblocks * 16;
    int rc;
    if ((rc = ensure_buf(ctx, ctx->d_img, ctx->img_cap, in_bytes, "cudaMalloc image"))) return rc;
    if ((rc = ensure_buf(ctx, ctx->d_out, ctx->out_cap, out_bytes, "cudaMalloc output"))) return rc;
    if (symbolic && (rc = ensure_buf(ctx, ctx->d_sym, ctx->sym_cap, (size_t)ctx->nblocks * 108 * 4, "cudaMalloc symbolic"))) return rc;
    HostResults res;
    if (out_blocks) res.add(out_blocks, ctx->d_out, out_bytes);
    if (symbolic) res.add(symbolic, ctx->d_sym, (size_t)ctx->nblocks * 108 * 4);
    if ((rc = res.reserve(ctx))) return rc;
    CK(cudaMemcpyAsync(ctx->d_img, rgba8, in_bytes, cudaMemcpyHostToDevice, ctx->stream), "H2D image");
    CK(cudaEventRecord(ctx->ev0, ctx->stream), "event");
    uint32_t launches = 0;
    if ((rc = run_search(ctx, ctx->d_img, ctx->d_out, symbolic ? ctx->d_sym : nullptr, ctx->stream, &launches))) return rc;
    CK(cudaEventRecord(ctx->ev1, ctx->stream), "event");
    if ((rc = res.queue(ctx, ctx->stream))) return rc;
    if ((rc = wait_stream(ctx, ctx->stream))) return rc;
    res.finish(ctx);
    if (stats) {
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
        stats->ms_device = ms;
        stats->ms_wall = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        stats->blocks = ctx->nblocks;
        stats->h2d_bytes = in_bytes;
        stats->d2h_bytes = (out_blocks ? out_bytes : 0) + (symbolic ? (size_t)ctx->nblocks * 108 * 4 : 0);
        stats->launches = launches;
    }
    return ASTCB200_OK;
}

int astcb200_encode(astcb200_ctx* ctx, const uint8_t* rgba8, uint8_t* out_blocks, size_t out_len, astcb200_stats* stats) {
    if (!ctx || !rgba8 || !out_blocks) return ASTCB200_BAD_ARG;
    if (!ctx->have_image) return ASTCB200_NO_IMAGE;
    if (out_len < (size_t)ctx->nblocks * 16) return ASTCB200_BAD_ARG;
    return encode_host(ctx, rgba8, out_blocks, nullptr, stats);
}

int astcb200_encode_symbolic(astcb200_ctx* ctx, const uint8_t* rgba8, uint32_t* symbolic, size_t words) {
    if (!ctx || !rgba8 || !symbolic) return ASTCB200_BAD_ARG;
    if (!ctx->have_image) return ASTCB200_NO_IMAGE;
    if (words < (size_t)ctx->nblocks * 108) return ASTCB200_BAD_ARG;
    return encode_host(ctx, rgba8, nullptr, symbolic, nullptr);
}

int astcb200_search_stages(astcb200_ctx* ctx, const uint8_t* rgba8, void* picks, size_t picks_bytes, void* records,
                           size_t records_bytes, void* snapshots, size_t snapshots_bytes) {
    if (!ctx || !rgba8 || !picks || !records) return ASTCB200_BAD_ARG;
    if (!ctx->have_image) return ASTCB200_NO_IMAGE;
    const size_t nb = ctx->nblocks;
    if (nb > ctx->chunk || picks_bytes < nb * sizeof(PartPicks) || records_bytes < nb * kSlotsPerBlock * sizeof(PBRec) ||
        (snapshots && snapshots_bytes < nb * kSlotsPerBlock * kNumCand * sizeof(Snap)))
        return ASTCB200_BAD_ARG;
    ASTCB200_DEVICE_SCOPE(ctx);
    const size_t in_bytes = (size_t)ctx->width * ctx->height * 4;
    int rc;
    if ((rc = ensure_buf(ctx, ctx->d_img, ctx->img_cap, in_bytes, "cudaMalloc image"))) return rc;
    if ((rc = ensure_scratch(ctx, ctx->scratch, nb, kSlotsPerBlock))) return rc;
    CK(cudaMemcpyAsync(ctx->d_img, rgba8, in_bytes, cudaMemcpyHostToDevice, ctx->stream), "H2D image");
    KernelArgs a;
    std::memset(&a, 0, sizeof(a));
    a.img = ctx->d_img;
    a.width = (int)ctx->width; a.height = (int)ctx->height; a.nbx = (int)ctx->nbx; a.nby = (int)ctx->nby;
    a.block_first = 0; a.nblocks = (int)nb;
    a.tables = ctx->cur->d; a.L = ctx->cur->L;
    a.picks = ctx->scratch.picks; a.pbrec = ctx->scratch.pbrec; a.snaps = ctx->scratch.snaps;
    a.slots = kSlotsPerBlock; a.topn = kNumCand;
    a.fixed = (ctx->cfg.flags & ASTCB200_FLAG_FIXED_SEMANTICS) ? 1 : 0;
    CK(launch_partition_search(a, ctx->stream), "k_partition_search");
    CK(launch_front(a, ctx->stream), "k_front");
    if (snapshots) {
        CK(launch_refine(a, ctx->stream), "k_refine");
        CK(cudaMemcpyAsync(snapshots, a.snaps, nb * kSlotsPerBlock * kNumCand * sizeof(Snap), cudaMemcpyDeviceToHost, ctx->stream),
           "D2H snapshots");
    }
    CK(cudaMemcpyAsync(picks, a.picks, nb * sizeof(PartPicks), cudaMemcpyDeviceToHost, ctx->stream), "D2H picks");
    CK(cudaMemcpyAsync(records, a.pbrec, nb * kSlotsPerBlock * sizeof(PBRec), cudaMemcpyDeviceToHost, ctx->stream), "D2H records");
    return wait_stream(ctx, ctx->stream);
}

int astcb200_stage_times(astcb200_ctx* ctx, float* ms4, uint32_t* n4) {
    if (!ctx || !ms4) return ASTCB200_BAD_ARG;
    for (int k = 0; k < 4; k++) { ms4[k] = 0.0f; if (n4) n4[k] = 0; }
    if (ctx->stage_chunks == 0) return ASTCB200_OK;
    constexpr int E = kStageIntervals + 1;
    for (int c = 0; c < ctx->stage_chunks; c++)
        for (int i = 0; i < kStageIntervals; i++) {
            const int kk = ctx->stage_kind[(size_t)kStageIntervals * c + i];
            if (kk < 0) break;
            const int k = kk & 3;
            cudaEvent_t e1 = ctx->stage_ev[(size_t)E * c + i + 1];
            CK(cudaEventSynchronize(e1), "stage event");
            float ms = 0.0f;
            CK(cudaEventElapsedTime(&ms, ctx->stage_ev[(size_t)E * c + i], e1), "cudaEventElapsedTime");
            ms4[k] += ms;
            if (n4) n4[k] += 1 + (kk >> 2);
        }
    return ASTCB200_OK;
}

int astcb200_stage_times_detail(astcb200_ctx* ctx, float* ms9, int32_t* stage9) {
    if (!ctx || !ms9) return ASTCB200_BAD_ARG;
    for (int i = 0; i < kStageIntervals; i++) { ms9[i] = 0.0f; if (stage9) stage9[i] = -1; }
    constexpr int E = kStageIntervals + 1;
    for (int c = 0; c < ctx->stage_chunks; c++)
        for (int i = 0; i < kStageIntervals; i++) {
            const int k = ctx->stage_kind[(size_t)kStageIntervals * c + i];
            if (k < 0) break;
            cudaEvent_t e1 = ctx->stage_ev[(size_t)E * c + i + 1];
            CK(cudaEventSynchronize(e1), "stage event");
            float ms = 0.0f;
            CK(cudaEventElapsedTime(&ms, ctx->stage_ev[(size_t)E * c + i], e1), "cudaEventElapsedTime");
            ms9[i] += ms;
            if (stage9) stage9[i] = k & 3;
        }
    return ASTCB200_OK;
}

int astcb200_work_counters(astcb200_ctx* ctx, uint64_t* counters16) {
    if (!ctx || !counters16) return ASTCB200_BAD_ARG;
    for (int i = 0; i < kWorkCounters; i++) counters16[i] = 0;
    if (!ctx->d_work) return ASTCB200_OK;
    ASTCB200_DEVICE_SCOPE(ctx);
    CK(cudaDeviceSynchronize(), "cudaDeviceSynchronize");
    CK(cudaMemcpy(counters16, ctx->d_work, kWorkCounters * sizeof(uint64_t), cudaMemcpyDeviceToHost), "read work counters");
    return ASTCB200_OK;
}

// astc_store.cpp:18-62: magic 0x5CA1AB13, block dims, 24-bit image dims, then the blocks.
// The .astc header (astc_store.cpp:18-62): magic, block size, image size (24-bit little-endian).
static void astc_header(uint32_t bx, uint32_t by, uint32_t dx, uint32_t dy, uint8_t* h) {
    const uint32_t bz = 1, dz = 1, magic = 0x5CA1AB13u;
    const uint8_t v[16] = {(uint8_t)(magic & 0xFF), (uint8_t)((magic >> 8) & 0xFF), (uint8_t)((magic >> 16) & 0xFF), (uint8_t)(magic >> 24),
                           (uint8_t)bx, (uint8_t)by, (uint8_t)bz,
                           (uint8_t)(dx & 0xFF), (uint8_t)((dx >> 8) & 0xFF), (uint8_t)((dx >> 16) & 0xFF),
                           (uint8_t)(dy & 0xFF), (uint8_t)((dy >> 8) & 0xFF), (uint8_t)((dy >> 16) & 0xFF),
                           (uint8_t)(dz & 0xFF), (uint8_t)((dz >> 8) & 0xFF), (uint8_t)((dz >> 16) & 0xFF)};
    std::memcpy(h, v, 16);
}

int astcb200_store_image(uint32_t bx, uint32_t by, uint32_t dx, uint32_t dy, const uint8_t* data, size_t len, const char* filename) {
    if (!filename || (!data && len)) return ASTCB200_BAD_ARG;
    uint8_t h[16];
    astc_header(bx, by, dx, dy, h);
    FILE* f = std::fopen(filename, "wb");
    if (!f) return ASTCB200_IO_ERROR;
    bool ok = std::fwrite(h, 1, 16, f) == 16 && (len == 0 || std::fwrite(data, 1, len, f) == len);
    ok = (std::fclose(f) == 0) && ok;
    return ok ? ASTCB200_OK : ASTCB200_IO_ERROR;
}

int astcb200_astc_containers_device(const astcb200_astc_image* images, uint32_t n, void* cuda_stream) {
    if (!images && n) return ASTCB200_BAD_ARG;
    for (uint32_t i = 0; i < n; i++) {  // every image is checked before anything is queued
        const astcb200_astc_image& m = images[i];
        if (!valid_footprint(m.block_x, m.block_y)) return ASTCB200_INVALID_FOOTPRINT;
        if (!m.d_blocks || !m.host_out || m.width == 0 || m.height == 0 || m.width >= (1u << 24) || m.height >= (1u << 24))
            return ASTCB200_BAD_ARG;
        const uint64_t blocks = (uint64_t)((m.width + m.block_x - 1) / m.block_x) * ((m.height + m.block_y - 1) / m.block_y);
        if (m.out_len < 16 + 16 * blocks) return ASTCB200_BAD_ARG;
    }
    const cudaStream_t s = (cudaStream_t)cuda_stream;
    for (uint32_t i = 0; i < n; i++) {
        const astcb200_astc_image& m = images[i];
        const size_t blocks = (size_t)((m.width + m.block_x - 1) / m.block_x) * ((m.height + m.block_y - 1) / m.block_y);
        astc_header(m.block_x, m.block_y, m.width, m.height, m.host_out);
        if (cudaMemcpyAsync(m.host_out + 16, m.d_blocks, blocks * 16, cudaMemcpyDeviceToHost, s) != cudaSuccess)
            return ASTCB200_CUDA_ERROR;
    }
    return ASTCB200_OK;
}

}  // extern "C"
