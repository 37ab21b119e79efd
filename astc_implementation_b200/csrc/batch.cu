// Batched encoding: many textures of any sizes and footprints in one call.
//
// The blocks of all textures that share a footprint form one work queue (one
// TexSeg per texture, block indices consecutive across the textures), searched
// by the same four kernels as a single image, chunk by chunk.  Chunks are
// spread round-robin over up to kMaxStreams concurrent streams, each with its
// own scratch, so small textures and the tails of one footprint's queue overlap
// with the others instead of leaving SMs idle.  The whole launch sequence of a
// batch shape (texture sizes and footprints) is captured once into a CUDA
// graph; later batches of that shape upload their texture descriptors and
// replay it.  astcb200_autotune_batch picks chunk size and stream count per
// shape by timing the candidates on the batch itself.
#include <algorithm>
#include <chrono>
#include <cstring>

#include "ctx.h"

using namespace astcb200;

namespace astcb200 {

constexpr uint32_t kMaxStreams = 4;

void release_batches(astcb200_ctx* ctx) {
    for (auto& kv : ctx->graphs)
        if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
    ctx->graphs.clear();
    for (Scratch& sc : ctx->bscratch) free_scratch(sc);
    ctx->bscratch.clear();
    for (cudaStream_t s : ctx->branch) cudaStreamDestroy(s);
    ctx->branch.clear();
    for (cudaEvent_t e : ctx->fork_ev) cudaEventDestroy(e);
    for (cudaEvent_t e : ctx->join_ev) cudaEventDestroy(e);
    ctx->fork_ev.clear();
    ctx->join_ev.clear();
    cudaFree(ctx->d_segs); cudaFree(ctx->d_bin); cudaFree(ctx->d_bout);
    ctx->d_segs = nullptr; ctx->d_bin = nullptr; ctx->d_bout = nullptr;
    ctx->segs_cap = ctx->bin_cap = ctx->bout_cap = 0;
}

namespace {

struct Group {
    const FootTables* ft;
    uint32_t first_seg, nsegs, nblocks;
    bool full_only;  // textures below mlp::kMinProposalTexels: the full search
};

struct Plan {
    BatchShape shape;
    std::vector<Group> groups;
    std::vector<TexSeg> segs;      // grouped by footprint; block_base counts from the group's start
    std::vector<uint32_t> tex_of;  // segs[i] describes textures[tex_of[i]]
    uint32_t max_group_blocks = 0;
};

size_t blocks_of(const astcb200_texture& t) {
    return (size_t)((t.width + t.block_x - 1) / t.block_x) * ((t.height + t.block_y - 1) / t.block_y);
}

constexpr size_t align256(size_t v) { return (v + 255) & ~size_t(255); }

int make_plan(astcb200_ctx* ctx, const astcb200_texture* tex, uint32_t n, bool device_ptrs, Plan& p) {
    if (!tex || n == 0) return ASTCB200_BAD_ARG;
    p.shape.assign(1, n);
    std::vector<std::pair<int, int>> feet;
    for (uint32_t i = 0; i < n; i++) {
        const astcb200_texture& t = tex[i];
        if (!t.rgba8 || !t.out_blocks || t.width == 0 || t.height == 0) return ASTCB200_BAD_ARG;
        if (!valid_footprint(t.block_x, t.block_y)) return ASTCB200_INVALID_FOOTPRINT;
        if (t.out_len < blocks_of(t) * 16) return ASTCB200_BAD_ARG;
        if (device_ptrs && (((uintptr_t)t.rgba8 & 3) || ((uintptr_t)t.out_blocks & 15))) return ASTCB200_BAD_ARG;
        p.shape.push_back(t.width); p.shape.push_back(t.height);
        p.shape.push_back(t.block_x * 256u + t.block_y);
        const std::pair<int, int> fp(t.block_x, t.block_y);
        if (std::find(feet.begin(), feet.end(), fp) == feet.end()) feet.push_back(fp);
    }
    // one queue per footprint and texture class (small textures take the full search)
    for (const auto& fp : feet)
      for (int small = 0; small < 2; small++) {
        Group g{nullptr, (uint32_t)p.segs.size(), 0, 0, small == 1};
        int rc = get_tables(ctx, fp.first, fp.second, &g.ft);
        if (rc) return rc;
        uint64_t base = 0;
        for (uint32_t i = 0; i < n; i++) {
            const astcb200_texture& t = tex[i];
            if (t.block_x != fp.first || t.block_y != fp.second) continue;
            if (((uint64_t)t.width * t.height < (uint64_t)mlp::kMinProposalTexels) != (small == 1)) continue;
            TexSeg s;
            s.img = t.rgba8; s.out = t.out_blocks;
            s.width = (int)t.width; s.height = (int)t.height;
            s.nbx = (int)((t.width + t.block_x - 1) / t.block_x);
            s.block_base = (int)base;
            base += blocks_of(t);
            if (base > 0x7FFFFFFFull) return ASTCB200_BAD_ARG;
            p.segs.push_back(s);
            p.tex_of.push_back(i);
        }
        g.nsegs = (uint32_t)p.segs.size() - g.first_seg;
        if (g.nsegs == 0) continue;
        g.nblocks = (uint32_t)base;
        p.max_group_blocks = std::max(p.max_group_blocks, g.nblocks);
        p.groups.push_back(g);
      }
    return ASTCB200_OK;
}

// Streams, events and per-stream scratch for `streams` streams of `chunk` blocks.
int prepare(astcb200_ctx* ctx, const Plan& p, uint32_t chunk, uint32_t streams, cudaStream_t s) {
    while (ctx->branch.size() + 1 < streams) {
        cudaStream_t s;
        CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "cudaStreamCreate");
        ctx->branch.push_back(s);
    }
    while (ctx->fork_ev.size() < kMaxStreams) {
        cudaEvent_t e1, e2;
        CK(cudaEventCreateWithFlags(&e1, cudaEventDisableTiming), "cudaEventCreate");
        ctx->fork_ev.push_back(e1);
        CK(cudaEventCreateWithFlags(&e2, cudaEventDisableTiming), "cudaEventCreate");
        ctx->join_ev.push_back(e2);
    }
    if (ctx->bscratch.size() < streams) ctx->bscratch.resize(streams);
    const size_t need = std::min<size_t>(chunk, p.max_group_blocks);
    for (uint32_t i = 0; i < streams; i++)
        for (const Group& g : p.groups) {  // sized for the largest need over the footprints
            int rc = ensure_chunk_scratch(ctx, ctx->bscratch[i], need, g.ft);
            if (rc) return rc;
        }
    size_t units = 0;
    for (const Group& g : p.groups) units += (g.nblocks + chunk - 1) / chunk;
    int rc = begin_routes(ctx, units, s);
    if (rc) return rc;
    return ensure_buf(ctx, ctx->d_segs, ctx->segs_cap, p.segs.size() * sizeof(TexSeg), "cudaMalloc batch descriptors");
}

// Device buffers a launch sequence with `streams` streams bakes in.
std::vector<const void*> baked_buffers(const astcb200_ctx* ctx, uint32_t streams) {
    std::vector<const void*> v{ctx->d_segs, ctx->d_counts, ctx->d_mlp_error};
    for (uint32_t i = 0; i < streams; i++) {
        const Scratch& sc = ctx->bscratch[i];
        for (const void* q : {(const void*)sc.picks, (const void*)sc.pbrec, (const void*)sc.snaps, (const void*)sc.logits,
                              (const void*)sc.lists, (const void*)sc.prop, (const void*)sc.masks, (const void*)sc.pbl, (const void*)sc.full_err})
            v.push_back(q);
    }
    return v;
}

// Queues the batch's kernels: chunk c of the footprint queues goes to stream c % streams.
int enqueue(astcb200_ctx* ctx, const Plan& p, cudaStream_t s, uint32_t chunk, uint32_t streams, uint32_t* launches) {
    cudaStream_t st[kMaxStreams];
    st[0] = s;
    for (uint32_t i = 1; i < streams; i++) st[i] = ctx->branch[i - 1];
    if (streams > 1) {
        CK(cudaEventRecord(ctx->fork_ev[0], s), "fork event");
        for (uint32_t i = 1; i < streams; i++) CK(cudaStreamWaitEvent(st[i], ctx->fork_ev[0], 0), "fork wait");
    }
    uint32_t unit = 0, n = 0;
    ctx->counts_used = 0;
    for (const Group& g : p.groups) {
        for (uint32_t first = 0; first < g.nblocks; first += chunk, unit++) {
            const uint32_t k = unit % streams;
            KernelArgs a;
            std::memset(&a, 0, sizeof(a));
            a.segs = ctx->d_segs + g.first_seg;
            a.nsegs = (int)g.nsegs;
            a.block_first = (int)first;
            a.nblocks = (int)std::min<uint32_t>(chunk, g.nblocks - first);
            int rc = enqueue_chunk(ctx, a, g.ft, ctx->bscratch[k], st[k], nullptr, nullptr, &n, g.full_only);
            if (rc) return rc;
        }
    }
    if (streams > 1) {
        for (uint32_t i = 1; i < streams; i++) {
            CK(cudaEventRecord(ctx->join_ev[i], st[i]), "join event");
            CK(cudaStreamWaitEvent(s, ctx->join_ev[i], 0), "join wait");
        }
    }
    if (launches) *launches = n;
    return ASTCB200_OK;
}

BatchTuning default_tuning(astcb200_ctx* ctx, const Plan& p) {
    auto it = ctx->tuned.find(p.shape);
    if (it != ctx->tuned.end()) return it->second;
    BatchTuning t;
    t.chunk = ctx->chunk;
    uint32_t units = 0;
    for (const Group& g : p.groups) units += (g.nblocks + t.chunk - 1) / t.chunk;
    t.streams = std::max<uint32_t>(1, std::min<uint32_t>(3, units));
    return t;
}

// Uploads the descriptors and queues (or replays) the batch on stream s.
int launch_plan(astcb200_ctx* ctx, Plan& p, cudaStream_t s, const BatchTuning& tu, bool use_graph, uint32_t* launches) {
    int rc = prepare(ctx, p, tu.chunk, tu.streams, s);
    if (rc) return rc;
    // pageable source: the descriptors are consumed before the call returns
    CK(cudaMemcpyAsync(ctx->d_segs, p.segs.data(), p.segs.size() * sizeof(TexSeg), cudaMemcpyHostToDevice, s), "upload batch descriptors");
    if (!use_graph) return enqueue(ctx, p, s, tu.chunk, tu.streams, launches);

    const std::vector<const void*> bufs = baked_buffers(ctx, tu.streams);
    auto it = ctx->graphs.find(p.shape);
    if (it != ctx->graphs.end() && (it->second.chunk != tu.chunk || it->second.streams != tu.streams || it->second.bufs != bufs)) {
        cudaGraphExecDestroy(it->second.exec);
        ctx->graphs.erase(it);
        it = ctx->graphs.end();
    }
    if (it == ctx->graphs.end()) {
        BatchGraph bg;
        bg.chunk = tu.chunk; bg.streams = tu.streams; bg.bufs = bufs;
        CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
        rc = enqueue(ctx, p, s, tu.chunk, tu.streams, &bg.launches);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(s, &g);
        if (rc) { if (g) cudaGraphDestroy(g); return rc; }
        if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaStreamEndCapture");
        bg.routes = ctx->counts_used;
        e = cudaGraphInstantiate(&bg.exec, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaGraphInstantiate");
        it = ctx->graphs.emplace(p.shape, bg).first;
    }
    CK(cudaGraphLaunch(it->second.exec, s), "cudaGraphLaunch");
    ctx->counts_used = it->second.routes;
    if (launches) *launches = it->second.launches;
    return ASTCB200_OK;
}

__global__ void k_downsample(const uchar4* __restrict__ src, int w, int h, uchar4* __restrict__ dst, int dw, int dh) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= dw || y >= dh) return;
    const int x0 = min(2 * x, w - 1), x1 = min(2 * x + 1, w - 1);
    const int y0 = min(2 * y, h - 1), y1 = min(2 * y + 1, h - 1);
    const uchar4 a = src[(size_t)y0 * w + x0], b = src[(size_t)y0 * w + x1];
    const uchar4 c = src[(size_t)y1 * w + x0], d = src[(size_t)y1 * w + x1];
    dst[(size_t)y * dw + x] = make_uchar4((uint8_t)((a.x + b.x + c.x + d.x + 2) >> 2), (uint8_t)((a.y + b.y + c.y + d.y + 2) >> 2),
                                          (uint8_t)((a.z + b.z + c.z + d.z + 2) >> 2), (uint8_t)((a.w + b.w + c.w + d.w + 2) >> 2));
}

}  // namespace
}  // namespace astcb200

extern "C" {

int astcb200_encode_batch_device(astcb200_ctx* ctx, const astcb200_texture* textures, uint32_t n, void* cuda_stream) {
    if (!ctx) return ASTCB200_BAD_ARG;
    ASTCB200_DEVICE_SCOPE(ctx);
    Plan p;
    int rc = make_plan(ctx, textures, n, true, p);
    if (rc) return rc;
    cudaStream_t s = cuda_stream ? (cudaStream_t)cuda_stream : ctx->stream;
    return launch_plan(ctx, p, s, default_tuning(ctx, p), !(ctx->cfg.flags & ASTCB200_FLAG_NO_GRAPH), nullptr);
}

int astcb200_encode_batch(astcb200_ctx* ctx, const astcb200_texture* textures, uint32_t n, astcb200_stats* stats) {
    if (!ctx) return ASTCB200_BAD_ARG;
    const auto t0 = std::chrono::steady_clock::now();
    ASTCB200_DEVICE_SCOPE(ctx);
    Plan check;
    int rc = make_plan(ctx, textures, n, false, check);
    if (rc) return rc;
    size_t in_bytes = 0, out_bytes = 0, in_need = 0, out_need = 0;
    for (uint32_t i = 0; i < n; i++) {
        in_need += align256((size_t)textures[i].width * textures[i].height * 4);
        out_need += align256(blocks_of(textures[i]) * 16);
    }
    if ((rc = ensure_buf(ctx, ctx->d_bin, ctx->bin_cap, in_need, "cudaMalloc batch input"))) return rc;
    if ((rc = ensure_buf(ctx, ctx->d_bout, ctx->bout_cap, out_need, "cudaMalloc batch output"))) return rc;
    std::vector<astcb200_texture> dev(textures, textures + n);
    size_t io = 0, oo = 0;
    for (uint32_t i = 0; i < n; i++) {
        const size_t ib = (size_t)textures[i].width * textures[i].height * 4, ob = blocks_of(textures[i]) * 16;
        CK(cudaMemcpyAsync(ctx->d_bin + io, textures[i].rgba8, ib, cudaMemcpyHostToDevice, ctx->stream), "H2D texture");
        dev[i].rgba8 = ctx->d_bin + io;
        dev[i].out_blocks = ctx->d_bout + oo;
        dev[i].out_len = ob;
        io += align256(ib); oo += align256(ob);
        in_bytes += ib; out_bytes += ob;
    }
    HostResults res;
    for (uint32_t i = 0; i < n; i++) res.add(textures[i].out_blocks, dev[i].out_blocks, dev[i].out_len);
    if ((rc = res.reserve(ctx))) return rc;
    Plan p;
    if ((rc = make_plan(ctx, dev.data(), n, true, p))) return rc;
    CK(cudaEventRecord(ctx->ev0, ctx->stream), "event");
    uint32_t launches = 0;
    if ((rc = launch_plan(ctx, p, ctx->stream, default_tuning(ctx, p), !(ctx->cfg.flags & ASTCB200_FLAG_NO_GRAPH), &launches))) return rc;
    CK(cudaEventRecord(ctx->ev1, ctx->stream), "event");
    if ((rc = res.queue(ctx, ctx->stream))) return rc;
    if ((rc = wait_stream(ctx, ctx->stream))) return rc;
    res.finish(ctx);
    if (stats) {
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
        stats->ms_device = ms;
        stats->ms_wall = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        uint64_t blocks = 0;
        for (uint32_t i = 0; i < n; i++) blocks += blocks_of(textures[i]);
        stats->blocks = blocks;
        stats->h2d_bytes = in_bytes;
        stats->d2h_bytes = out_bytes;
        stats->launches = launches;
    }
    return ASTCB200_OK;
}

int astcb200_autotune_batch(astcb200_ctx* ctx, const astcb200_texture* textures, uint32_t n, astcb200_tuning* best,
                            astcb200_tuning* tried, uint32_t max_tried, uint32_t* n_tried) {
    if (!ctx || !best) return ASTCB200_BAD_ARG;
    ASTCB200_DEVICE_SCOPE(ctx);
    Plan p;
    int rc = make_plan(ctx, textures, n, true, p);
    if (rc) return rc;
    static const uint32_t kChunks[] = {32768, 65536, 131072};
    std::vector<BatchTuning> cands;
    bool covered = false;  // chunks beyond the largest queue all behave alike: keep the first
    for (uint32_t c : kChunks) {
        if (covered) break;
        covered = c >= p.max_group_blocks;
        uint32_t units = 0;
        for (const Group& g : p.groups) units += (g.nblocks + c - 1) / c;
        for (uint32_t st = 1; st <= kMaxStreams && st <= units; st++) cands.push_back({c, st});
    }
    uint32_t nt = 0;
    double best_ms = 1e300;
    BatchTuning win = cands.front();
    for (const BatchTuning& tu : cands) {
        if ((rc = launch_plan(ctx, p, ctx->stream, tu, false, nullptr))) return rc;  // warm-up
        CK(cudaEventRecord(ctx->ev0, ctx->stream), "event");
        const int reps = 1;
        for (int r = 0; r < reps; r++)
            if ((rc = launch_plan(ctx, p, ctx->stream, tu, false, nullptr))) return rc;
        CK(cudaEventRecord(ctx->ev1, ctx->stream), "event");
        if ((rc = wait_stream(ctx, ctx->stream))) return rc;
        float ms = 0.0f;
        CK(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1), "cudaEventElapsedTime");
        const double per = ms / reps;
        if (tried && nt < max_tried) tried[nt] = {tu.chunk, tu.streams, per};
        nt++;
        if (per < best_ms) { best_ms = per; win = tu; }
    }
    ctx->tuned[p.shape] = win;
    *best = {win.chunk, win.streams, best_ms};
    if (n_tried) *n_tried = std::min(nt, max_tried);
    return ASTCB200_OK;
}

int astcb200_downsample_device(const uint8_t* d_src, uint32_t width, uint32_t height, uint8_t* d_dst, void* cuda_stream) {
    if (!d_src || !d_dst || width == 0 || height == 0 || ((uintptr_t)d_src & 3) || ((uintptr_t)d_dst & 3)) return ASTCB200_BAD_ARG;
    const int dw = (int)std::max<uint32_t>(1, width / 2), dh = (int)std::max<uint32_t>(1, height / 2);
    const dim3 blk(32, 8), grid((dw + 31) / 32, (dh + 7) / 8);
    k_downsample<<<grid, blk, 0, (cudaStream_t)cuda_stream>>>(reinterpret_cast<const uchar4*>(d_src), (int)width, (int)height,
                                                              reinterpret_cast<uchar4*>(d_dst), dw, dh);
    return cudaGetLastError() == cudaSuccess ? ASTCB200_OK : ASTCB200_CUDA_ERROR;
}

}  // extern "C"
