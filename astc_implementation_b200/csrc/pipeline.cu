// The launch sequence of one chunk of blocks, shared by single-image and
// batched encodes, and the proposal network's host side (upload, pruning
// settings, statistics).
//
// Full search, per chunk:
//   k_partition_search -> k_front -> k_refine -> k_select_pack
// Proposal search, per chunk (footprints with a network, pruning enabled):
//   k_mlp_logits -> k_select
//   -> k_front -> k_refine -> k_select_pack      over the proposal-search list
//      (1 + kmax partitioned blocks per block, masked block modes, topn candidates)
//   -> k_partition_search -> k_front -> k_refine -> k_select_pack   over the
//      full-search list (low-confidence blocks, and proposal-search blocks that
//      ended without any candidate, which the first select-pack appends)
// The two passes use separate record and snapshot regions.  Kernels past a
// list's device-side count return at once.
#include <cstring>
#include <vector>

#include "ctx.h"

using namespace astcb200;

namespace astcb200 {

// A chunk's route counters: [0, 1] routes, [2, 5] partitioned blocks by P, [6] refinement-tail
// entries reserved, [7] entries claimed by k_refine_tail.
static_assert(mlp::kRouteCounters >= 8, "the refinement tail uses route counters 6 and 7");

const NetDev* net_for(const astcb200_ctx* ctx, const FootTables* ft) {
    if (!ctx->pruning.enable) return nullptr;
    for (const NetDev* n : ctx->nets)
        if (n->bx == ft->bx && n->by == ft->by) return n;
    return nullptr;
}

int ensure_chunk_scratch(astcb200_ctx* ctx, Scratch& sc, size_t blocks, const FootTables* ft) {
    const NetDev* nd = net_for(ctx, ft);
    if (!nd) {
        const int rc = ensure_scratch(ctx, sc, blocks, kSlotsPerBlock);
        if (rc || ft->L.T > kTailMaxTexels) return rc;
        return ensure_buf(ctx, sc.tail, sc.cap_tail, blocks * kTailPerBlockFull * kTailWords * sizeof(uint4), "cudaMalloc refinement tail");
    }
    int rc;
    if ((rc = ensure_scratch(ctx, sc, blocks, kSlotsPerBlock + kMaxSlots))) return rc;
    if ((rc = ensure_buf(ctx, sc.logits, sc.cap_logits, blocks * nd->net.s.nout * sizeof(float), "cudaMalloc logits"))) return rc;
    if ((rc = ensure_buf(ctx, sc.lists, sc.cap_lists, blocks * 2 * sizeof(int), "cudaMalloc block lists"))) return rc;
    if ((rc = ensure_buf(ctx, sc.prop, sc.cap_prop, blocks * sizeof(PropPicks), "cudaMalloc proposals"))) return rc;
    if ((rc = ensure_buf(ctx, sc.masks, sc.cap_masks, blocks * 4 * kMaskWords * sizeof(uint64_t), "cudaMalloc block-mode masks"))) return rc;
    if ((rc = ensure_buf(ctx, sc.full_err, sc.cap_ferr, blocks * sizeof(float), "cudaMalloc full-search errors"))) return rc;
    if (ft->L.T <= kTailMaxTexels &&
        (rc = ensure_buf(ctx, sc.tail, sc.cap_tail, blocks * kTailPerBlock * kTailWords * sizeof(uint4), "cudaMalloc refinement tail")))
        return rc;
    return ensure_buf(ctx, sc.pbl, sc.cap_pbl, blocks * 4 * kMaxProposals * sizeof(uint32_t), "cudaMalloc work lists");
}

int ensure_error_flag(astcb200_ctx* ctx) {
    if (ctx->d_mlp_error) return ASTCB200_OK;
    size_t cap = 0;
    int rc = ensure_buf(ctx, ctx->d_mlp_error, cap, 2 * sizeof(int), "cudaMalloc error flag");
    if (rc) return rc;
    CK(cudaMemset(ctx->d_mlp_error, 0, 2 * sizeof(int)), "cudaMemset");
    return ASTCB200_OK;
}

int begin_routes(astcb200_ctx* ctx, size_t chunks, cudaStream_t s) {
    ctx->counts_used = 0;
    int rc = ensure_buf(ctx, ctx->d_counts, ctx->counts_cap, std::max<size_t>(chunks, 1) * mlp::kRouteCounters * sizeof(int), "cudaMalloc route counters");
    if (rc) return rc;
    if ((rc = ensure_error_flag(ctx))) return rc;
    CK(cudaMemsetAsync(ctx->d_mlp_error, 0, sizeof(int), s), "reset error flag");  // this call's give-ups only
    return ASTCB200_OK;
}

int enqueue_chunk(astcb200_ctx* ctx, const KernelArgs& base, const FootTables* ft, Scratch& sc, cudaStream_t s,
                  cudaEvent_t* ev, int8_t* kinds, uint32_t* launches, bool full_only) {
    KernelArgs a = base;
    a.fixed = (ctx->cfg.flags & ASTCB200_FLAG_FIXED_SEMANTICS) ? 1 : 0;
    // optional encodings after the search (not timed by the stage events)
    const int ext = ((ctx->cfg.flags & ASTCB200_FLAG_VOID_EXTENT) ? 1 : 0) | ((ctx->cfg.flags & ASTCB200_FLAG_DUAL_PLANE) ? 2 : 0);
    a.tables = ft->d;
    a.L = ft->L;
    a.picks = sc.picks;
    a.pbrec = sc.pbrec;
    a.snaps = sc.snaps;
    int ni = 0;  // launches queued so far; ev[ni] precedes launch ni
    if (ev) {
        for (int i = 0; i < kStageIntervals; i++) kinds[i] = -1;
        CK(cudaEventRecord(ev[0], s), "stage event");
    }
    auto done = [&](cudaError_t e, const char* what, int kind, int nl = 1) -> int {
        if (e != cudaSuccess) return cuda_fail(ctx, e, what);
        if (ev) {
            kinds[ni] = (int8_t)(kind | (nl - 1) << 2);  // stage, then the interval's extra launches
            CK(cudaEventRecord(ev[ni + 1], s), "stage event");
        }
        ni++;
        return ASTCB200_OK;
    };
    int rc;
    const NetDev* nd = full_only ? nullptr : net_for(ctx, ft);
    if (!nd) {
        a.slots = kSlotsPerBlock;
        a.topn = kNumCand;
        int nl = 1;  // launches of the refinement interval
        if (sc.tail && ft->L.T <= kTailMaxTexels &&
            (ctx->counts_used + 1) * mlp::kRouteCounters <= ctx->counts_cap / sizeof(int)) {
            // the refinement hands its last candidates to the tail, as in the proposal pass
            int* counts = ctx->d_counts + mlp::kRouteCounters * ctx->counts_used++;
            CK(cudaMemsetAsync(counts, 0, mlp::kRouteCounters * sizeof(int), s), "reset tail counter");
            a.tail = sc.tail;
            a.tail_cap = (int)std::min<size_t>(sc.cap_tail / (kTailWords * sizeof(uint4)), (size_t)1 << 30);
            a.spill_live = kSpillLive;
            a.tail_count = counts + 6;  // and its claim counter, counts[7]
            nl = 2;
        }
        if ((rc = done(launch_partition_search(a, s), "k_partition_search", 0))) return rc;
        if ((rc = done(launch_front(a, s), "k_front", 1))) return rc;
        {
            cudaError_t e = launch_refine(a, s);
            if (e == cudaSuccess && a.tail) e = launch_refine_tail(a, s);
            if ((rc = done(e, "k_refine", 2, nl))) return rc;
        }
        if ((rc = done(launch_select_pack(a, s), "k_select_pack", 3))) return rc;
        if (ext) { CK(launch_extend(a, ext, s), "k_extend"); ni++; }
        if (launches) *launches += ni + (nl - 1);
        return ASTCB200_OK;
    }
    const Pruning pr = resolve_pruning(ctx->pruning, ft->L.T);
    const size_t n = (size_t)a.nblocks;
    if ((ctx->counts_used + 1) * mlp::kRouteCounters > ctx->counts_cap / sizeof(int)) {
        ctx->err = "route counters exhausted";
        return ASTCB200_BAD_ARG;
    }
    int* counts = ctx->d_counts + mlp::kRouteCounters * ctx->counts_used++;
    mlp::Select sel;
    sel.kmax = pr.kmax; sel.coverage = pr.coverage; sel.threshold = pr.threshold; sel.kbm = pr.kbm;
    sel.p1_floor = pr.p1_floor;
    mlp::Routes r;
    r.counts = counts;
    r.pruned = sc.lists;
    r.full = sc.lists + n;
    r.full_err = sc.full_err;
    r.prop = sc.prop;
    r.masks = sc.masks;
    r.confidence = nullptr;
    r.pb_list = sc.pbl;
    r.pb_stride = (int)(n * kMaxProposals);

    KernelArgs ap = a;  // proposal-search pass
    ap.block_first = 0;
    ap.block_list = r.pruned; ap.block_count = counts;
    ap.prop = r.prop; ap.bm_mask = r.masks;
    ap.slots = 1 + pr.kmax; ap.topn = pr.topn;
    // small blocks: two warps per partitioned block keep twice as many of them resident
    ap.front_threads = pr.front_threads ? pr.front_threads : (ft->L.T <= 16 ? 64 : 128);
    ap.refine_iters = pr.refine_iters;
    ap.reroute_list = r.full; ap.reroute_count = counts + 1;  // blocks left without a candidate
    ap.pb_list = r.pb_list; ap.pb_count = counts + 2; ap.pb_stride = r.pb_stride;
    ap.reroute_err = r.full_err;
    {   // the threshold in the search's error units: 8-bit per-texel error x texels x (65536/255)^2
        const float s8 = 65536.0f / 255.0f;
        ap.reroute_above = pr.reroute_error > 0.0f ? pr.reroute_error * (float)ft->L.T * s8 * s8 : 0.0f;
    }
    KernelArgs af = a;  // full-search pass over the low-confidence and rerouted blocks
    af.block_first = 0;
    af.block_list = r.full; af.block_count = counts + 1;
    af.prev_err = r.full_err;
    af.slots = kSlotsPerBlock; af.topn = kNumCand;
    af.refine_iters = pr.fallback_iters;  // the candidates' serial refinement chain sets this pass's duration
    af.pbrec = sc.pbrec + n * kMaxSlots;
    af.snaps = sc.snaps + n * kMaxSlots * kNumCand;
    if (sc.tail && ft->L.T <= kTailMaxTexels) {
        // The proposal pass hands its last candidates to the tail.  The fallback pass does not:
        // it holds few blocks, so its duration is one CTA's chain, which a second, serial
        // kernel would only lengthen.
        ap.tail = sc.tail;
        ap.tail_cap = (int)std::min<size_t>(sc.cap_tail / (kTailWords * sizeof(uint4)), (size_t)1 << 30);
        ap.spill_live = kSpillLiveProposal;
        ap.tail_count = counts + 6;  // two free route counters: reservations, claims
    }
    int tails = 0;  // tail launches (timed with their pass's refinement)
    auto refine = [&](const KernelArgs& k, const char* what) -> int {
        cudaError_t e = launch_refine(k, s);
        const int nl = k.tail ? 2 : 1;
        if (e == cudaSuccess && k.tail) { e = launch_refine_tail(k, s); tails++; }
        return done(e, what, 2, nl);
    };

    CK(cudaMemsetAsync(counts, 0, mlp::kRouteCounters * sizeof(int), s), "reset route counters");
    if ((rc = done(mlp::launch_mlp_logits(a, nd->net, sc.logits, ctx->d_mlp_error, s), "k_mlp_logits", 0))) return rc;
    if ((rc = done(mlp::launch_select(a, nd->net, sc.logits, sel, r, s), "k_select", 0))) return rc;
    if ((rc = done(launch_front(ap, s), "k_front", 1, 2))) return rc;  // the P = 1 list, then the others
    if ((rc = refine(ap, "k_refine"))) return rc;
    if ((rc = done(launch_select_pack(ap, s), "k_select_pack", 3))) return rc;
    if ((rc = done(launch_partition_search(af, s), "k_partition_search", 0))) return rc;
    if ((rc = done(launch_front(af, s), "k_front", 1))) return rc;
    if ((rc = refine(af, "k_refine"))) return rc;
    if ((rc = done(launch_select_pack(af, s), "k_select_pack", 3))) return rc;
    if (ext) { CK(launch_extend(a, ext, s), "k_extend"); ni++; }  // every block of the chunk, after both passes
    if (launches) *launches += ni + tails;
    return ASTCB200_OK;
}

}  // namespace astcb200

namespace {

uint16_t to_bf16(float f) {  // round to nearest even (finite inputs)
    uint32_t u;
    std::memcpy(&u, &f, 4);
    u += 0x7FFFu + ((u >> 16) & 1u);
    return (uint16_t)(u >> 16);
}

size_t a256(size_t v) { return (v + 255) & ~size_t(255); }

}  // namespace

extern "C" {

int astcb200_proposal_layout(uint8_t bx, uint8_t by, uint32_t* inputs, uint32_t* inputs_padded, uint32_t* outputs,
                             uint32_t* block_modes, uint32_t* head_base, uint32_t* head_stride, uint32_t* sel3) {
    if (!valid_footprint(bx, by)) return ASTCB200_INVALID_FOOTPRINT;
    TableLayout L;
    std::vector<uint8_t> blob;
    if (!build_tables(bx, by, L, blob)) return ASTCB200_INVALID_FOOTPRINT;
    const mlp::Shape s = mlp::shape_for(L.T, L.nbm, L.count_selected + 1);
    if (inputs) *inputs = s.k0;
    if (inputs_padded) *inputs_padded = s.k0p;
    if (outputs) *outputs = s.nout;
    if (block_modes) *block_modes = s.nbm;
    if (head_base) *head_base = s.head_base;
    if (head_stride) *head_stride = s.nbm_pad;
    if (sel3) for (int i = 0; i < 3; i++) sel3[i] = L.count_selected[i + 1];
    return ASTCB200_OK;
}

int astcb200_set_proposal_net(astcb200_ctx* ctx, const astcb200_proposal_net* w) {
    if (!ctx || !w || w->struct_size < sizeof(astcb200_proposal_net)) return ASTCB200_BAD_ARG;
    if (!w->w1 || !w->b1 || !w->w2 || !w->b2 || !w->w3 || !w->b3) return ASTCB200_BAD_ARG;
    ASTCB200_DEVICE_SCOPE(ctx);
    const FootTables* ft = nullptr;
    int rc = get_tables(ctx, w->block_x, w->block_y, &ft);
    if (rc) return rc;
    const mlp::Shape s = mlp::shape_for(ft->L.T, ft->L.nbm, ft->L.count_selected + 1);
    if (w->inputs != (uint32_t)s.k0 || w->hidden != (uint32_t)mlp::kHidden || w->outputs != (uint32_t)s.nout) {
        ctx->err = "network shape does not match astcb200_proposal_layout";
        return ASTCB200_BAD_ARG;
    }
    if (ft->L.nbm > 64 * kMaskWords || ft->L.ndm > 128) {
        ctx->err = "footprint has too many block modes for the proposal search";
        return ASTCB200_BAD_ARG;
    }
    const size_t H = mlp::kHidden, K = s.k0, KP = s.k0p, NO = s.nout;
    const size_t o_w1 = 0, o_w2 = a256(o_w1 + H * KP * 2), o_w3 = a256(o_w2 + H * H * 2), o_b1 = a256(o_w3 + NO * H * 2),
                 o_b2 = a256(o_b1 + H * 4), o_b3 = a256(o_b2 + H * 4), total = a256(o_b3 + NO * 4);
    std::vector<uint8_t> host(total, 0);
    uint16_t* w1 = reinterpret_cast<uint16_t*>(host.data() + o_w1);
    uint16_t* w2 = reinterpret_cast<uint16_t*>(host.data() + o_w2);
    uint16_t* w3 = reinterpret_cast<uint16_t*>(host.data() + o_w3);
    for (size_t n = 0; n < H; n++)
        for (size_t k = 0; k < KP; k++) w1[mlp::core_index(n, k, H)] = k < K ? to_bf16(w->w1[n * K + k]) : 0;
    for (size_t n = 0; n < H; n++)
        for (size_t k = 0; k < H; k++) w2[mlp::core_index(n, k, H)] = to_bf16(w->w2[n * H + k]);
    for (size_t n = 0; n < NO; n++) {
        const size_t c = n / mlp::kChunkN, nn = n % mlp::kChunkN;
        for (size_t k = 0; k < H; k++) w3[c * mlp::kChunkN * H + mlp::core_index(nn, k, mlp::kChunkN)] = to_bf16(w->w3[n * H + k]);
    }
    std::memcpy(host.data() + o_b1, w->b1, H * 4);
    std::memcpy(host.data() + o_b2, w->b2, H * 4);
    std::memcpy(host.data() + o_b3, w->b3, NO * 4);

    NetDev* nd = nullptr;
    for (NetDev* x : ctx->nets)
        if (x->bx == w->block_x && x->by == w->block_y) nd = x;
    if (!nd) {
        nd = new NetDev();
        nd->bx = w->block_x; nd->by = w->block_y;
        ctx->nets.push_back(nd);
    }
    CK(cudaStreamSynchronize(ctx->stream), "cudaStreamSynchronize");
    if (nd->mem) { cudaFree(nd->mem); nd->mem = nullptr; }
    CK(cudaMalloc(&nd->mem, total), "cudaMalloc network");
    CK(cudaMemcpy(nd->mem, host.data(), total, cudaMemcpyHostToDevice), "upload network");
    CK(mlp::configure_mlp(), "configure k_mlp_logits");
    uint8_t* d = static_cast<uint8_t*>(nd->mem);
    nd->net.w1 = reinterpret_cast<const uint16_t*>(d + o_w1);
    nd->net.w2 = reinterpret_cast<const uint16_t*>(d + o_w2);
    nd->net.w3 = reinterpret_cast<const uint16_t*>(d + o_w3);
    nd->net.b1 = reinterpret_cast<const float*>(d + o_b1);
    nd->net.b2 = reinterpret_cast<const float*>(d + o_b2);
    nd->net.b3 = reinterpret_cast<const float*>(d + o_b3);
    nd->net.s = s;
    release_batches(ctx);  // captured graphs hold the previous network
    return ASTCB200_OK;
}

int astcb200_set_pruning(astcb200_ctx* ctx, const astcb200_pruning* cfg) {
    if (!ctx || !cfg || cfg->struct_size < sizeof(astcb200_pruning)) return ASTCB200_BAD_ARG;
    if (cfg->enable && (cfg->max_partitionings > (uint32_t)kMaxProposals || cfg->block_modes > 64 ||
                        cfg->refine_candidates > (uint32_t)kNumCand || !(cfg->coverage >= 0.0f) ||
                        !(cfg->threshold >= 0.0f) || !(cfg->reroute_error >= 0.0f) ||
                        (cfg->front_threads && cfg->front_threads != 32 && cfg->front_threads != 64 && cfg->front_threads != 128) ||
                        cfg->refine_iterations > 6 || !(cfg->single_partition_floor >= 0.0f) || cfg->fallback_iterations > 6))
        return ASTCB200_BAD_ARG;
    Pruning& p = ctx->pruning;
    p.enable = cfg->enable != 0;
    p.kmax = (int)cfg->max_partitionings;
    p.kbm = (int)cfg->block_modes;
    p.topn = (int)cfg->refine_candidates;
    p.coverage = cfg->coverage;
    p.threshold = cfg->threshold;
    p.reroute_error = cfg->reroute_error;
    p.front_threads = (int)cfg->front_threads;
    p.refine_iters = (int)cfg->refine_iterations;
    p.p1_floor = cfg->single_partition_floor;
    p.fallback_iters = (int)cfg->fallback_iterations;
    release_batches(ctx);  // captured graphs hold the previous settings
    return ASTCB200_OK;
}

int astcb200_set_inference_wait_limit(astcb200_ctx* ctx, uint32_t polls) {
    if (!ctx || polls > 0x7FFFFFFFu) return ASTCB200_BAD_ARG;
    ASTCB200_DEVICE_SCOPE(ctx);
    int rc = ensure_error_flag(ctx);
    if (rc) return rc;
    const int v = (int)polls;
    CK(cudaStreamSynchronize(ctx->stream), "cudaStreamSynchronize");
    CK(cudaMemcpy(ctx->d_mlp_error + 1, &v, sizeof(int), cudaMemcpyHostToDevice), "set wait limit");
    return ASTCB200_OK;
}

int astcb200_pruning_stats(astcb200_ctx* ctx, uint64_t* proposal_blocks, uint64_t* full_blocks) {
    if (!ctx || !proposal_blocks || !full_blocks) return ASTCB200_BAD_ARG;
    *proposal_blocks = *full_blocks = 0;
    if (!ctx->counts_used) return ASTCB200_OK;
    ASTCB200_DEVICE_SCOPE(ctx);
    CK(cudaDeviceSynchronize(), "cudaDeviceSynchronize");
    std::vector<int> c((size_t)mlp::kRouteCounters * ctx->counts_used);
    CK(cudaMemcpy(c.data(), ctx->d_counts, c.size() * sizeof(int), cudaMemcpyDeviceToHost), "read route counters");
    for (uint32_t i = 0; i < ctx->counts_used; i++) {
        *proposal_blocks += (uint64_t)c[mlp::kRouteCounters * i];
        *full_blocks += (uint64_t)c[mlp::kRouteCounters * i + 1];
    }
    int err = 0;
    if (ctx->d_mlp_error) CK(cudaMemcpy(&err, ctx->d_mlp_error, sizeof(int), cudaMemcpyDeviceToHost), "read error flag");
    if (err) { ctx->err = "a network inference CTA gave up waiting for its copies or MMAs"; return ASTCB200_TIMEOUT; }
    return ASTCB200_OK;
}

int astcb200_proposal_logits(astcb200_ctx* ctx, const uint8_t* rgba8, float* logits, size_t len) {
    if (!ctx || !rgba8 || !logits) return ASTCB200_BAD_ARG;
    if (!ctx->have_image) return ASTCB200_NO_IMAGE;
    const NetDev* nd = nullptr;
    for (const NetDev* x : ctx->nets)
        if (x->bx == (int)ctx->bx && x->by == (int)ctx->by) nd = x;
    if (!nd) { ctx->err = "no network for this footprint"; return ASTCB200_BAD_ARG; }
    const size_t nout = nd->net.s.nout;
    if (len < (size_t)ctx->nblocks * nout) return ASTCB200_BAD_ARG;
    ASTCB200_DEVICE_SCOPE(ctx);
    const size_t in_bytes = (size_t)ctx->width * ctx->height * 4;
    int rc;
    if ((rc = ensure_buf(ctx, ctx->d_img, ctx->img_cap, in_bytes, "cudaMalloc image"))) return rc;
    const size_t chunk = std::min<size_t>(ctx->chunk, ctx->nblocks);
    if ((rc = ensure_buf(ctx, ctx->scratch.logits, ctx->scratch.cap_logits, chunk * nout * 4, "cudaMalloc logits"))) return rc;
    if ((rc = begin_routes(ctx, 1, ctx->stream))) return rc;
    CK(cudaMemcpyAsync(ctx->d_img, rgba8, in_bytes, cudaMemcpyHostToDevice, ctx->stream), "H2D image");
    KernelArgs a;
    std::memset(&a, 0, sizeof(a));
    a.img = ctx->d_img;
    a.width = (int)ctx->width; a.height = (int)ctx->height; a.nbx = (int)ctx->nbx; a.nby = (int)ctx->nby;
    a.tables = ctx->cur->d;
    a.L = ctx->cur->L;
    for (uint32_t first = 0; first < ctx->nblocks; first += (uint32_t)chunk) {
        a.block_first = (int)first;
        a.nblocks = (int)std::min<size_t>(chunk, ctx->nblocks - first);
        CK(mlp::launch_mlp_logits(a, nd->net, ctx->scratch.logits, ctx->d_mlp_error, ctx->stream), "k_mlp_logits");
        CK(cudaMemcpyAsync(logits + (size_t)first * nout, ctx->scratch.logits, (size_t)a.nblocks * nout * 4, cudaMemcpyDeviceToHost,
                           ctx->stream), "D2H logits");
    }
    if ((rc = wait_stream(ctx, ctx->stream))) return rc;
    int err = 0;
    CK(cudaMemcpy(&err, ctx->d_mlp_error, sizeof(int), cudaMemcpyDeviceToHost), "read error flag");
    if (err) { ctx->err = "a network inference CTA gave up waiting for its copies or MMAs"; return ASTCB200_TIMEOUT; }
    return ASTCB200_OK;
}

int astcb200_proposal_selection(astcb200_ctx* ctx, const uint8_t* rgba8, uint8_t* route, uint16_t* picks,
                                uint64_t* masks, size_t nblocks) {
    if (!ctx || !rgba8 || !route || !picks || !masks) return ASTCB200_BAD_ARG;
    if (!ctx->have_image) return ASTCB200_NO_IMAGE;
    if (nblocks < ctx->nblocks) return ASTCB200_BAD_ARG;
    const NetDev* nd = nullptr;
    for (const NetDev* x : ctx->nets)
        if (x->bx == (int)ctx->bx && x->by == (int)ctx->by) nd = x;
    if (!nd) { ctx->err = "no network for this footprint"; return ASTCB200_BAD_ARG; }
    ASTCB200_DEVICE_SCOPE(ctx);
    const size_t in_bytes = (size_t)ctx->width * ctx->height * 4;
    const size_t chunk = std::min<size_t>(ctx->chunk, ctx->nblocks);
    const size_t nchunks = (ctx->nblocks + chunk - 1) / chunk;
    Scratch& sc = ctx->scratch;
    int rc;
    if ((rc = ensure_buf(ctx, ctx->d_img, ctx->img_cap, in_bytes, "cudaMalloc image"))) return rc;
    if ((rc = ensure_buf(ctx, sc.logits, sc.cap_logits, chunk * nd->net.s.nout * sizeof(float), "cudaMalloc logits"))) return rc;
    if ((rc = ensure_buf(ctx, sc.lists, sc.cap_lists, chunk * 2 * sizeof(int), "cudaMalloc block lists"))) return rc;
    if ((rc = ensure_buf(ctx, sc.prop, sc.cap_prop, chunk * sizeof(PropPicks), "cudaMalloc proposals"))) return rc;
    if ((rc = ensure_buf(ctx, sc.masks, sc.cap_masks, chunk * 4 * kMaskWords * sizeof(uint64_t), "cudaMalloc block-mode masks"))) return rc;
    if ((rc = ensure_buf(ctx, sc.full_err, sc.cap_ferr, chunk * sizeof(float), "cudaMalloc full-search errors"))) return rc;
    if ((rc = ensure_buf(ctx, sc.pbl, sc.cap_pbl, chunk * 4 * kMaxProposals * sizeof(uint32_t), "cudaMalloc work lists"))) return rc;
    if ((rc = begin_routes(ctx, nchunks, ctx->stream))) return rc;
    CK(cudaMemcpyAsync(ctx->d_img, rgba8, in_bytes, cudaMemcpyHostToDevice, ctx->stream), "H2D image");
    KernelArgs a;
    std::memset(&a, 0, sizeof(a));
    a.img = ctx->d_img;
    a.width = (int)ctx->width; a.height = (int)ctx->height; a.nbx = (int)ctx->nbx; a.nby = (int)ctx->nby;
    a.tables = ctx->cur->d;
    a.L = ctx->cur->L;
    const Pruning pr = resolve_pruning(ctx->pruning, ctx->cur->L.T);
    mlp::Select sel;
    sel.kmax = pr.kmax; sel.coverage = pr.coverage; sel.threshold = pr.threshold; sel.kbm = pr.kbm;
    sel.p1_floor = pr.p1_floor;
    std::memset(route, 1, ctx->nblocks);
    std::memset(picks, 0, ctx->nblocks * 18 * sizeof(uint16_t));
    std::memset(masks, 0, ctx->nblocks * 4 * kMaskWords * sizeof(uint64_t));
    if ((uint64_t)ctx->width * ctx->height < (uint64_t)mlp::kMinProposalTexels) return ASTCB200_OK;  // full search
    std::vector<int> lst(chunk);
    std::vector<PropPicks> pp(chunk);
    std::vector<uint64_t> mk(chunk * 4 * kMaskWords);
    int counts[mlp::kRouteCounters];
    for (uint32_t first = 0; first < ctx->nblocks; first += (uint32_t)chunk) {
        a.block_first = (int)first;
        a.nblocks = (int)std::min<size_t>(chunk, ctx->nblocks - first);
        mlp::Routes r;
        r.counts = ctx->d_counts + mlp::kRouteCounters * ctx->counts_used++;
        r.pruned = sc.lists; r.full = sc.lists + chunk; r.full_err = sc.full_err;
        r.prop = sc.prop; r.masks = sc.masks; r.confidence = nullptr;
        r.pb_list = sc.pbl; r.pb_stride = (int)(chunk * kMaxProposals);
        CK(cudaMemsetAsync(r.counts, 0, mlp::kRouteCounters * sizeof(int), ctx->stream), "reset route counters");
        CK(mlp::launch_mlp_logits(a, nd->net, sc.logits, ctx->d_mlp_error, ctx->stream), "k_mlp_logits");
        CK(mlp::launch_select(a, nd->net, sc.logits, sel, r, ctx->stream), "k_select");
        CK(cudaMemcpyAsync(counts, r.counts, sizeof(counts), cudaMemcpyDeviceToHost, ctx->stream), "D2H route counters");
        CK(cudaMemcpyAsync(lst.data(), sc.lists, (size_t)a.nblocks * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream), "D2H list");
        CK(cudaMemcpyAsync(pp.data(), sc.prop, (size_t)a.nblocks * sizeof(PropPicks), cudaMemcpyDeviceToHost, ctx->stream), "D2H picks");
        CK(cudaMemcpyAsync(mk.data(), sc.masks, (size_t)a.nblocks * 4 * kMaskWords * sizeof(uint64_t), cudaMemcpyDeviceToHost,
                           ctx->stream), "D2H masks");
        if ((rc = wait_stream(ctx, ctx->stream))) return rc;
        for (int pos = 0; pos < counts[0] && pos < a.nblocks; pos++) {
            const int blk = lst[pos];
            if (blk < 0 || (uint32_t)blk >= ctx->nblocks) { ctx->err = "selection list out of range"; return ASTCB200_CUDA_ERROR; }
            route[blk] = 0;
            uint16_t* o = picks + (size_t)blk * 18;
            o[0] = pp[pos].n; o[1] = pp[pos].flags;
            for (int j = 0; j < 16; j++) o[2 + j] = pp[pos].v[j];
            std::memcpy(masks + (size_t)blk * 4 * kMaskWords, mk.data() + (size_t)pos * 4 * kMaskWords, 4 * kMaskWords * sizeof(uint64_t));
        }
    }
    int err = 0;
    CK(cudaMemcpy(&err, ctx->d_mlp_error, sizeof(int), cudaMemcpyDeviceToHost), "read error flag");
    if (err) { ctx->err = "a network inference CTA gave up waiting for its copies or MMAs"; return ASTCB200_TIMEOUT; }
    return ASTCB200_OK;
}

}  // extern "C"
