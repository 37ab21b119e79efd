// Encoder context shared by the single-image entry points (capi.cu) and the
// batched ones (batch.cu).  Host-side only.
#pragma once
#include <cuda_runtime.h>

#include <map>
#include <string>
#include <vector>

#include "astcb200.h"
#include "device_guard.h"
#include "kernels.h"
#include "mlp.h"
#include "tables.h"

namespace astcb200 {

// Tables of one footprint, uploaded once per context.
struct FootTables {
    int bx = 0, by = 0;
    TableLayout L{};
    uint8_t* d = nullptr;
};

// Per-chunk intermediates of one launch stream: partition picks, 13
// partitioned-block records and 104 candidate snapshots per block.
struct Scratch {
    PartPicks* picks = nullptr;
    PBRec* pbrec = nullptr;
    Snap* snaps = nullptr;
    size_t cap_picks = 0, cap_rec = 0, cap_snap = 0;
    // proposal search: logits and the routes of one chunk
    float* logits = nullptr;
    int* lists = nullptr;          // [2][blocks]: proposal-search blocks, full-search blocks
    float* full_err = nullptr;     // [blocks]: error already written for a full-search block
    PropPicks* prop = nullptr;
    uint64_t* masks = nullptr;
    uint32_t* pbl = nullptr;       // [4][blocks * kMaxProposals] partitioned-block work lists
    uint4* tail = nullptr;         // refinement-tail entries (kTailWords words each)
    size_t cap_logits = 0, cap_lists = 0, cap_prop = 0, cap_masks = 0, cap_pbl = 0, cap_ferr = 0, cap_tail = 0;
};
// Refinement-tail entries per block of a chunk (a CTA that finds the tail full finishes its
// candidates itself), and the live candidates at or below which a refinement CTA hands
// them to the tail.
constexpr size_t kTailPerBlock = 4;       // proposal search (about 2.5 spilled per 4x4 block)
constexpr size_t kTailPerBlockFull = 16;  // full search (104 candidates per block)
constexpr int kSpillLive = 32;            // full search
constexpr int kSpillLiveProposal = 64;    // proposal pass

// A footprint's proposal network on the device.
struct NetDev {
    int bx = 0, by = 0;
    mlp::Net net{};
    void* mem = nullptr;  // one allocation holding weights and biases
};

// Proposal-search settings as the caller gave them; 0 in kmax, kbm, topn, refine_iters or
// fallback_iters selects the footprint's tuned value (resolve_pruning).
struct Pruning {
    bool enable = false;
    int kmax = 0, kbm = 0, topn = 0;
    float coverage = 0.8f, threshold = 0.5f;
    float reroute_error = 8.0f;  // per-texel weighted squared error (8-bit units) above which
                                 // a proposal-search block also takes the full search; 0: off
    int front_threads = 0;  // 0: by footprint (64 up to 16 texels, else 128)
    int refine_iters = 0;
    int fallback_iters = 0;  // refinement iterations of the full-search pass over the fallback list
    float p1_floor = 0.0f;
};

// The settings for a footprint of T texels, zeros replaced by its tuned values.  Tuned on
// held-out 2048x2048 synthetic textures against the full search with FIXED semantics for
// the least time at a mean PSNR loss below 0.1 dB with no image losing more (coverage 0.8):
// blocks of up to 16 texels need the whole refinement (8 partitionings, 8 block modes, 8
// candidates, 6 iterations); larger blocks gain from the network's partitionings and need
// far less (3, 4, 3, 6).  The network's block-mode ranking is good enough that the front's
// error estimate over more modes adds nothing.
inline Pruning resolve_pruning(const Pruning& p, int T) {
    const bool small = T <= 16;
    Pruning r = p;
    if (!r.kmax) r.kmax = small ? 8 : 3;
    if (!r.kbm) r.kbm = small ? 8 : 4;
    if (!r.topn) r.topn = small ? 8 : 3;
    if (!r.refine_iters) r.refine_iters = 6;
    if (!r.fallback_iters) r.fallback_iters = 3;
    return r;
}

// A batch shape: texture sizes and footprints in call order.
using BatchShape = std::vector<uint32_t>;

// A captured batch: the graph of one batch shape and launch configuration.
struct BatchGraph {
    uint32_t chunk = 0, streams = 0;
    std::vector<const void*> bufs;  // device buffers baked into the graph
    cudaGraphExec_t exec = nullptr;
    uint32_t launches = 0;
    uint32_t routes = 0;  // route-counter entries the captured sequence writes
};

struct BatchTuning {
    uint32_t chunk = 0, streams = 0;
};

}  // namespace astcb200

struct astcb200_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    astcb200_config cfg{};
    uint32_t width = 0, height = 0, bx = 0, by = 0, nbx = 0, nby = 0, nblocks = 0;
    bool have_image = false;
    const astcb200::FootTables* cur = nullptr;      // tables of the set_image footprint
    std::vector<astcb200::FootTables*> feet;        // every footprint used so far
    uint32_t chunk = 65536;
    astcb200::Scratch scratch;                      // single-image scratch
    uint8_t* d_img = nullptr;
    size_t img_cap = 0;
    uint8_t* d_out = nullptr;
    size_t out_cap = 0;
    uint32_t* d_sym = nullptr;
    size_t sym_cap = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::vector<cudaEvent_t> stage_ev;  // kStageIntervals + 1 per chunk
    std::vector<int8_t> stage_kind;     // kStageIntervals per chunk
    int stage_chunks = 0;               // chunks recorded by the last encode
    // batches
    std::vector<cudaStream_t> branch;                // extra streams of batched launches
    std::vector<cudaEvent_t> fork_ev, join_ev;
    std::vector<astcb200::Scratch> bscratch;         // one per batch stream
    astcb200::TexSeg* d_segs = nullptr;
    size_t segs_cap = 0;
    uint8_t* d_bin = nullptr;                        // host-pointer batches: staged inputs
    size_t bin_cap = 0;
    uint8_t* d_bout = nullptr;                       // and outputs
    size_t bout_cap = 0;
    std::map<astcb200::BatchShape, astcb200::BatchGraph> graphs;
    std::map<astcb200::BatchShape, astcb200::BatchTuning> tuned;
    // learned proposal search
    std::vector<astcb200::NetDev*> nets;
    astcb200::Pruning pruning;
    int* d_counts = nullptr;     // [chunks][mlp::kRouteCounters] routed blocks of the last encode
    size_t counts_cap = 0;
    uint32_t counts_used = 0;    // chunk entries written by the last encode
    int* d_mlp_error = nullptr;  // [0] set by an inference CTA that gave up waiting, [1] its wait limit
    unsigned long long* d_work = nullptr;  // work counters of the last timed encode (kWorkCounters)
    // Pinned staging for results bound for pageable host memory: the device-to-host copies
    // stay asynchronous (so a bounded wait can time out) and a call that times out never
    // writes into the caller's buffers afterwards.
    uint8_t* h_stage = nullptr;
    size_t stage_cap = 0;
    std::string err;
};

namespace astcb200 {

int cuda_fail(astcb200_ctx* c, cudaError_t e, const char* what);
int wait_stream(astcb200_ctx* ctx, cudaStream_t s);
int get_tables(astcb200_ctx* ctx, int bx, int by, const FootTables** out);
int ensure_scratch(astcb200_ctx* ctx, Scratch& sc, size_t blocks, int slots);
// Scratch for `blocks` blocks per chunk of footprint ft (proposal buffers when it is pruned).
int ensure_chunk_scratch(astcb200_ctx* ctx, Scratch& sc, size_t blocks, const FootTables* ft);
const NetDev* net_for(const astcb200_ctx* ctx, const FootTables* ft);  // null: full search
// Room for `chunks` route counters; resets the per-call counter index and (on stream s)
// the inference kernel's give-up flag.
int begin_routes(astcb200_ctx* ctx, size_t chunks, cudaStream_t s);
// The inference kernel's flag pair: [0] set by a CTA that gave up waiting, [1] the polls
// per wait (0: the default 2^24).
int ensure_error_flag(astcb200_ctx* ctx);
// Stage timing: per chunk, an event before the first launch and after each timed interval
// (at most kStageIntervals; an interval is one launch, or the refinement and its tail), and
// per interval its stage (0 partition search or network, 1 front, 2 refine, 3 select-pack)
// | (launches - 1) << 2, -1 past the last.
constexpr int kStageIntervals = 9;
// Queues the search of one chunk (base: addressing, block_first, nblocks) on s; ev and
// kinds, when not null, receive kStageIntervals + 1 events and the launches' stages.
// full_only: the full search even when the footprint has a network (small textures).
int enqueue_chunk(astcb200_ctx* ctx, const KernelArgs& base, const FootTables* ft, Scratch& sc, cudaStream_t s,
                  cudaEvent_t* ev, int8_t* kinds, uint32_t* launches, bool full_only = false);
void free_scratch(Scratch& sc);
void release_batches(astcb200_ctx* ctx);

// Device-to-host results of one call.  Pinned destinations are copied into directly;
// pageable ones go through ctx->h_stage and reach the caller in finish() after a
// successful wait.
struct HostResults {
    struct Item { void* dst; const void* src; size_t bytes; bool pinned; size_t off; };
    std::vector<Item> items;
    void add(void* dst, const void* src, size_t bytes) { items.push_back({dst, src, bytes, false, 0}); }
    // Classifies the destinations and grows the staging; call it before queuing the call's
    // work (growing waits for earlier calls' work on the context's stream, never for this one's).
    int reserve(astcb200_ctx* ctx);
    int queue(astcb200_ctx* ctx, cudaStream_t s);  // queues the copies
    void finish(astcb200_ctx* ctx) const;          // staged bytes to the caller (after the wait)
};

template <class T>
int ensure_buf(astcb200_ctx* ctx, T*& p, size_t& cap, size_t need, const char* what) {
    if (cap >= need && p) return ASTCB200_OK;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    cudaError_t e = cudaMalloc((void**)&p, need);
    if (e != cudaSuccess) return cuda_fail(ctx, e, what);
    cap = need;
    return ASTCB200_OK;
}

}  // namespace astcb200

#define CK(call, what)                                          \
    do {                                                        \
        cudaError_t e_ = (call);                                \
        if (e_ != cudaSuccess) return cuda_fail(ctx, e_, what); \
    } while (0)
