// Records exchanged between the encoder's kernels and their launch entry points.
//
// One ASTC block is searched as 13 "partitioned blocks" (the reference's name,
// compression_pipeline.cpp:411): slot 0 is the single-partition block, slots
// 1+4*(P-2)+i hold the i-th partitioning picked for P = 2, 3, 4 partitions.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "tables.h"

namespace astcb200 {

constexpr int kSlotsPerBlock = 13;   // full search: P = 1 plus 4 partitionings for each of P = 2, 3, 4
constexpr int kMaxProposals = 16;    // proposal search: P = 1 plus up to 16 proposed partitionings
constexpr int kMaxSlots = 1 + kMaxProposals;
constexpr int kMaskWords = 4;        // block-mode masks cover up to 256 block modes

// Partitionings picked by the partition search for one block and P = 2..4:
// picks[(P-2)*5 + i] = table entry (i < 4), picks[(P-2)*5 + 4] = count.
struct PartPicks { uint16_t v[15]; uint16_t pad; };

// Partitionings proposed for one block (proposal search): v[i] = (P - 2) << 10 | table entry,
// best first; slot 1 + i of the block searches v[i]; flags bit 0: slot 0 (P = 1) is not searched.
struct PropPicks { uint16_t n, flags; uint16_t v[kMaxProposals]; };

// Initial state of one refinement candidate (pass12 output).
struct CandInit {
    uint16_t bm;        // block-mode trial lookup index
    uint8_t ql, qlm;    // colour quant level and its "mod" variant (pass11)
    uint8_t fmt[4];     // endpoint formats per partition
    uint8_t qw[64];     // quantised weights on the 0..64 scale
};

// Output of the front kernel for one partitioned block.
struct __align__(16) PBRec {
    float4 avg[4], ep0[4], ep1[4];   // ideal endpoints (pass01), copied into every candidate
    uint32_t P, entry, ncand, seed;  // partition count, table entry, valid candidates, partition seed
    CandInit c[kNumCand];
};

// Best state a candidate reached during refinement (pass17's top_candidates).
struct Snap {
    float err;
    uint16_t bm;
    uint8_t final_q, matched;
    uint8_t ffmt[4];
    uint8_t pad[4];
    uint8_t packed[32];
    uint8_t qw[64];
};

// One texture of a batch as the kernels address it.  A batch launch numbers
// the blocks of all its textures (one footprint) consecutively: texture i owns
// blocks [block_base, block_base + nbx * nby).
struct TexSeg {
    const uint8_t* img;       // RGBA8, row-major, device memory
    uint8_t* out;             // its 16-byte blocks, row-major
    int width, height, nbx, block_base;
};

struct KernelArgs {
    const uint8_t* img;       // RGBA8, row-major, device memory (single image: nsegs == 0)
    int width, height, nbx, nby;
    int block_first, nblocks; // the chunk of blocks handled by this launch sequence
    const TexSeg* segs;       // batch textures sorted by block_base (nsegs > 0), device memory
    int nsegs;
    const uint8_t* tables;    // device table blob
    TableLayout L;
    PartPicks* picks;         // [nblocks]
    PBRec* pbrec;             // [nblocks * slots]
    Snap* snaps;              // [nblocks * slots * 8]
    uint8_t* out_blocks;      // [total blocks * 16], indexed by global block index
    uint32_t* symbolic;       // optional [total blocks * 108]
    int slots;                // partitioned blocks per block: 13 (full search) or 1 + kMaxProposals
    int topn;                 // refinement candidates kept per partitioned block (<= 8)
    // Block lists (proposal search and its full-search fallback): the chunk's
    // blocks are block_list[block_first + lb] while block_first + lb < *block_count.
    const int* block_list;
    const int* block_count;
    const PropPicks* prop;    // per list position: proposed partitionings (replaces the partition search)
    const uint64_t* bm_mask;  // per list position and P = 1..4: block modes the front evaluates
    int* reroute_list;        // blocks that end without any candidate are appended here (and
    int* reroute_count;       // left unwritten) instead of being encoded; null: never
    float reroute_above;      // blocks whose best error exceeds this are encoded and also appended
    float* reroute_err;       // [list position]: error of the block already written (3e38: none)
    const float* prev_err;    // full-search pass: write a block only if its error is below this
    // Partitioned-block work list of the proposal pass: four lists (P = 1..4) of
    // position << 5 | slot, pb_stride apart, with counts pb_count[0..3].  Null: every
    // slot of every block is an item.
    const uint32_t* pb_list;
    const int* pb_count;
    int pb_stride;
    int pb_from, pb_to;       // the lists a launch takes: [pb_from, pb_to), pb_to 0 = up to the last
    // Work counters (null: not counted): [0..3] partitioned blocks searched by the front,
    // by P; [4] decimation modes and [5] block modes it evaluated; [6..9] candidates
    // refined, by P; [10..12] partition searches, P = 2..4; [13] candidates the refinement
    // handed to its tail pass.
    unsigned long long* work;
    int front_threads;        // threads per front CTA: 128 (0 selects it), 64 or 32
    int refine_iters;         // refinement iterations (0 selects the reference's 6)
    int fixed;                // 1: FIXED semantics (ASTCB200_FLAG_FIXED_SEMANTICS), 0: the reference's
    // Refinement tail (null: off): once a refinement CTA has at most spill_live candidates
    // left, it writes their state here (kTailWords uint4 each, up to tail_cap entries,
    // tail_count[0] reserved so far) and takes its next group; k_refine_tail finishes them,
    // claiming entries from tail_count[1] (zero at its launch).
    uint4* tail;
    int* tail_count;
    int tail_cap;
    int spill_live;
};
constexpr int kTailWords = 13;        // uint4 words of one refinement-tail entry
constexpr int kTailMaxTexels = 36;    // blocks of more texels are never handed to the tail
constexpr int kWorkCounters = 16;

// Launch grid caps for kernels that walk device-side lists (grid-stride loops).
constexpr int kListGridFront = 148 * 8 * 4;
constexpr int kListGridRefine = 148 * 6 * 4;
constexpr int kListGridSearch = 148 * 4 * 4;
constexpr int kListGridPack = 148 * 8;

// Global index of the chunk's lb-th block, or -1 past the end of a block list.
__host__ __device__ inline int chunk_block(const KernelArgs& a, int lb) {
    const int pos = a.block_first + lb;
    if (!a.block_list) return pos;
    return pos < *a.block_count ? a.block_list[pos] : -1;
}

#ifdef __CUDACC__
// Blocks a launch covers: the chunk, or the device-side count of its block list.
__device__ __forceinline__ int list_blocks(const KernelArgs& a) {
    return a.block_list ? min(*a.block_count, a.nblocks) : a.nblocks;
}

// Partitioned blocks of the proposal pass, and item i's list position and slot.
__device__ __forceinline__ int pb_total(const KernelArgs& a) {
    const int to = a.pb_to ? a.pb_to : 4;
    int n = 0;
    for (int p = a.pb_from; p < to; p++) n += a.pb_count[p];
    return n;
}
__device__ __forceinline__ void pb_item(const KernelArgs& a, int i, int& lb, int& slot) {
    const int last = (a.pb_to ? a.pb_to : 4) - 1;
    int p = a.pb_from;
    while (p < last && i >= a.pb_count[p]) { i -= a.pb_count[p]; p++; }
    const uint32_t v = a.pb_list[(size_t)p * a.pb_stride + i];
    lb = (int)(v >> 5);
    slot = (int)(v & 31);
}

// Where block blk's texels come from: the image, its size and the block's
// top-left texel.
struct BlockSrc {
    const uchar4* img;
    int width, height, x0, y0;
    int seg;  // batch texture index, -1 for a single image
};

__device__ __forceinline__ BlockSrc block_src(const KernelArgs& a, int blk) {
    if (a.nsegs == 0) {
        const int bxi = blk % a.nbx, byi = blk / a.nbx;
        return {reinterpret_cast<const uchar4*>(a.img), a.width, a.height, bxi * a.L.bx, byi * a.L.by, -1};
    }
    int lo = 0, hi = a.nsegs - 1;  // last texture whose first block is <= blk
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (a.segs[mid].block_base <= blk) lo = mid; else hi = mid - 1;
    }
    const TexSeg& s = a.segs[lo];
    const int local = blk - s.block_base;
    const int bxi = local % s.nbx, byi = local / s.nbx;
    return {reinterpret_cast<const uchar4*>(s.img), s.width, s.height, bxi * a.L.bx, byi * a.L.by, lo};
}

// Texel t of the block, edge-clamped, as stored.
__device__ __forceinline__ uchar4 src_rgba8(const BlockSrc& s, int bx, int t) {
    const int x = min(s.x0 + t % bx, s.width - 1);
    const int y = min(s.y0 + t / bx, s.height - 1);
    return s.img[(size_t)y * s.width + x];
}

// Texel t of the block, edge-clamped, as (v / 255) * 65536 (compression_pipeline.cpp:32-46).
__device__ __forceinline__ float4 src_texel(const BlockSrc& s, int bx, int t) {
    const int x = min(s.x0 + t % bx, s.width - 1);
    const int y = min(s.y0 + t / bx, s.height - 1);
    const uchar4 p = s.img[(size_t)y * s.width + x];
    return make_float4(((float)p.x / 255.0f) * 65536.0f, ((float)p.y / 255.0f) * 65536.0f,
                       ((float)p.z / 255.0f) * 65536.0f, ((float)p.w / 255.0f) * 65536.0f);
}

// Destination of block blk's 16 bytes.
__device__ __forceinline__ uint4* block_dst(const KernelArgs& a, int blk) {
    if (a.nsegs == 0) return reinterpret_cast<uint4*>(a.out_blocks) + blk;
    const BlockSrc s = block_src(a, blk);
    const TexSeg& t = a.segs[s.seg];
    return reinterpret_cast<uint4*>(t.out) + (blk - t.block_base);
}
#endif

// Shared-memory sizes the launches need for one footprint.
size_t front_smem_bytes(const TableLayout& L, int threads = 128, bool list = false);
size_t refine_smem_bytes(const TableLayout& L);
size_t search_smem_bytes(const TableLayout& L);

cudaError_t configure_kernels(const TableLayout& L);
cudaError_t launch_partition_search(const KernelArgs& a, cudaStream_t s);
cudaError_t launch_front(const KernelArgs& a, cudaStream_t s);
cudaError_t launch_refine(const KernelArgs& a, cudaStream_t s);
// Finishes the candidates k_refine handed to the tail (a.tail, a.tail_count).
cudaError_t launch_refine_tail(const KernelArgs& a, cudaStream_t s);
cudaError_t launch_select_pack(const KernelArgs& a, cudaStream_t s);
// Optional encodings over the chunk's blocks after the search (flags: bit 0 void extent,
// bit 1 dual plane); nothing is launched when neither is set.
cudaError_t launch_extend(const KernelArgs& a, int flags, cudaStream_t s);

}  // namespace astcb200
