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

constexpr int kSlotsPerBlock = 13;

// Partitionings picked by the partition search for one block and P = 2..4:
// picks[(P-2)*5 + i] = table entry (i < 4), picks[(P-2)*5 + 4] = count.
struct PartPicks { uint16_t v[15]; uint16_t pad; };

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

struct KernelArgs {
    const uint8_t* img;       // RGBA8, row-major, device memory
    int width, height, nbx, nby;
    int block_first, nblocks; // the chunk of blocks handled by this launch sequence
    const uint8_t* tables;    // device table blob
    TableLayout L;
    PartPicks* picks;         // [nblocks]
    PBRec* pbrec;             // [nblocks * 13]
    Snap* snaps;              // [nblocks * 13 * 8]
    uint8_t* out_blocks;      // [total blocks * 16], indexed by global block index
    uint32_t* symbolic;       // optional [total blocks * 108]
};

// Shared-memory sizes the launches need for one footprint.
size_t front_smem_bytes(const TableLayout& L);
size_t refine_smem_bytes(const TableLayout& L);
size_t search_smem_bytes(const TableLayout& L);

cudaError_t configure_kernels(const TableLayout& L);
cudaError_t launch_partition_search(const KernelArgs& a, cudaStream_t s);
cudaError_t launch_front(const KernelArgs& a, cudaStream_t s);
cudaError_t launch_refine(const KernelArgs& a, cudaStream_t s);
cudaError_t launch_select_pack(const KernelArgs& a, cudaStream_t s);

}  // namespace astcb200
