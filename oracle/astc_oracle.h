// CPU oracle for the ASTC LDR block-compression search (TEST INFRASTRUCTURE).
//
// This is a plain C++ restatement of the reference's GPU search, written pass by
// pass after the WGSL sources of Jure-Z/ASTC_implementation and its host driver
// (code/compression_pipeline.cpp:323-535).  Only tests/, __graft_entry__.smoke()
// and bench.py's CPU-baseline leg may load it, and only as the checker.  The
// product (astc_implementation_b200/) never links it.
//
// Parity status:
//  * integer tables and physical packing are pinned bit-exactly against the
//    reference's own compiled CPU code (oracle/_ref, tests/golden/*);
//  * the constant tables embedded in the WGSL are pinned against the WGSL text;
//  * the floating-point search itself is "parity unpinned" against reference
//    outputs: the reference runs only through WebGPU/Dawn, which cannot run on
//    these machines, so no reference output exists.  The restatement fixes every
//    behaviour the WGSL leaves open (see the semantics list in astc_oracle.cpp).
#pragma once
#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

// One SymbolicBlock in the reference layout (code/astc.h:639-655): 108 u32.
#define ORC_SYMBOLIC_WORDS 108

// Selects the semantics of every later call: 0 = REF (the parity target, the default),
// 1 = FIXED (REF plus the repairs F1-F4 listed in astc_oracle.cpp: full pass005 sort,
// pass007 emits the ordered table entry, pass07 keeps every weight, pass006 sees every
// partition's average and direction).  Returns the previous setting.  Not thread-safe:
// set it between calls.
int orc_set_semantics(int fixed);

// Selects the encodings beyond the reference's (no counterpart in it) for later calls:
// bit 0 = void-extent blocks for blocks of one colour, bit 1 = single-partition dual-plane
// blocks where their exact decoded error is lower than the search's result.  Symbolic
// words of such blocks: [6] = 1 + plane-2 component, [7] = 1 for void extent (colour in
// [12..15]), plane-2 weights at [76..].  Returns the previous flags.  Not thread-safe.
int orc_set_extensions(int flags);

// Encodes an RGBA8 image (row-major, 4 bytes per texel) into physical ASTC
// blocks (16 bytes each, blocks in raster order).  `threads` <= 0 uses all
// OpenMP threads.  `symbolic` (optional) receives ORC_SYMBOLIC_WORDS u32 per block.
// Returns 0 on success, negative on bad arguments.
int orc_encode(const uint8_t* rgba, int width, int height, int bx, int by, int threads,
               uint8_t* out_blocks, uint32_t* symbolic);

// orc_encode with `refine_iters` refinement iterations instead of the reference's 6 (the
// proposal search's full-search pass over its fallback blocks runs fewer).
int orc_encode_iters(const uint8_t* rgba, int width, int height, int bx, int by, int threads, int refine_iters,
                     uint8_t* out_blocks, uint32_t* symbolic);

// Runs the search for a list of blocks given as pre-split texel data (T texels of
// 4 floats each, already scaled to 0..65536) and returns symbolic results.
int orc_encode_blocks(const float* texels, int nblocks, int bx, int by, int threads,
                      uint32_t* symbolic, uint8_t* out_blocks);

// The search restricted to given candidates, the checker of the learned proposal
// search (no counterpart in the reference).  Per block: picks[ORC_PICK_WORDS] = count n
// (<= 16), flags (bit 0: skip P = 1), then n partitionings (P - 2) << 10 | table entry;
// masks[16] = for P = 1..4, 4 words of block-mode bits (valid block-mode order).  The
// first `topn` (1..8) trials are refined `refine_iters` times.  found[i] = 0 when no
// candidate reached an error below 1e30 (that block's outputs are then zero).
// Footprints with more than 256 valid block modes are rejected (-1).
#define ORC_PICK_WORDS 18
int orc_encode_restricted(const uint8_t* rgba, int width, int height, int bx, int by, int threads,
                          const uint16_t* picks, const uint64_t* masks, int topn, int refine_iters,
                          uint8_t* out_blocks, uint32_t* symbolic, uint8_t* found);

// Packs one SymbolicBlock into a physical block (restatement of
// code/physical_compression.cpp:843).
int orc_symbolic_to_physical(int bx, int by, const uint32_t* symbolic, uint8_t* out16);

// Table dumps with the same layouts as oracle/ref_shim.cpp (for digests).
int orc_counts(int bx, int by, uint32_t* counts);
int orc_block_modes(int bx, int by, uint32_t* bm_index, uint32_t* bms);
int orc_decimation(int bx, int by, uint32_t* dmodes, uint32_t* dinfo);
int orc_maps(int bx, int by, uint32_t* t2w_idx, float* t2w_c, uint32_t* w2t_idx, float* w2t_c);
int orc_partitions(int bx, int by, uint32_t* pinfo, uint64_t* cov2, uint64_t* cov3, uint64_t* cov4,
                   uint32_t* kmeans, uint16_t* packed_index);
int orc_angular(float* sin_out, float* cos_out);
// valid_dms[0..n) and valid_bms[0..m) x 2 (packed block mode, dm lookup index)
int orc_trial_modes(int bx, int by, uint32_t* n_dm, uint32_t* valid_dms, uint32_t* n_bm, uint32_t* valid_bms);
// constant tables: quant_to_unquant[142], quant_mode_table[10*128],
// color_unquant_to_uquant[17*512], prev_next[12*65], baseline_quant_error[17],
// integer_of_trits[243], integer_of_quints[125], weight_scramble[12*32], color_scramble[17*256]
int orc_const_tables(int32_t* q2u, int32_t* qmt, int32_t* cu2u, int32_t* prev_next, float* bqe,
                     uint8_t* trits, uint8_t* quints, uint8_t* wscr, uint8_t* cscr);
// Partition search for one block and one partition count (passes 001-007):
// returns the number of partitioned blocks (<= 4) and their packed table entries.
int orc_partition_search(int bx, int by, const float* texels, int partition_count, uint32_t* entries);
// The same search's intermediate order: mismatch[1024] (pass004, 0xFFFFFFFF past the
// selected partitionings) and order[128] (pass005's first 128 table entries, in the
// current semantics).  Returns the number of selected partitionings.
int orc_partition_order(int bx, int by, const float* texels, int partition_count, uint32_t* mismatch, uint32_t* order);
// Passes 01-12 of one partitioned block (P = 1, or table entry `entry` of P = 2..4) in the
// current semantics, no refinement: ep[48] receives per partition the average, ep0 and ep1
// (pass01; 4 floats each), cands[8][71] pass12's candidates (trial block-mode index, colour
// quant level and its "mod" level, 4 endpoint formats, 64 quantised weights).  Returns the
// number of candidates.
int orc_front_candidates(int bx, int by, const float* texels, int partition_count, int entry, float* ep, uint32_t* cands);
// The same block refined `iters` times (1..6): out[8][104] receives each candidate's best
// state (pass17's snapshot): error (float bits; ERR_DEFAULT for an inert slot, the rest then
// 0), trial block-mode index, final quant level, matched flag, 4 endpoint formats, 32 packed
// endpoint values, 64 weights.  Returns the number of candidates.
int orc_refined_candidates(int bx, int by, const float* texels, int partition_count, int entry, int iters, uint32_t* out);

#ifdef __cplusplus
}
#endif
