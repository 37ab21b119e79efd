/*
 * astcb200 -- ASTC LDR block-compression search on one NVIDIA B200 (sm_100a).
 *
 * A drop-in for the GPU stage of Jure-Z/ASTC_implementation: the reference's
 * ASTCEncoder facade (code/astc.h:724-733) driven by code/compression_pipeline.cpp
 * and main.cpp, plus its .astc writer (code/astc_store.h:8-16).  Plain C types
 * only; every call returns an astcb200_status code and no exception crosses
 * this boundary.  One context per host thread; each context owns one CUDA
 * stream and its device buffers.
 */
#ifndef ASTCB200_H
#define ASTCB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum astcb200_status {
    ASTCB200_OK = 0,
    ASTCB200_INVALID_FOOTPRINT = 1, /* not one of the 14 2D sizes of main.cpp:127-128 */
    ASTCB200_BAD_ARG = 2,           /* null pointer, zero size, buffer too small */
    ASTCB200_OOM = 3,               /* device or host allocation failed */
    ASTCB200_CUDA_ERROR = 4,        /* a CUDA call failed; see astcb200_last_error */
    ASTCB200_TIMEOUT = 5,           /* the host wait exceeded astcb200_config.timeout_ms */
    ASTCB200_NO_IMAGE = 6,          /* astcb200_set_image has not been called */
    ASTCB200_IO_ERROR = 7,          /* astcb200_store_image could not write the file */
    ASTCB200_TOO_LARGE = 8          /* the request exceeds astcb200_encode_noalloc's fixed scratch */
} astcb200_status;

typedef struct astcb200_ctx astcb200_ctx;

typedef struct astcb200_config {
    uint32_t struct_size;  /* sizeof(astcb200_config); 0 selects all defaults */
    uint32_t chunk_blocks; /* blocks searched per launch sequence; 0 = 65536 */
    uint32_t timeout_ms;   /* bound on each host wait for the device; 0 = no bound.  A call
                              that returns ASTCB200_TIMEOUT leaves its work queued on the
                              context's stream, where it completes and later calls queue
                              behind it.  Its results never reach pageable host buffers (they
                              go through the context's pinned staging); pinned host buffers
                              passed to it, inputs and outputs, are still read or written by
                              that work, so keep them valid until a later call on the context
                              has returned or the context is destroyed. */
    uint32_t flags;        /* ASTCB200_FLAG_* */
} astcb200_config;

/* Record CUDA events around every kernel launch (on the launching stream) so that
 * astcb200_stage_times reports per-kernel device time. */
#define ASTCB200_FLAG_STAGE_TIMING 1u
/* Batched encodes launch their kernels directly instead of replaying a captured CUDA graph. */
#define ASTCB200_FLAG_NO_GRAPH 2u
/* FIXED semantics: the search with four deterministic bugs of the reference's shaders
 * repaired (the default reproduces them, bit for bit):
 *   - pass005 sorts all 1024 candidates (shaders/pass005_partition_ordering.wgsl:66-94
 *     runs a bitonic network whose comparisons stop at index 256, a partial sort);
 *   - pass007 emits the table entry each candidate was evaluated for, not its rank
 *     (pass007_prepare_partitioned_blocks.wgsl:93,107,156-157);
 *   - pass07 keeps all of a block mode's quantised weights, not floor(W/4)*4 of them
 *     (pass07_weights_and_error_for_bm.wgsl:322);
 *   - pass006's error estimate sees every partition's average and direction (its
 *     per-invocation arrays, pass006_evaluate_partition_candidates.wgsl:124-135,186-217,
 *     leave all but one texel per partition with zeros).
 * Partitionings then come from the k-means mismatch order and the error estimate as
 * designed; decoded quality rises by several dB on most images. */
#define ASTCB200_FLAG_FIXED_SEMANTICS 4u
/* Encodings the reference never emits (no counterpart in it; both off by default), applied
 * to every block after the search:
 *   VOID_EXTENT: a block whose texels are all one colour is written as an LDR void-extent
 *     block (the colour as 16-bit UNORM, no extent); it decodes to the same texels.
 *   DUAL_PLANE: single-partition dual-plane encodings are tried (each colour channel as the
 *     second plane, every dual-plane block mode whose weight grid the search uses, RGB or
 *     RGBA direct endpoints at the finest colour quantisation that fits) and the best one
 *     replaces the search's block when its decoded error is lower.  Errors are those of the
 *     decoded 8-bit texels, weighted R 0.675, G 1.3275, B 0.2475, A 1.
 * astcb200_encode_symbolic describes such blocks in the reference's record with two of its
 * padding words: [6] = 1 + the second plane's channel, [7] = 1 for void extent (colour in
 * packed_color_values[0..3]); the second plane's weights are quantized_weights[32..]. */
#define ASTCB200_FLAG_VOID_EXTENT 8u
#define ASTCB200_FLAG_DUAL_PLANE 16u

typedef struct astcb200_stats {
    double ms_wall;       /* host time of the call */
    double ms_device;     /* device time of the search kernels (CUDA events) */
    uint64_t blocks;      /* blocks encoded */
    uint64_t h2d_bytes;   /* host-to-device bytes copied by the call */
    uint64_t d2h_bytes;   /* device-to-host bytes copied by the call */
    uint32_t launches;    /* kernels launched by the call */
    uint32_t reserved;
} astcb200_stats;

/* Replaces ASTCEncoder::ASTCEncoder(device) + init() (compression_pipeline.cpp:200-233). */
int astcb200_create(astcb200_ctx** out, int device_ordinal, const astcb200_config* cfg);
/* Replaces ASTCEncoder::~ASTCEncoder (compression_pipeline.cpp:537). */
int astcb200_destroy(astcb200_ctx* ctx);

/* Replaces ASTCEncoder::secondaryInit(textureWidth, textureHeight, blockXDim, blockYDim)
 * (compression_pipeline.cpp:263-321): builds the footprint's tables on the device. */
int astcb200_set_image(astcb200_ctx* ctx, uint32_t width, uint32_t height, uint8_t block_x, uint8_t block_y);
/* Changes astcb200_config.timeout_ms for later calls (no reference counterpart: the
 * reference's blocking map has no bound, webgpu_utils.h:79-87). */
int astcb200_set_timeout(astcb200_ctx* ctx, uint32_t timeout_ms);

/* ASTCEncoder::blocksX / blocksY (astc.h:736-737). */
int astcb200_blocks(const astcb200_ctx* ctx, uint32_t* blocks_x, uint32_t* blocks_y);

/* Replaces ASTCEncoder::encode(imageData, dataOut, dataLen) (compression_pipeline.cpp:323-535):
 * rgba8 is width*height*4 bytes in host memory; out_blocks receives blocks_x*blocks_y*16
 * bytes of physical ASTC blocks in raster order (out_len must be at least that). */
int astcb200_encode(astcb200_ctx* ctx, const uint8_t* rgba8, uint8_t* out_blocks, size_t out_len,
                    astcb200_stats* stats);

/* Same search with both buffers already in device memory of the context's GPU; work is
 * queued on cuda_stream (a cudaStream_t, or NULL for the context's stream) and the call
 * returns without waiting.  d_rgba8 must be 4-byte aligned, d_out_blocks 16-byte aligned. */
int astcb200_encode_device(astcb200_ctx* ctx, const uint8_t* d_rgba8, uint8_t* d_out_blocks, void* cuda_stream);

/* Encode without allocating (no counterpart in the reference).  For callers that cannot
 * call cudaMalloc -- an engine whose allocator owns the whole device heap, a plug-in in a
 * process with a fixed allocation policy.  Inputs and outputs are the caller's device
 * buffers (as for astcb200_encode_device); every intermediate, and the search tables of
 * each footprint used so far, live in one 52 MiB file-scope device array.  The CUDA
 * runtime commits that array on a device when the first call there resolves its address
 * (cudaGetSymbolAddress), and the device holds it until the process exits: make the
 * first call at start-up, before the caller's allocator reserves the heap
 * (ASTCB200_OOM if no room is left then).  The first call of each footprint on a device
 * also uploads that footprint's tables into the array (a synchronous copy) and sets the
 * kernels' shared-memory limits; make these first calls before any stream capture.
 * Later calls only queue kernels.  At most 2048 blocks per call (ASTCB200_TOO_LARGE
 * beyond).  All calls share the array and it keeps the last call's contents: calls that
 * overlap on the GPU race and must be serialised by the caller.  Always the exhaustive
 * search with the reference's semantics: no proposal network, no pruning.  Work is
 * queued on cuda_stream (NULL = the legacy default stream); no wait.  The caller's
 * current device is left as it was. */
int astcb200_encode_noalloc(int device_ordinal, const uint8_t* d_rgba8, uint32_t width, uint32_t height,
                            uint8_t block_x, uint8_t block_y, uint8_t* d_out_blocks, void* cuda_stream);

/* One texture of a batch (no reference counterpart: the reference encodes one image per
 * ASTCEncoder::encode call).  out_blocks receives ceil(width/block_x)*ceil(height/block_y)*16
 * bytes of physical blocks in raster order; out_len must be at least that. */
typedef struct astcb200_texture {
    const uint8_t* rgba8;  /* width*height*4 bytes, rows of width texels */
    uint8_t* out_blocks;
    size_t out_len;
    uint32_t width, height;
    uint8_t block_x, block_y; /* any of the 14 footprints; a batch may mix them */
    uint8_t reserved[6];
} astcb200_texture;

/* Encodes n textures of any sizes and footprints as one batch: the blocks of all textures
 * with the same footprint form one work queue searched by one launch sequence per chunk, the
 * footprints' queues run on concurrent streams, and the whole sequence is captured once per
 * batch shape (sizes and footprints) into a CUDA graph that later calls replay.  Host
 * pointers; blocks until the blocks are in out_blocks.  Each texture gets exactly the blocks
 * astcb200_encode gives it alone. */
int astcb200_encode_batch(astcb200_ctx* ctx, const astcb200_texture* textures, uint32_t n, astcb200_stats* stats);

/* Same with rgba8 and out_blocks in device memory of the context's GPU (rgba8 4-byte
 * aligned, out_blocks 16-byte aligned); queued on cuda_stream (NULL = the context's
 * stream), no wait.  The textures array itself is host memory and is consumed before the
 * call returns. */
int astcb200_encode_batch_device(astcb200_ctx* ctx, const astcb200_texture* textures, uint32_t n, void* cuda_stream);

/* Launch configuration of a batch shape, chosen by astcb200_autotune_batch. */
typedef struct astcb200_tuning {
    uint32_t chunk_blocks; /* blocks per launch sequence within one footprint's queue */
    uint32_t streams;      /* concurrent streams the footprints' queues are spread over */
    double ms;             /* device time of one batch with this configuration */
} astcb200_tuning;

/* Times every candidate configuration (chunk_blocks x streams) on this batch (device
 * pointers, as for astcb200_encode_batch_device; the outputs are written), keeps the
 * fastest for later batches of the same shape and returns it in best.  Candidates tried
 * are written to tried[0..*n_tried) when tried is not NULL (capacity max_tried).  Blocks. */
int astcb200_autotune_batch(astcb200_ctx* ctx, const astcb200_texture* textures, uint32_t n,
                            astcb200_tuning* best, astcb200_tuning* tried, uint32_t max_tried, uint32_t* n_tried);

/* Box-filters a device RGBA8 image to the next mip level: dst is max(1, width/2) x
 * max(1, height/2) texels, each the rounded mean (sum + 2) / 4 of the 2x2 source texels at
 * (2x, 2y)..(2x+1, 2y+1), source coordinates clamped to the image.  Queued on cuda_stream;
 * no wait.  (No reference counterpart: the reference encodes the image it is given.) */
int astcb200_downsample_device(const uint8_t* d_src, uint32_t width, uint32_t height, uint8_t* d_dst, void* cuda_stream);

/* ---- Learned proposal search (no reference counterpart) ----
 * A small network (inputs: a block's texels / 255 in bf16; two hidden layers of 256 ReLU
 * units; outputs: one logit per partitioning of P = 2..4, one for the single-partition
 * block, and one per block mode for each partition count) ranks the candidates; only the
 * best partitionings and, per partition count, the best block modes enter the search,
 * with fewer refinement candidates.  Blocks whose best partitionings carry too little
 * probability take the full search.  The final-error comparison still picks every block's
 * encoding.  Inference runs on the tensor cores (tcgen05, bf16 operands, FP32 accumulation). */

/* Output layout of a footprint's network: inputs (4 * texels), padded inputs, outputs
 * (a multiple of 128), block-mode classes per head, first block-mode logit and head
 * stride, and the number of selected partitionings of P = 2, 3, 4 (sel3[0..2]). */
int astcb200_proposal_layout(uint8_t block_x, uint8_t block_y, uint32_t* inputs, uint32_t* inputs_padded,
                             uint32_t* outputs, uint32_t* block_modes, uint32_t* head_base, uint32_t* head_stride,
                             uint32_t* sel3);

/* FP32 weights of one footprint's network (row-major, PyTorch Linear convention:
 * w1 [256 x inputs], w2 [256 x 256], w3 [outputs x 256]); converted to bf16 on upload. */
typedef struct astcb200_proposal_net {
    uint32_t struct_size;
    uint8_t block_x, block_y, reserved[2];
    uint32_t inputs, hidden, outputs; /* must match astcb200_proposal_layout and hidden = 256 */
    const float* w1;
    const float* b1;
    const float* w2;
    const float* b2;
    const float* w3;
    const float* b3;
} astcb200_proposal_net;
int astcb200_set_proposal_net(astcb200_ctx* ctx, const astcb200_proposal_net* net);

/* Zero in max_partitionings, block_modes, refine_candidates, refine_iterations or
 * fallback_iterations selects the footprint's tuned value, chosen on held-out synthetic
 * textures as the fastest setting within 0.1 dB mean PSNR of the full search with FIXED
 * semantics, no image losing more (with coverage 0.8): for blocks of up to 16 texels 8, 8,
 * 8, 6 and 3; for larger blocks 3, 4, 3, 6 and 3. */
typedef struct astcb200_pruning {
    uint32_t struct_size;
    uint32_t enable;            /* 0: full search everywhere */
    uint32_t max_partitionings; /* proposed partitionings per block, at most 16 (0 = tuned) */
    uint32_t block_modes;       /* block modes evaluated per partition count, at most 64 (0 = tuned) */
    uint32_t refine_candidates; /* refinement candidates per partitioned block, at most 8 (0 = tuned) */
    float coverage;             /* stop proposing once P=1 plus the proposed probability reaches this
                                   (0.8 suggested) */
    float threshold;            /* full search when P=1 plus the best max_partitionings carry less
                                   (textures of fewer than 1024 texels always take the full search,
                                   with the reference's 6 refinement iterations) */
    float reroute_error;        /* a block whose proposal-search result has a larger per-texel error
                                   (weighted squared, 8-bit units; weights R 0.675, G 1.3275,
                                   B 0.2475, A 1) also takes the full search, and the better of
                                   the two results is kept; 0 disables */
    uint32_t front_threads;     /* threads per CTA of the proposal pass's front kernel: 32, 64 or
                                   128 (0 = 64 for blocks of up to 16 texels, else 128); results
                                   do not depend on it */
    uint32_t refine_iterations; /* refinement iterations of the proposal pass, 1..6 (0 = tuned: 6,
                                   as the reference and the full search) */
    float single_partition_floor; /* blocks with proposed partitionings skip the single-partition
                                   candidate when its probability is below this (0 = never) */
    uint32_t fallback_iterations; /* refinement iterations of the full-search pass over the
                                   low-confidence and rerouted blocks, 1..6 (0 = tuned; 6 makes
                                   that pass the reference's full search) */
} astcb200_pruning;
/* Applies to later encodes of footprints that have a network (the others use the full search). */
int astcb200_set_pruning(astcb200_ctx* ctx, const astcb200_pruning* cfg);
/* Polls of each mbarrier wait in the network's inference kernel before its CTA gives up
 * (0 = the default, 2^24).  A CTA that gives up records it, waits for its own copies and
 * tensor-core work in flight to land (bounded by 2^24 polls) and returns; the encode that
 * launched it then reports ASTCB200_TIMEOUT from astcb200_pruning_stats,
 * astcb200_proposal_logits or astcb200_proposal_selection.  Small values exercise that
 * path in tests; limits below 65536 poll without suspending, so they give up as soon as a
 * wait finds the work still in flight. */
int astcb200_set_inference_wait_limit(astcb200_ctx* ctx, uint32_t polls);
/* Blocks that took the proposal search and the full search in the last encode call. */
int astcb200_pruning_stats(astcb200_ctx* ctx, uint64_t* proposal_blocks, uint64_t* full_blocks);
/* Test hook: the network's logits (blocks x outputs, FP32) for the image set by
 * astcb200_set_image, from host RGBA8. */
int astcb200_proposal_logits(astcb200_ctx* ctx, const uint8_t* rgba8, float* logits, size_t logits_len);
/* Test hook (no reference counterpart): the selection the proposal search makes for the
 * image set by astcb200_set_image, from host RGBA8, with the current pruning settings.
 * Per block (raster order, nblocks >= the image's block count): route[i] = 0 proposal
 * search, 1 full search; picks[i * 18 ...] = count n, flags (bit 0: P = 1 skipped), then
 * n partitionings (P - 2) << 10 | table entry; masks[i * 16 ...] = for P = 1..4, four
 * words of block-mode bits (valid block-mode order).  Full-search blocks get zeros. */
int astcb200_proposal_selection(astcb200_ctx* ctx, const uint8_t* rgba8, uint8_t* route, uint16_t* picks,
                                uint64_t* masks, size_t nblocks);

/* Training primitives of the proposal network (device pointers, FP32, queued on
 * cuda_stream, deterministic).  C[i][j] = sum_l A[i*sa_i + l*sa_l] * B[l*sb_l + j*sb_j]
 * (+ C when accumulate) (+ bias[j]) (ReLU when relu); C is row-major M x N. */
int astcb200_train_gemm(const float* A, const float* B, float* C, int M, int N, int K, int64_t sa_i, int64_t sa_l,
                        int64_t sb_l, int64_t sb_j, const float* bias, int relu, int accumulate, void* cuda_stream);
/* Softmax cross-entropy of the partition head and of the block-mode head of the label's
 * partition count; dZ (batch x outputs) receives the gradient divided by batch and
 * loss_rows (batch x 2) the two losses of each row.  sel3 is host memory. */
int astcb200_train_xent(const float* Z, uint32_t outputs, const int32_t* part_label, const int32_t* bm_label,
                        uint32_t batch, uint32_t block_modes, uint32_t head_stride, const uint32_t* sel3, float* dZ,
                        float* loss_rows, void* cuda_stream);
/* dH[i] = 0 where H[i] <= 0. */
int astcb200_train_relu_backward(float* dH, const float* H, size_t n, void* cuda_stream);
/* db[j] = sum over rows of dY[r][j]. */
int astcb200_train_colsum(const float* dY, float* db, uint32_t rows, uint32_t cols, void* cuda_stream);
/* One Adam step (bias-corrected with the 1-based step). */
int astcb200_train_adam(float* w, const float* g, float* m, float* v, size_t n, float lr, float beta1, float beta2,
                        float eps, uint32_t step, void* cuda_stream);

/* Debug / parity hook: returns the chosen SymbolicBlock of every block in the reference
 * layout (astc.h:639-655, 108 u32 per block) instead of physical blocks. */
int astcb200_encode_symbolic(astcb200_ctx* ctx, const uint8_t* rgba8, uint32_t* symbolic, size_t symbolic_words);

/* Replaces store_image(block_x, block_y, dim_x, dim_y, data, data_len, filename)
 * (astc_store.cpp:18-62): 16-byte .astc header then the blocks. */
int astcb200_store_image(uint32_t block_x, uint32_t block_y, uint32_t dim_x, uint32_t dim_y,
                         const uint8_t* data, size_t data_len, const char* filename);

/* .astc containers of images whose blocks are in device memory, for batch and mip-chain
 * outputs (no reference counterpart: store_image above writes one image from host memory).
 * For each image, host_out (pinned host memory for an asynchronous copy) receives the same
 * 16 bytes store_image writes, then the image's blocks copied from d_blocks by one
 * device-to-host copy queued on cuda_stream; the call returns once the copies are queued
 * (synchronise the stream before reading host_out).  out_len must be at least
 * 16 + 16 * blocks. */
typedef struct astcb200_astc_image {
    const uint8_t* d_blocks;  /* device, the image's blocks in raster order */
    uint8_t* host_out;
    size_t out_len;
    uint32_t width, height;
    uint8_t block_x, block_y;
    uint8_t reserved[6];
} astcb200_astc_image;
int astcb200_astc_containers_device(const astcb200_astc_image* images, uint32_t n, void* cuda_stream);

/* ASTC LDR decoder (no reference counterpart: the reference has none).  Decodes
 * blocks_x*blocks_y blocks of an image of dim_x*dim_y texels into rgba8_out
 * (dim_x*dim_y*4 bytes, UNORM8 with round-to-nearest from the 16-bit result). */
int astcb200_decode(uint32_t block_x, uint32_t block_y, uint32_t dim_x, uint32_t dim_y,
                    const uint8_t* blocks, size_t blocks_len, uint8_t* rgba8_out);
/* The same decoder on the GPU (no reference counterpart), between device buffers on the
 * current device, queued on cuda_stream: d_blocks holds the image's blocks in raster
 * order, d_rgba8 (4-byte aligned) receives dim_x*dim_y RGBA8 texels, exactly the texels
 * astcb200_decode gives. */
int astcb200_decode_device(uint32_t block_x, uint32_t block_y, uint32_t dim_x, uint32_t dim_y,
                           const uint8_t* d_blocks, uint8_t* d_rgba8, void* cuda_stream);
/* Decode and compare on the GPU without writing the image: d_sse[0..3] (device) receives,
 * per channel R, G, B, A, the sum over texels of the squared difference between the
 * decoded texels and the reference image d_ref_rgba8 (4-byte aligned).  PSNR over all
 * channels is 10 log10(255^2 * 4 * dim_x * dim_y / (d_sse[0] + ... + d_sse[3])). */
int astcb200_decode_error_device(uint32_t block_x, uint32_t block_y, uint32_t dim_x, uint32_t dim_y,
                                 const uint8_t* d_blocks, const uint8_t* d_ref_rgba8, uint64_t* d_sse,
                                 void* cuda_stream);

/* Test hook: the full search's first two stages for the image set by astcb200_set_image
 * (host RGBA8, at most one chunk of blocks): the partition search's picks (per block, 32
 * bytes: for P = 2, 3, 4 four table entries and their count, then padding) and the front's
 * partitioned-block records (per block 13 slots -- P = 1, then four per P = 2, 3, 4 -- of
 * 784 bytes: per partition the average, ep0 and ep1 as 4 floats each, then P, table entry,
 * candidate count and seed, then 8 candidates of 72 bytes: trial block-mode index (uint16),
 * colour quant level and its "mod" level, 4 endpoint formats, 64 quantised weights);
 * snapshots (optional): after the refinement's 6 iterations, each candidate's best state
 * (per block 13 x 8 records of 112 bytes: error, trial block-mode index (uint16), final quant
 * level, matched flag, 4 endpoint formats, 4 padding bytes, 32 packed endpoint values, 64
 * weights; inert slots have error 1e37). */
int astcb200_search_stages(astcb200_ctx* ctx, const uint8_t* rgba8, void* picks, size_t picks_bytes, void* records,
                           size_t records_bytes, void* snapshots, size_t snapshots_bytes);

/* Device milliseconds spent in each of the four kernels (partition search, front,
 * refine, select/pack) by the last encode call, summed over chunks; needs
 * ASTCB200_FLAG_STAGE_TIMING.  launches[4] receives the launch counts (optional).  The
 * proposal pass's refinement includes its tail pass, a second launch. */
int astcb200_stage_times(astcb200_ctx* ctx, float* ms4, uint32_t* launches4);

/* Per-launch device milliseconds of the last encode, summed over chunks by the launch's
 * position in its chunk's sequence (full search: 4 launches; proposal search: network,
 * selection, front, refine, select-pack of the proposal pass, then partition search, front,
 * refine, select-pack of the full-search pass); stage9 receives each position's stage
 * (0-3 as for astcb200_stage_times, -1 unused).  Needs ASTCB200_FLAG_STAGE_TIMING. */
int astcb200_stage_times_detail(astcb200_ctx* ctx, float* ms9, int32_t* stage9);

/* Work the search kernels did in the last encode with ASTCB200_FLAG_STAGE_TIMING (for
 * an operation-count roofline): [0..3] partitioned blocks searched by the front kernel by
 * partition count; [4] decimation modes and [5] block modes it evaluated; [6..9]
 * candidates refined by partition count; [10..12] partition searches for P = 2, 3, 4;
 * [13] candidates whose last iterations the refinement left to its tail pass (reserved
 * entries included). */
int astcb200_work_counters(astcb200_ctx* ctx, uint64_t* counters16);

const char* astcb200_status_string(int status);
const char* astcb200_last_error(const astcb200_ctx* ctx);

#ifdef __cplusplus
}
#endif

#endif /* ASTCB200_H */
