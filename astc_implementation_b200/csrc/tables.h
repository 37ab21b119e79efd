// Host-side construction of the per-footprint search tables and of the
// footprint-independent quantisation tables, laid out for device memory.
//
// Reference counterparts (Jure-Z/ASTC_implementation):
//   construct_metadata_structures  code/metadata_structures.cpp:338-461
//   init_partition_tables(_GPU)    code/partition_tables.cpp:415-464
//   construct_angular_tables       code/metadata_structures.cpp:463-481
//   ASTCEncoder::initTrialModes    code/compression_pipeline.cpp:146-198
//   constant tables embedded in shaders/pass07, pass09, pass11, pass14, pass16
//   and code/physical_compression.cpp (ISE and scramble tables)
#pragma once
#include <stdint.h>
#include <vector>

namespace astcb200 {

constexpr int kMaxTexels = 144;
constexpr int kMaxWeights = 64;
constexpr int kMaxDms = 87;
constexpr int kMaxValidBms = 600;      // 12x12 has 521 single-plane trial block modes
constexpr int kNumCand = 8;            // TUNE_MAX_TRIAL_CANDIDATES (astc.h:72)
constexpr int kPartCandLimit = 128;    // TUNE_MAX_PARTITIONING_CANDIDATE_LIMIT (astc.h:25)

// One valid decimation mode, indexed by its trial lookup index.
struct DevDm {
    uint8_t W, wx, wy, max_quant_level;
    uint8_t max_angular_steps, max_quant_steps, pad0, pad1;
    uint16_t tw_base;   // first entry of this mode's per-texel lists in t2w[]
    uint16_t wt_base;   // first entry of this mode's per-weight lists in w2t[]
};

// One valid single-plane block mode, indexed by its trial lookup index.
struct DevBm {
    uint16_t mode_index;   // the 11-bit ASTC block mode
    uint8_t dm;            // decimation-mode trial lookup index
    uint8_t quant;         // weight quant method
    uint8_t weight_bits;
    uint8_t pad[3];
};

// Byte offsets of every table inside the device blob; passed to kernels by value.
struct TableLayout {
    int32_t bx, by, T, ndm, nbm;
    int32_t max_w;            // largest weight count over the valid decimation modes
    uint32_t count_selected[4];
    uint32_t kmeans[64];
    // footprint tables
    uint32_t off_dm;          // DevDm[ndm]
    uint32_t off_bm;          // DevBm[nbm]
    uint32_t off_tw_count;    // u8 [ndm][T]      weights per texel
    uint32_t off_tw_start;    // u16[ndm][T]      start entry (relative to dm.tw_base)
    uint32_t off_wt_count;    // u8 [ndm][64]     texels per weight
    uint32_t off_wt_start;    // u16[ndm][64]     start entry (relative to dm.wt_base)
    uint32_t off_t2w;         // u16 entries: weight index | (contribution*16) << 8
    uint32_t off_tw4;         // u64[ndm][T]: the texel's (up to 4) entries of t2w, padded with 0
                              // (weight 0, contribution 0), four u16 in list order
    uint32_t off_bm_order;    // u16[nbm]: block-mode trial indices sorted by decimation mode
    uint32_t off_dual;        // DevBm[ndual]: dual-plane block modes on trial decimation modes, in
                              // block-mode order (the optional dual-plane search; no reference use)
    int32_t ndual;
    uint32_t off_w2t;         // u16 entries: texel index  | (contribution*16) << 8
    uint32_t off_part_texel;  // u8 [3][1024][T]  partition of texel (P = 2..4)
    uint32_t off_part_info;   // u32[3][1024]     seed | count0<<10 | ... (see kernels)
    uint32_t off_part_counts; // u8 [3][1024][4]  texels per partition
    uint32_t off_cov;         // u64[3][1024][4]  coverage bitmaps over k-means texels
    uint32_t off_sin, off_cos;// f32[1024*16]
    // footprint-independent tables
    uint32_t off_q2u;         // u8 [142]  weight unquant values, sorted (pass07:12-37)
    uint32_t off_q2u_start;   // u8 [12]
    uint32_t off_qmt;         // i8 [10][128] quant mode table (pass11)
    uint32_t off_cu2u;        // u8 [17][512] colour quantise-unquantise (pass14), non-decreasing in idx
    uint32_t off_prev_next;   // u16[12][65] (pass16)
    uint32_t off_bqe;         // f32[17]    baseline quant error (pass09)
    uint32_t off_wscr;        // u8 [12][32] weight scramble map
    uint32_t off_cscr;        // u8 [17][256] colour uquant -> scrambled ISE value
    uint32_t off_trits;       // u8 [243]
    uint32_t off_quints;      // u8 [125]
    uint32_t total_bytes;
};

// Builds the tables for one footprint.  Returns false for footprints outside
// the 14 two-dimensional ASTC sizes the reference accepts (main.cpp:123-133).
bool build_tables(int bx, int by, TableLayout& layout, std::vector<uint8_t>& blob);

// Table dumps in the layout of oracle/ref_shim.cpp, so tests can digest them.
struct HostTables;
const HostTables* host_tables(int bx, int by);
bool valid_footprint(int bx, int by);

}  // namespace astcb200
