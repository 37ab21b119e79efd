// Test-only C shim over the reference's own CPU sources (compiled by
// oracle/build_ref.sh into oracle/_ref/libastcref.so).
//
// It is NOT part of the product and is never linked into it.  The tests use it
// to pin, bit for bit, the oracle's and the product's integer tables and
// physical packing against the reference implementation itself:
//   construct_metadata_structures   code/metadata_structures.cpp:338
//   init_partition_tables(_GPU)     code/partition_tables.cpp:415,438
//   construct_angular_tables        code/metadata_structures.cpp:463
//   get_ise_sequence_bitcount       code/physical_compression.cpp:625
//   encode_ise                      code/physical_compression.cpp:672
//   symbolic_to_physical            code/physical_compression.cpp:843
//   store_image                     code/astc_store.cpp:18
// The reference keeps its block_descriptor inside a heap-allocated
// ASTCEncoder (main.cpp: `new ASTCEncoder(device)`), so untouched table
// entries read as zero; the shim value-initialises its copy the same way.
#include <cstring>
#include <string>
#include <memory>
#include <map>
#include <vector>
#include "astc.h"
#include "astc_store.h"

namespace {

struct RefTables {
    block_descriptor* bd = nullptr;
    std::vector<float> sin_table, cos_table;
};

std::map<int, std::unique_ptr<block_descriptor>>& cache() {
    static std::map<int, std::unique_ptr<block_descriptor>> c;
    return c;
}

block_descriptor* get_bd(int bx, int by) {
    int key = bx * 256 + by;
    auto& c = cache();
    auto it = c.find(key);
    if (it != c.end()) return it->second.get();
    std::unique_ptr<block_descriptor> bd(new block_descriptor());
    construct_metadata_structures(bx, by, *bd);
    init_partition_tables(*bd, false, 4);
    init_partition_tables_GPU(*bd);
    block_descriptor* raw = bd.get();
    c[key] = std::move(bd);
    return raw;
}

}  // namespace

extern "C" {

// counts[0]=texel_count [1]=block_mode_count [2]=decimation_mode_count
// [3]=t2w entries [4]=w2t entries [5..8]=partitioning_count_selected[0..3]
// [9..12]=partitioning_count_all[0..3]
int astcref_counts(int bx, int by, uint32_t* counts) {
    block_descriptor* bd = get_bd(bx, by);
    counts[0] = bd->uniform_variables.texel_count;
    counts[1] = bd->uniform_variables.block_mode_count;
    counts[2] = bd->uniform_variables.decimation_mode_count;
    counts[3] = (uint32_t)bd->decimation_info_packed.texel_to_weight_map_data.size();
    counts[4] = (uint32_t)bd->decimation_info_packed.weight_to_texel_map_data.size();
    for (int i = 0; i < 4; i++) counts[5 + i] = bd->partitioning_count_selected[i];
    for (int i = 0; i < 4; i++) counts[9 + i] = bd->partitioning_count_all[i];
    return 0;
}

// bm_index: 2048 u32; bms: block_mode_count x 5 u32
// (mode_index, decimation_mode, quant_mode, weight_bits, is_dual_plane)
int astcref_block_modes(int bx, int by, uint32_t* bm_index, uint32_t* bms) {
    block_descriptor* bd = get_bd(bx, by);
    for (int i = 0; i < 2048; i++) bm_index[i] = bd->block_mode_index[i];
    for (uint32_t i = 0; i < bd->uniform_variables.block_mode_count; i++) {
        const block_mode& b = bd->block_modes[i];
        bms[i * 5 + 0] = b.mode_index;
        bms[i * 5 + 1] = b.decimation_mode;
        bms[i * 5 + 2] = b.quant_mode;
        bms[i * 5 + 3] = b.weight_bits;
        bms[i * 5 + 4] = b.is_dual_plane;
    }
    return 0;
}

// dmodes: dm_count x 4 u32; dinfo: dm_count x (8 + 144 + 144 + 64 + 64) u32
int astcref_decimation(int bx, int by, uint32_t* dmodes, uint32_t* dinfo) {
    block_descriptor* bd = get_bd(bx, by);
    const int stride = 8 + 144 + 144 + 64 + 64;
    for (uint32_t i = 0; i < bd->uniform_variables.decimation_mode_count; i++) {
        const decimation_mode& m = bd->decimation_modes[i];
        dmodes[i * 4 + 0] = m.maxprec_1plane;
        dmodes[i * 4 + 1] = m.maxprec_2planes;
        dmodes[i * 4 + 2] = m.refprec_1plane;
        dmodes[i * 4 + 3] = m.refprec_2planes;
        const decimation_info& d = bd->decimation_info_metadata[i];
        uint32_t* o = dinfo + (size_t)i * stride;
        o[0] = d.texel_count; o[1] = d.weight_count; o[2] = d.weight_x; o[3] = d.weight_y;
        o[4] = d.max_quant_level; o[5] = d.max_angular_steps; o[6] = d.max_quant_steps; o[7] = 0;
        for (int t = 0; t < 144; t++) o[8 + t] = d.texel_weight_count[t];
        for (int t = 0; t < 144; t++) o[152 + t] = d.texel_weights_offset[t];
        for (int w = 0; w < 64; w++) o[296 + w] = d.weight_texel_count[w];
        for (int w = 0; w < 64; w++) o[360 + w] = d.weight_texels_offset[w];
    }
    return 0;
}

int astcref_maps(int bx, int by, uint32_t* t2w_idx, float* t2w_c, uint32_t* w2t_idx, float* w2t_c) {
    block_descriptor* bd = get_bd(bx, by);
    const auto& a = bd->decimation_info_packed.texel_to_weight_map_data;
    const auto& b = bd->decimation_info_packed.weight_to_texel_map_data;
    for (size_t i = 0; i < a.size(); i++) { t2w_idx[i] = a[i].weight_index; t2w_c[i] = a[i].contribution; }
    for (size_t i = 0; i < b.size(); i++) { w2t_idx[i] = b[i].texel_index; w2t_c[i] = b[i].contribution; }
    return 0;
}

// pinfo: 3073 x (2 + 4 + 144) u32; cov2/3/4: 1024 x P u64; kmeans: 64 u32;
// packed_index: 3 x 1024 u16
int astcref_partitions(int bx, int by, uint32_t* pinfo, uint64_t* cov2, uint64_t* cov3,
                       uint64_t* cov4, uint32_t* kmeans, uint16_t* packed_index) {
    block_descriptor* bd = get_bd(bx, by);
    const int n = 3 * 1024 + 1;
    for (int i = 0; i < n; i++) {
        const partition_info_GPU& p = bd->partitionings_GPU[i];
        uint32_t* o = pinfo + (size_t)i * 150;
        o[0] = p.partition_count; o[1] = p.partition_index;
        for (int k = 0; k < 4; k++) o[2 + k] = p.partition_texel_count[k];
        for (int t = 0; t < 144; t++) o[6 + t] = p.partition_of_texel[t];
    }
    std::memcpy(cov2, bd->coverage_bitmaps_2, sizeof(bd->coverage_bitmaps_2));
    std::memcpy(cov3, bd->coverage_bitmaps_3, sizeof(bd->coverage_bitmaps_3));
    std::memcpy(cov4, bd->coverage_bitmaps_4, sizeof(bd->coverage_bitmaps_4));
    for (int i = 0; i < 64; i++) kmeans[i] = bd->kmeans_texels[i];
    std::memcpy(packed_index, bd->partitioning_packed_index, sizeof(bd->partitioning_packed_index));
    return 0;
}

int astcref_angular(float* sin_out, float* cos_out) {
    std::vector<float> s, c;
    construct_angular_tables(s, c);
    std::memcpy(sin_out, s.data(), s.size() * sizeof(float));
    std::memcpy(cos_out, c.data(), c.size() * sizeof(float));
    return (int)s.size();
}

unsigned int astcref_ise_bitcount(unsigned int count, int quant) {
    return get_ise_sequence_bitcount(count, static_cast<quant_method>(quant));
}

void astcref_encode_ise(int quant, unsigned int count, const uint8_t* in, uint8_t* out, unsigned int bit_offset) {
    encode_ise(static_cast<quant_method>(quant), count, in, out, bit_offset);
}

// sym: one SymbolicBlock in the reference layout (astc.h:639-655), 108 u32.
int astcref_symbolic_to_physical(int bx, int by, const uint32_t* sym, uint8_t* out16) {
    block_descriptor* bd = get_bd(bx, by);
    SymbolicBlock sb;
    static_assert(sizeof(SymbolicBlock) == 108 * 4, "SymbolicBlock layout");
    std::memcpy(&sb, sym, sizeof(SymbolicBlock));
    symbolic_to_physical(*bd, sb, out16);
    return 0;
}

int astcref_store_image(unsigned bx, unsigned by, unsigned w, unsigned h, uint8_t* data, size_t len, const char* path) {
    try {
        return store_image(bx, by, w, h, data, len, std::string(path));
    } catch (...) {
        return -1;
    }
}

}  // extern "C"
