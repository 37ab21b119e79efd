// CPU oracle for the ASTC LDR block-compression search -- TEST INFRASTRUCTURE.
// See astc_oracle.h for the contract and parity status.  Only tests/,
// __graft_entry__.smoke() and bench.py's CPU-baseline leg use this library.
//
// Every function below cites the reference file:line it restates.  Paths are
// relative to the Jure-Z/ASTC_implementation checkout.
//
// Semantics fixed where the reference leaves them open (the "REF" mode):
//  S1  f32 arithmetic is IEEE single precision with no fused multiply-add; sums
//      the WGSL accumulates with float CAS atomics (order-dependent there) are
//      taken in ascending texel / weight order.
//  S2  WGSL min/max on floats return the non-NaN operand (IEEE minNum/maxNum);
//      clamp(x,lo,hi) = min(max(x,lo),hi).
//  S3  normalize(v) = v / sqrt(dot(v,v)), component-wise, so a zero vector gives NaN.
//  S4  dot(a,b) sums the component products left to right.
//  S5  f32 -> u32 / i32 conversions follow Tint's polyfill (saturating; NaN
//      gives the type's maximum), because Dawn compiles the WGSL with Tint.
//  S6  WGSL round() is round-half-to-even (nearbyint in the default mode).
//  S7  atan2 is the Cephes single-precision atan (S. L. Moshier) with quadrant
//      fix-up; atan2(0,0) = 0.  The product uses the same published method.
//  S8  pass001 ties in the farthest-point search: the highest texel index wins
//      ("last store wins" when invocations run in index order).
//  S9  REF-BUG-1 (pass004:184 stores at block*1024*i): stored at block*1024+i.
//      REF-BUG-3/5 (stride mismatches): in-bounds buffers of the shader's stride;
//      pass05 slots a dm never writes read 0.
//      REF-BUG-6 (pass07:322 packs floor(W/4) words): the tail weights read 0,
//      which is what the never-written words of the zero-initialised buffer hold.
//  S10 Partitioned-block slots pass007 does not fill (fewer than 4 distinct
//      picks) and candidate slots pass12 does not fill (fewer than 8 trials under
//      1e37) hold stale data of other blocks in the reference; here they are
//      inert: never refined, never chosen.
//  S11 Deterministic quirks are reproduced as written: the partial bitonic
//      network of pass005, the rank used as table index in pass007 (REF-BUG-4),
//      the per-invocation `avg`/`dir` arrays of pass006 (function-scope, so each
//      invocation only sees its own partition's values, the rest zero), integer
//      truncation of sums in pass003/006, pass17's float weight interpolation.
//
// The "FIXED" mode (orc_set_semantics(1)) keeps S1-S10 and repairs the
// deterministic bugs whose intent the source makes evident:
//  F1  REF-BUG-2: pass005 sorts all 1024 (score, index) pairs (the network of
//      pass005:66-94 compares only pairs whose lower index is below 256).
//  F2  REF-BUG-4: pass007 emits partition_ordering[rank], the table entry the
//      candidate was evaluated for, not the rank (pass007:93,107,156-157).
//  F3  REF-BUG-6: pass07 stores all W quantised weights (pass07:322 packs
//      floor(W/4) words, so the tail weights read 0).
//  F4  pass006 keeps `avg` and `dir` in function-scope arrays that each
//      invocation fills only for its own index (pass006:124-135,186-217), so
//      most texels see a zero average and direction; here every texel sees its
//      partition's values, as the workgroup-wide sums they come from intend.
#include "astc_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// ---------------------------------------------------------------- constants
constexpr int MAX_TEXELS = 144;
constexpr int MAX_WEIGHTS = 64;
constexpr int MAX_DMS = 87;
constexpr int NUM_CAND = 8;              // TUNE_MAX_TRIAL_CANDIDATES (astc.h:72)
constexpr int PART_CAND_LIMIT = 128;     // TUNE_MAX_PARTITIONING_CANDIDATE_LIMIT (astc.h:25)
constexpr float ERR_DEFAULT = 1e37f;     // ERROR_CALC_DEFAULT in the shaders
const float CW[4] = {0.30f * 2.25f, 0.59f * 2.25f, 0.11f * 2.25f, 1.0f};  // astc.h:60-63
const int LEVELS[21] = {2, 3, 4, 5, 6, 8, 10, 12, 16, 20, 24, 32, 40, 48, 64, 80, 96, 128, 160, 192, 256};
const int STEPS_FOR_QUANT[12] = {2, 3, 4, 5, 6, 8, 10, 12, 16, 20, 24, 32};  // astc.h:157
const int FREE_BITS[4] = {111, 111 - 4 - 10, 108 - 4 - 10, 105 - 4 - 10};    // pass07:5

// 0: REF semantics (the parity target), 1: FIXED (F1-F4 in the header).  Set before a call,
// read by every thread of it.
int g_fixed = 0;

enum {
    FMT_LUMINANCE = 0, FMT_LUMINANCE_DELTA = 1, FMT_LUMINANCE_ALPHA = 4, FMT_LUMINANCE_ALPHA_DELTA = 5,
    FMT_RGB_SCALE = 6, FMT_RGB = 8, FMT_RGB_DELTA = 9, FMT_RGB_SCALE_ALPHA = 10, FMT_RGBA = 12, FMT_RGBA_DELTA = 13
};

// ---------------------------------------------------------------- semantics helpers
struct v4 { float x, y, z, w; };
inline v4 V(float a) { return {a, a, a, a}; }
inline v4 operator+(v4 a, v4 b) { return {a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w}; }
inline v4 operator-(v4 a, v4 b) { return {a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w}; }
inline v4 operator*(v4 a, v4 b) { return {a.x * b.x, a.y * b.y, a.z * b.z, a.w * b.w}; }
inline v4 operator*(v4 a, float s) { return {a.x * s, a.y * s, a.z * s, a.w * s}; }
inline v4 operator/(v4 a, v4 b) { return {a.x / b.x, a.y / b.y, a.z / b.z, a.w / b.w}; }
inline v4 operator/(v4 a, float s) { return {a.x / s, a.y / s, a.z / s, a.w / s}; }
inline float dot4(v4 a, v4 b) { float r = a.x * b.x; r = r + a.y * b.y; r = r + a.z * b.z; r = r + a.w * b.w; return r; }
inline float dot3(v4 a, v4 b) { float r = a.x * b.x; r = r + a.y * b.y; r = r + a.z * b.z; return r; }
inline float fmn(float a, float b) { return std::fmin(a, b); }
inline float fmx(float a, float b) { return std::fmax(a, b); }
inline float clampf(float x, float lo, float hi) { return fmn(fmx(x, lo), hi); }
inline v4 vmax(v4 a, v4 b) { return {fmx(a.x, b.x), fmx(a.y, b.y), fmx(a.z, b.z), fmx(a.w, b.w)}; }
inline v4 vmin(v4 a, v4 b) { return {fmn(a.x, b.x), fmn(a.y, b.y), fmn(a.z, b.z), fmn(a.w, b.w)}; }
inline v4 normalize4(v4 v) { float l = std::sqrt(dot4(v, v)); return v / l; }
inline float rne(float x) { return std::nearbyint(x); }
inline uint32_t f2u(float v) {  // S5
    if (!(v <= 4294967040.0f)) return 4294967295u;
    if (v < 0.0f) return 0u;
    return (uint32_t)v;
}
inline int32_t f2i(float v) {  // S5
    if (!(v <= 2147483520.0f)) return 2147483647;
    if (v < -2147483648.0f) return (int32_t)0x80000000u;
    return (int32_t)v;
}
inline float& comp(v4& v, int c) { return (&v.x)[c]; }
inline float compc(const v4& v, int c) { return (&v.x)[c]; }

// S7: Cephes atanf, then atan2 quadrant logic.
float atan_pos(float x) {
    float y0;
    if (x > 2.414213562373095f) { y0 = 1.5707963267948966f; x = -1.0f / x; }
    else if (x > 0.4142135623730950f) { y0 = 0.7853981633974483f; x = (x - 1.0f) / (x + 1.0f); }
    else { y0 = 0.0f; }
    float z = x * x;
    float p = 8.05374449538e-2f * z;
    p = p - 1.38776856032e-1f; p = p * z;
    p = p + 1.99777106478e-1f; p = p * z;
    p = p - 3.33329491539e-1f; p = p * z;
    p = p * x; p = p + x;
    return y0 + p;
}
float atan2_ref(float y, float x) {
    if (std::isnan(x) || std::isnan(y)) return std::nanf("");
    float ax = std::fabs(x), ay = std::fabs(y);
    if (ax == 0.0f && ay == 0.0f) return 0.0f;
    float r = atan_pos(ay / ax);
    if (x < 0.0f) r = 3.14159265358979323846f - r;
    if (y < 0.0f) r = -r;
    return r;
}

// ---------------------------------------------------------------- ISE / quant tables (ASTC spec)
void btq(int q, int& bits, int& trits, int& quints) {
    int L = LEVELS[q];
    trits = quints = 0;
    if (L % 3 == 0) { trits = 1; L /= 3; } else if (L % 5 == 0) { quints = 1; L /= 5; }
    bits = 0; while ((1 << bits) < L) bits++;
}
// code/physical_compression.cpp:625 get_ise_sequence_bitcount
unsigned ise_bitcount(unsigned n, int q) {
    if (q < 0 || q > 20) return 1024;
    int b, t, qu; btq(q, b, t, qu);
    if (t) return (n * (8 + 5 * b) + 4) / 5;
    if (qu) return (n * (7 + 3 * b) + 2) / 3;
    return n * b;
}
// Weight unquantisation (ASTC spec, weight unquantisation), value 0..64.
int unq_weight(int q, int v) {
    int b, t, qu; btq(q, b, t, qu);
    int r;
    if (!t && !qu) {
        int val = 0, nb = 0;
        while (nb < 6) { val = (val << b) | v; nb += b; }
        r = val >> (nb - 6);
    } else {
        int D = v >> b, m = v & ((1 << b) - 1);
        int A = (m & 1) ? 0x7F : 0;
        int bb = (m >> 1) & 1, cc = (m >> 2) & 1;
        if (b == 0) {
            r = t ? (D == 0 ? 0 : D == 1 ? 32 : 63) : (D == 0 ? 0 : D == 1 ? 16 : D == 2 ? 32 : D == 3 ? 47 : 63);
        } else {
            int B, C;
            if (t) {
                if (b == 1) { B = 0; C = 50; }
                else if (b == 2) { B = (bb << 6) | (bb << 2) | bb; C = 23; }
                else { B = (cc << 6) | (bb << 5) | (cc << 1) | bb; C = 11; }
            } else {
                if (b == 1) { B = 0; C = 28; }
                else { B = (bb << 6) | (bb << 1); C = 13; }
            }
            int T = D * C + B; T ^= A; r = (A & 0x20) | (T >> 2);
        }
    }
    if (r > 32) r++;
    return r;
}
// Colour endpoint unquantisation (ASTC spec), value 0..255.
int unq_color(int q, int v) {
    int b, t, qu; btq(q, b, t, qu);
    if (!t && !qu) {
        int val = 0, nb = 0;
        while (nb < 8) { val = (val << b) | v; nb += b; }
        return val >> (nb - 8);
    }
    int D = v >> b, m = v & ((1 << b) - 1);
    int A = (m & 1) ? 0x1FF : 0;
    auto bit = [&](int i) { return (m >> i) & 1; };
    int B = 0, C = 0;
    if (t) {
        static const int Cs[7] = {0, 204, 93, 44, 22, 11, 5};
        C = Cs[b];
        if (b == 2) B = (bit(1) << 8) | (bit(1) << 4) | (bit(1) << 2) | (bit(1) << 1);
        else if (b == 3) B = (bit(2) << 8) | (bit(1) << 7) | (bit(2) << 3) | (bit(1) << 2) | (bit(2) << 1) | bit(1);
        else if (b == 4) B = (bit(3) << 8) | (bit(2) << 7) | (bit(1) << 6) | (bit(3) << 2) | (bit(2) << 1) | bit(1);
        else if (b == 5) B = (bit(4) << 8) | (bit(3) << 7) | (bit(2) << 6) | (bit(1) << 5) | (bit(4) << 1) | bit(3);
        else if (b == 6) B = (bit(5) << 8) | (bit(4) << 7) | (bit(3) << 6) | (bit(2) << 5) | (bit(1) << 4) | bit(5);
    } else {
        static const int Cs[6] = {0, 113, 54, 26, 13, 6};
        C = Cs[b];
        if (b == 2) B = (bit(1) << 8) | (bit(1) << 3) | (bit(1) << 2);
        else if (b == 3) B = (bit(2) << 8) | (bit(1) << 7) | (bit(2) << 2) | (bit(1) << 1) | bit(2);
        else if (b == 4) B = (bit(3) << 8) | (bit(2) << 7) | (bit(1) << 6) | (bit(3) << 1) | bit(2);
        else if (b == 5) B = (bit(4) << 8) | (bit(3) << 7) | (bit(2) << 6) | (bit(1) << 5) | bit(4);
    }
    int T = D * C + B; T ^= A;
    return (A & 0x80) | (T >> 2);
}
void decode_trits(int T, int out[5]) {
    auto bit = [](int x, int i) { return (x >> i) & 1; };
    int C, t4, t3, t2, t1, t0;
    if (((T >> 2) & 7) == 7) { C = (((T >> 5) & 7) << 2) | (T & 3); t4 = 2; t3 = 2; }
    else {
        C = T & 31;
        if (((T >> 5) & 3) == 3) { t4 = 2; t3 = bit(T, 7); } else { t4 = bit(T, 7); t3 = (T >> 5) & 3; }
    }
    if ((C & 3) == 3) { t2 = 2; t1 = bit(C, 4); t0 = (bit(C, 3) << 1) | (bit(C, 2) & (1 - bit(C, 3))); }
    else if (((C >> 2) & 3) == 3) { t2 = 2; t1 = 2; t0 = C & 3; }
    else { t2 = bit(C, 4); t1 = (C >> 2) & 3; t0 = (bit(C, 1) << 1) | (bit(C, 0) & (1 - bit(C, 1))); }
    out[0] = t0; out[1] = t1; out[2] = t2; out[3] = t3; out[4] = t4;
}
void decode_quints(int Q, int out[3]) {
    auto bit = [](int x, int i) { return (x >> i) & 1; };
    int q0, q1, q2, C;
    if (((Q >> 1) & 3) == 3 && ((Q >> 5) & 3) == 0) {
        q2 = (bit(Q, 0) << 2) | ((bit(Q, 4) & (1 - bit(Q, 0))) << 1) | (bit(Q, 3) & (1 - bit(Q, 0)));
        q1 = 4; q0 = 4;
    } else {
        if (((Q >> 1) & 3) == 3) { q2 = 4; C = (((Q >> 3) & 3) << 3) | (((~Q >> 5) & 3) << 1) | (Q & 1); }
        else { q2 = (Q >> 5) & 3; C = Q & 31; }
        if ((C & 7) == 5) { q1 = 4; q0 = (C >> 3) & 3; } else { q1 = (C >> 3) & 3; q0 = C & 7; }
    }
    out[0] = q0; out[1] = q1; out[2] = q2;
}

struct ConstTables {
    int32_t q2u[142];             // pass07:12-37
    int32_t q2u_off[12];          // pass07:8
    int32_t qmt[10][128];         // pass11_*:12-64
    int32_t cu2u[17][512];        // pass14:29-319
    int32_t prev_next[12][65];    // pass16:13-74
    float bqe[17];                // pass09:10-28
    uint8_t trits[3][3][3][3][3]; // physical_compression.cpp:44 (indexed [t4][t3][t2][t1][t0])
    uint8_t quints[5][5][5];      // physical_compression.cpp:207 (indexed [q2][q1][q0])
    uint8_t wscr[12][32];         // physical_compression.cpp:249
    uint8_t cscr[17][256];        // physical_compression.cpp:284
    ConstTables() {
        int off = 0;
        for (int q = 0; q < 12; q++) {
            int L = LEVELS[q];
            std::vector<std::pair<int, int>> vals;
            for (int v = 0; v < L; v++) vals.push_back({unq_weight(q, v), v});
            std::sort(vals.begin(), vals.end());
            q2u_off[q] = off;
            std::memset(wscr[q], 0, 32);
            for (int k = 0; k < L; k++) { q2u[off + k] = vals[k].first; wscr[q][k] = (uint8_t)vals[k].second; }
            for (int v = 0; v <= 64; v++) prev_next[q][v] = 0;
            for (int k = 0; k < L; k++) {
                int prev = vals[std::max(k - 1, 0)].first, next = vals[std::min(k + 1, L - 1)].first;
                prev_next[q][vals[k].first] = prev | (next << 8);
            }
            off += L;
        }
        for (int i = 0; i < 10; i++) for (int j = 0; j < 128; j++) qmt[i][j] = -1;
        for (int i = 0; i < 21; i++)
            for (int j = 1; j <= 9; j++) { unsigned p = ise_bitcount(2 * j, i); if (p < 128) qmt[j][p] = i; }
        for (int i = 0; i < 10; i++) { int l = -1; for (int j = 0; j < 128; j++) { l = std::max(l, qmt[i][j]); qmt[i][j] = l; } }
        for (int qi = 0; qi < 17; qi++) {
            int q = qi + 4, L = LEVELS[q];
            std::vector<int> vals(L);
            for (int v = 0; v < L; v++) vals[v] = unq_color(q, v);
            std::vector<int> sorted = vals; std::sort(sorted.begin(), sorted.end());
            for (int i = 0; i < 512; i++) {  // nearest; ties: even index -> lower, odd -> upper
                int v = i >> 1, bd = 1 << 30, bu = 0;
                for (int u : sorted) { int d = std::abs(u - v); if (d < bd || (d == bd && (i & 1))) { bd = d; bu = u; } }
                cu2u[qi][i] = bu;
            }
            for (int v = 0; v < 256; v++) {  // nearest; ties -> higher ISE code
                int bd = 1 << 30, be = 0;
                for (int e = 0; e < L; e++) { int d = std::abs(vals[e] - v); if (d <= bd) { bd = d; be = e; } }
                cscr[qi][v] = (uint8_t)be;
            }
        }
        const float base = (65536.0f * 65536.0f) / 18.0f;
        const int divs[17] = {5, 7, 9, 11, 15, 19, 23, 31, 39, 47, 63, 79, 95, 127, 159, 191, 255};
        for (int i = 0; i < 17; i++) bqe[i] = base / (float)(divs[i] * divs[i]);
        // trits/quints: the largest code that decodes to each tuple
        for (int T = 0; T < 256; T++) { int d[5]; decode_trits(T, d); trits[d[4]][d[3]][d[2]][d[1]][d[0]] = (uint8_t)T; }
        for (int Q = 0; Q < 128; Q++) { int d[3]; decode_quints(Q, d); quints[d[2]][d[1]][d[0]] = (uint8_t)Q; }
    }
};
const ConstTables& CT() { static ConstTables t; return t; }

// ---------------------------------------------------------------- footprint tables
struct BlockMode { uint32_t mode_index, dm, quant, weight_bits, dual; };
struct DecInfo {
    uint32_t T, W, wx, wy, max_quant_level, max_angular_steps, max_quant_steps;
    uint32_t tw_count[MAX_TEXELS], tw_off[MAX_TEXELS], wt_count[MAX_WEIGHTS], wt_off[MAX_WEIGHTS];
};
struct DecMode { uint32_t maxprec1, maxprec2, refprec1, refprec2; };
struct PartInfo { uint32_t count, index, texel_count[4], of_texel[MAX_TEXELS]; };
struct Footprint {
    int bx, by, T;
    uint32_t bm_index[2048];
    std::vector<BlockMode> bms;
    std::vector<DecInfo> dis;
    std::vector<DecMode> dms;
    std::vector<uint32_t> t2w_idx, w2t_idx;
    std::vector<float> t2w_c, w2t_c;
    std::vector<PartInfo> pinfo;           // 3*1024+1
    uint32_t count_selected[4], count_all[4];
    std::vector<uint64_t> cov[5];          // cov[P]: 1024*P
    uint32_t kmeans[64];
    uint16_t packed_index[3][1024];
    std::vector<uint32_t> valid_dms;
    std::vector<std::pair<uint32_t, uint32_t>> valid_bms;  // (packed bm, dm lookup)
    std::vector<float> sin_t, cos_t;
};

// code/metadata_structures.cpp:72-173
bool decode_block_mode_2d(unsigned bm, unsigned& xw, unsigned& yw, bool& dual, unsigned& qm, unsigned& wbits) {
    unsigned base_q = (bm >> 4) & 1, H = (bm >> 9) & 1, D = (bm >> 10) & 1, A = (bm >> 5) & 3;
    xw = yw = 0;
    if ((bm & 3) != 0) {
        base_q |= (bm & 3) << 1;
        unsigned B = (bm >> 7) & 3;
        switch ((bm >> 2) & 3) {
            case 0: xw = B + 4; yw = A + 2; break;
            case 1: xw = B + 8; yw = A + 2; break;
            case 2: xw = A + 2; yw = B + 8; break;
            default:
                B &= 1;
                if (bm & 0x100) { xw = B + 2; yw = A + 2; } else { xw = A + 2; yw = B + 6; }
        }
    } else {
        base_q |= ((bm >> 2) & 3) << 1;
        if (((bm >> 2) & 3) == 0) return false;
        unsigned B = (bm >> 9) & 3;
        switch ((bm >> 7) & 3) {
            case 0: xw = 12; yw = A + 2; break;
            case 1: xw = A + 2; yw = 12; break;
            case 2: xw = A + 6; yw = B + 6; D = 0; H = 0; break;
            default:
                switch ((bm >> 5) & 3) {
                    case 0: xw = 6; yw = 10; break;
                    case 1: xw = 10; yw = 6; break;
                    default: return false;
                }
        }
    }
    unsigned wc = xw * yw * (D + 1);
    qm = (base_q - 2) + 6 * H;
    dual = D != 0;
    wbits = ise_bitcount(wc, (int)qm);
    return wc <= 64 && wbits >= 24 && wbits <= 96;
}

// code/metadata_structures.cpp:176-275
void init_decimation(Footprint& f, unsigned xw, unsigned yw, DecInfo& d) {
    unsigned xt = f.bx, yt = f.by, T = xt * yt, W = xw * yw;
    uint8_t wcount_t[MAX_TEXELS] = {0}, gw_t[MAX_TEXELS][4], w_t[MAX_TEXELS][4];
    uint8_t tcount_w[MAX_WEIGHTS] = {0};
    static thread_local uint8_t t_w[MAX_WEIGHTS][MAX_TEXELS], tw_w[MAX_WEIGHTS][MAX_TEXELS];
    for (unsigned y = 0; y < yt; y++)
        for (unsigned x = 0; x < xt; x++) {
            unsigned texel = y * xt + x;
            unsigned x_weight = (((1024 + xt / 2) / (xt - 1)) * x * (xw - 1) + 32) >> 6;
            unsigned y_weight = (((1024 + yt / 2) / (yt - 1)) * y * (yw - 1) + 32) >> 6;
            unsigned xf = x_weight & 0xF, yf = y_weight & 0xF, xi = x_weight >> 4, yi = y_weight >> 4;
            unsigned qw[4], w[4];
            qw[0] = xi + yi * xw; qw[1] = qw[0] + 1; qw[2] = qw[0] + xw; qw[3] = qw[2] + 1;
            unsigned prod = xf * yf;
            w[3] = (prod + 8) >> 4; w[1] = xf - w[3]; w[2] = yf - w[3]; w[0] = 16 - xf - yf + w[3];
            for (int i = 0; i < 4; i++)
                if (w[i] != 0) {
                    uint8_t ti = wcount_t[texel]++;
                    gw_t[texel][ti] = (uint8_t)qw[i]; w_t[texel][ti] = (uint8_t)w[i];
                    uint8_t wi = tcount_w[qw[i]]++;
                    t_w[qw[i]][wi] = (uint8_t)texel; tw_w[qw[i]][wi] = (uint8_t)w[i];
                }
        }
    std::memset(&d, 0, sizeof(d));
    d.tw_off[0] = (uint32_t)f.t2w_idx.size();
    for (unsigned i = 0; i < T; i++) {
        d.tw_count[i] = wcount_t[i];
        if (i > 0) d.tw_off[i] = d.tw_off[i - 1] + d.tw_count[i - 1];
        for (unsigned j = 0; j < wcount_t[i]; j++) {
            f.t2w_idx.push_back(gw_t[i][j]);
            f.t2w_c.push_back((float)w_t[i][j] * (1.0f / 16.0f));
        }
    }
    d.wt_off[0] = (uint32_t)f.w2t_idx.size();
    for (unsigned i = 0; i < W; i++) {
        d.wt_count[i] = tcount_w[i];
        if (i > 0) d.wt_off[i] = d.wt_off[i - 1] + d.wt_count[i - 1];
        for (unsigned j = 0; j < tcount_w[i]; j++) {
            f.w2t_idx.push_back(t_w[i][j]);
            f.w2t_c.push_back((float)tw_w[i][j] * (1.0f / 16.0f));
        }
    }
    d.T = T; d.W = W; d.wx = xw; d.wy = yw;
}

uint64_t rotl64(uint64_t v, int c) { return (v << c) | (v >> (64 - c)); }

// code/partition_tables.cpp:92-241
uint32_t hash52(uint32_t inp) {
    inp ^= inp >> 15; inp *= 0xEEDE0891; inp ^= inp >> 5; inp += inp << 16;
    inp ^= inp >> 7; inp ^= inp >> 3; inp ^= inp << 6; inp ^= inp >> 17;
    return inp;
}
uint8_t select_partition(int seed, int x, int y, int z, int pc, bool small) {
    if (small) { x <<= 1; y <<= 1; z <<= 1; }
    seed += (pc - 1) * 1024;
    uint32_t rnum = hash52(seed);
    uint8_t s[13];
    s[1] = rnum & 0xF; s[2] = (rnum >> 4) & 0xF; s[3] = (rnum >> 8) & 0xF; s[4] = (rnum >> 12) & 0xF;
    s[5] = (rnum >> 16) & 0xF; s[6] = (rnum >> 20) & 0xF; s[7] = (rnum >> 24) & 0xF; s[8] = (rnum >> 28) & 0xF;
    s[9] = (rnum >> 18) & 0xF; s[10] = (rnum >> 22) & 0xF; s[11] = (rnum >> 26) & 0xF;
    s[12] = ((rnum >> 30) | (rnum << 2)) & 0xF;
    for (int i = 1; i <= 12; i++) s[i] = (uint8_t)(s[i] * s[i]);
    int sh1, sh2;
    if (seed & 1) { sh1 = (seed & 2 ? 4 : 5); sh2 = (pc == 3 ? 6 : 5); }
    else { sh1 = (pc == 3 ? 6 : 5); sh2 = (seed & 2 ? 4 : 5); }
    int sh3 = (seed & 0x10) ? sh1 : sh2;
    s[1] >>= sh1; s[2] >>= sh2; s[3] >>= sh1; s[4] >>= sh2; s[5] >>= sh1; s[6] >>= sh2; s[7] >>= sh1; s[8] >>= sh2;
    s[9] >>= sh3; s[10] >>= sh3; s[11] >>= sh3; s[12] >>= sh3;
    int a = s[1] * x + s[2] * y + s[11] * z + (rnum >> 14);
    int b = s[3] * x + s[4] * y + s[12] * z + (rnum >> 10);
    int c = s[5] * x + s[6] * y + s[9] * z + (rnum >> 6);
    int d = s[7] * x + s[8] * y + s[10] * z + (rnum >> 2);
    a &= 0x3F; b &= 0x3F; c &= 0x3F; d &= 0x3F;
    if (pc <= 3) d = 0;
    if (pc <= 2) c = 0;
    if (pc <= 1) b = 0;
    if (a >= b && a >= c && a >= d) return 0;
    if (b >= c && b >= d) return 1;
    if (c >= d) return 2;
    return 3;
}

std::unique_ptr<Footprint> build_footprint(int bx, int by) {
    std::unique_ptr<Footprint> fp(new Footprint());
    Footprint& f = *fp;
    f.bx = bx; f.by = by; f.T = bx * by;
    // code/metadata_structures.cpp:338-461 construct_metadata_structures
    int dm_index[12 * 16 + 12 + 1];
    for (auto& v : dm_index) v = -1;
    f.dis.reserve(MAX_DMS);
    for (unsigned i = 0; i < 2048; i++) {
        unsigned xw, yw, qm, wb; bool dual;
        bool valid = decode_block_mode_2d(i, xw, yw, dual, qm, wb);
        if (!valid || xw > (unsigned)bx || yw > (unsigned)by) { f.bm_index[i] = 0xFFFF; continue; }
        if (dual) { if ((int)(109 - wb) <= 0) { f.bm_index[i] = 0xFFFF; continue; } }
        else { if ((int)(111 - wb) <= 0) { f.bm_index[i] = 0xFFFF; continue; } }
        int dm = dm_index[yw * 16 + xw];
        if (dm < 0) {
            DecInfo d; init_decimation(f, xw, yw, d);
            unsigned W = xw * yw;
            bool try2 = 2 * W <= 64;
            int mp1 = -1, mp2 = -1;
            for (int q = 0; q < 12; q++) {
                unsigned b1 = ise_bitcount(W, q);
                if (b1 >= 24 && b1 <= 96) mp1 = q;
                if (try2) { unsigned b2 = ise_bitcount(2 * W, q); if (b2 >= 24 && b2 <= 96) mp2 = q; }
            }
            DecMode m;
            m.maxprec1 = (uint32_t)(int32_t)(int8_t)mp1; m.maxprec2 = (uint32_t)(int32_t)(int8_t)mp2;
            m.refprec1 = 0; m.refprec2 = 0;
            if (mp1 >= 0) {  // metadata_structures.cpp:327-335 (mp1 < 0 is masked to 0)
                int maxp = std::min(std::min(mp1, 7), 7);
                d.max_quant_level = maxp; d.max_angular_steps = STEPS_FOR_QUANT[maxp];
                d.max_quant_steps = STEPS_FOR_QUANT[maxp];
            }
            f.dis.push_back(d); f.dms.push_back(m);
            dm = (int)f.dis.size() - 1;
            dm_index[yw * 16 + xw] = dm;
        }
        BlockMode b{i, (uint32_t)dm, qm, wb, (uint32_t)dual};
        if (dual) f.dms[dm].refprec2 |= 1u << qm; else f.dms[dm].refprec1 |= 1u << qm;
        f.bm_index[i] = (uint32_t)f.bms.size();
        f.bms.push_back(b);
    }
    // code/metadata_structures.cpp:33-70 assign_kmeans_texels
    std::memset(f.kmeans, 0, sizeof(f.kmeans));
    if (f.T <= 64) { for (int i = 0; i < f.T; i++) f.kmeans[i] = i; }
    else {
        uint64_t st[2] = {0xfaf9e171cea1ec6bULL, 0xf1b318cc06af5d71ULL};
        bool seen[MAX_TEXELS] = {false};
        unsigned set = 0;
        while (set < 64) {
            uint64_t s0 = st[0], s1 = st[1], res = s0 + s1;
            s1 ^= s0; st[0] = rotl64(s0, 24) ^ s1 ^ (s1 << 16); st[1] = rotl64(s1, 37);
            uint8_t texel = (uint8_t)res; texel = texel % f.T;
            if (!seen[texel]) { f.kmeans[set++] = texel; seen[texel] = true; }
        }
    }
    // code/partition_tables.cpp:243-436
    f.pinfo.assign(3 * 1024 + 1, PartInfo());
    for (auto& p : f.pinfo) std::memset(&p, 0, sizeof(p));
    std::memset(f.packed_index, 0, sizeof(f.packed_index));
    for (int P = 2; P <= 4; P++) f.cov[P].assign(1024 * P, 0);
    bool small = f.T < 32;
    auto gen_entry = [&](int pc, int idx, int remap, PartInfo& pi) {
        int counts[4] = {0, 0, 0, 0}, t = 0;
        for (int y = 0; y < by; y++)
            for (int x = 0; x < bx; x++) {
                uint8_t part = select_partition(idx, x, y, 0, pc, small);
                counts[part]++;
                pi.of_texel[t++] = part;
            }
        for (int i = t; i < MAX_TEXELS; i++) pi.of_texel[i] = 0;
        pi.count = counts[0] == 0 ? 0 : counts[1] == 0 ? 1 : counts[2] == 0 ? 2 : counts[3] == 0 ? 3 : 4;
        pi.index = idx;
        for (int i = 0; i < 4; i++) pi.texel_count[i] = counts[i];
        if (pc >= 2) {
            uint64_t* bm = &f.cov[pc][(size_t)remap * pc];
            for (int i = 0; i < pc; i++) bm[i] = 0;
            int n = std::min(f.T, 64);
            for (int i = 0; i < n; i++) bm[pi.of_texel[f.kmeans[i]]] |= 1ULL << i;
        }
        return (int)pi.count == pc;
    };
    gen_entry(1, 0, 0, f.pinfo[3 * 1024]);
    f.count_selected[0] = f.count_all[0] = 1;
    for (int P = 2; P <= 4; P++) {
        PartInfo* tab = &f.pinfo[(P - 2) * 1024];
        std::vector<uint64_t> canon(1024 * 5, 0);
        auto canonical = [&](const PartInfo& pi, uint64_t* bp) {
            for (int i = 0; i < 5; i++) bp[i] = 0;
            int mapped[4] = {-1, -1, -1, -1}, n = 0;
            for (int i = 0; i < f.T; i++) {
                int index = pi.of_texel[i];
                if (mapped[index] < 0) mapped[index] = n++;
                uint64_t xl = (uint64_t)mapped[index];
                bp[i >> 5] |= xl << (2 * (i & 0x1F));
            }
        };
        unsigned next = 0; f.count_selected[P - 1] = 0; f.count_all[P - 1] = 0;
        uint8_t built[1024] = {0};
        for (int pass = 0; pass < 2; pass++)
            for (int i = 0; i < 1024; i++) {
                if (pass == 1 && built[i]) continue;
                bool useful = gen_entry(P, i, next, tab[next]);
                if (pass == 0 && !useful) continue;
                canonical(tab[next], &canon[next * 5]);
                bool keep = true;
                // partition_tables.cpp:59-83: the `#if BIT_PATTERN_WORDS > N` guards see the
                // undefined macro operand as 0, so only the first word (texels 0..31) is compared.
                for (unsigned j = 0; j < next; j++)
                    if (canon[next * 5] == canon[j * 5]) { keep = false; break; }
                if (useful && keep) {
                    if (pass == 0) {
                        f.packed_index[P - 2][i] = (uint16_t)next; f.count_selected[P - 1]++; f.count_all[P - 1]++;
                        built[i] = 1; next++;
                    }
                } else if (pass == 1) {
                    f.packed_index[P - 2][i] = (uint16_t)next; f.count_all[P - 1]++; next++;
                }
            }
    }
    // code/compression_pipeline.cpp:146-198 initTrialModes
    std::vector<uint32_t> remap(MAX_DMS, 0xFFFF);
    uint32_t mask = (1u << (7 + 1)) - 1;  // min(QUANT_32, quant_limit=QUANT_12)
    for (uint32_t m = 0; m < f.dms.size(); m++) {
        if ((f.dms[m].refprec1 & mask) == 0) continue;
        remap[m] = (uint32_t)f.valid_dms.size();
        f.valid_dms.push_back(m);
    }
    for (uint32_t i = 0; i < 2048; i++) {
        uint32_t p = f.bm_index[i];
        if (p == 0xFFFF) continue;
        const BlockMode& b = f.bms[p];
        if (b.dual) continue;
        if (remap[b.dm] == 0xFFFF) continue;
        f.valid_bms.push_back({p, remap[b.dm]});
    }
    // code/metadata_structures.cpp:463-481 construct_angular_tables
    f.sin_t.resize(1024 * 16); f.cos_t.resize(1024 * 16);
    const float PIf = 3.14159265358979323846f;
    for (unsigned i = 0; i < 16; i++) {
        float step = (float)(i + 1);
        for (unsigned j = 0; j < 1024; j++) {
            float angle = (2.0f * PIf / (1024u - 1.0f)) * step * (float)j;
            f.sin_t[j * 16 + i] = std::sin(angle);
            f.cos_t[j * 16 + i] = std::cos(angle);
        }
    }
    return fp;
}

const Footprint* get_fp(int bx, int by) {
    static std::mutex mu;
    static std::map<int, std::unique_ptr<Footprint>> cache;
    std::lock_guard<std::mutex> lock(mu);
    int key = bx * 256 + by;
    auto it = cache.find(key);
    if (it != cache.end()) return it->second.get();
    auto fp = build_footprint(bx, by);
    const Footprint* raw = fp.get();
    cache[key] = std::move(fp);
    return raw;
}

bool valid_footprint(int bx, int by) {
    static const int v[14][2] = {{4, 4}, {5, 4}, {5, 5}, {6, 5}, {6, 6}, {8, 5}, {8, 6}, {10, 5}, {10, 6}, {8, 8}, {10, 8}, {10, 10}, {12, 10}, {12, 12}};
    for (auto& p : v) if (p[0] == bx && p[1] == by) return true;
    return false;
}

// ---------------------------------------------------------------- per-block data
struct InputBlock {  // code/astc.h:508-517
    v4 px[MAX_TEXELS];
    uint32_t tp[MAX_TEXELS];
    uint32_t pcount[4];
    uint32_t pidx, gray, calpha;
};
struct PartEW { v4 avg, dir, ep0, ep1; };
struct IdealEW { PartEW part[4]; float w[MAX_TEXELS]; float wes[MAX_TEXELS]; uint32_t is_const; float min_cutoff; };
struct LHW { float lowest; int32_t span; float err, cl, ch; };
struct QuantRes { float error; int32_t bitcount; uint32_t qw[MAX_WEIGHTS]; };
struct ECE { float rgb_scale, rgb_luma, lum, alpha_drop; uint32_t can_offset, can_bc; };
struct Combo { float error; uint32_t fmt[4]; };
struct CCR { float total; uint32_t ql, qlm; uint32_t fmt[4]; };
struct Cand {
    uint32_t bm, bm_lookup; float total_error; uint32_t ql, qlm, matched, final_q;
    uint32_t fmt[4]; uint32_t qw[MAX_WEIGHTS]; PartEW part[4]; uint32_t ffmt[4]; uint32_t packed[32];
};
struct Sym { float err; uint32_t mode_index, pc, pidx, matched, quant; uint32_t fmt[4]; uint32_t packed[32]; uint32_t qw[MAX_WEIGHTS]; };

// code/compression_pipeline.cpp:7-86 SplitImageIntoBlocks (one block)
void make_block(const uint8_t* img, int w, int h, int bx, int by, int bxi, int byi, InputBlock& b) {
    std::memset(&b, 0, sizeof(b));
    float amin = 1e38f, amax = 0.0f;
    bool gray = true;
    int t = 0;
    for (int dy = 0; dy < by; dy++) {
        int y = std::min(byi * by + dy, h - 1);
        for (int dx = 0; dx < bx; dx++) {
            int x = std::min(bxi * bx + dx, w - 1);
            const uint8_t* p = img + ((size_t)y * w + x) * 4;
            for (int c = 0; c < 4; c++) {
                float v = (p[c] / 255.0f) * 65536.0f;
                comp(b.px[t], c) = v;
                if (c == 3) { amax = std::max(amax, v); amin = std::min(amin, v); }
            }
            gray = gray && (b.px[t].x == b.px[t].y && b.px[t].x == b.px[t].z);
            t++;
        }
    }
    b.gray = gray ? 1 : 0;
    b.calpha = (amax == amin) ? 1 : 0;
    b.pcount[0] = bx * by;
}
void flags_from_texels(InputBlock& b, int T) {
    float amin = 1e38f, amax = 0.0f; bool gray = true;
    for (int t = 0; t < T; t++) {
        amax = std::max(amax, b.px[t].w); amin = std::min(amin, b.px[t].w);
        gray = gray && (b.px[t].x == b.px[t].y && b.px[t].x == b.px[t].z);
    }
    b.gray = gray; b.calpha = amax == amin; b.pcount[0] = T;
}

inline float dist_sq(v4 a, v4 b) { v4 d = a - b; return dot4(d * d, {CW[0], CW[1], CW[2], CW[3]}); }
const v4 CWV = {0.30f * 2.25f, 0.59f * 2.25f, 0.11f * 2.25f, 1.0f};

// The partitioned block of table entry `entry` (0..1023) for P = 2..4, as pass007
// emits it (compression_pipeline.cpp passes 001-007 output).
void make_pb(const Footprint& f, const InputBlock& blk, int P, int entry, InputBlock& nb) {
    const PartInfo& pi = f.pinfo[(P - 2) * 1024 + entry];
    std::memcpy(nb.px, blk.px, sizeof(nb.px));
    nb.gray = blk.gray; nb.calpha = blk.calpha;
    nb.pidx = pi.index;
    for (int p = 0; p < 4; p++) nb.pcount[p] = pi.texel_count[p];
    for (int t = 0; t < MAX_TEXELS; t++) nb.tp[t] = pi.of_texel[t];
}

// ---------------------------------------------------------------- partition search, passes 001-007
// Returns the number of partitioned blocks written to out[].
int partition_search(const Footprint& f, const InputBlock& blk, int P, InputBlock* out, uint32_t* entries_out,
                     uint32_t* mismatch_out = nullptr, uint32_t* order_out = nullptr) {
    const int T = f.T;
    const v4* px = blk.px;
    // pass001_init_kmeans.wgsl:61-131
    v4 centers[4];
    float dist[MAX_TEXELS];
    centers[0] = px[145897 % T];
    for (int t = 0; t < T; t++) dist[t] = dist_sq(centers[0], px[t]);
    for (int p = 1; p < P; p++) {
        uint32_t mx = 0; int idx = 0;
        for (int t = 0; t < T; t++) { uint32_t b; std::memcpy(&b, &dist[t], 4); mx = std::max(mx, b); }
        for (int t = 0; t < T; t++) { uint32_t b; std::memcpy(&b, &dist[t], 4); if (b == mx) idx = t; }  // S8
        centers[p] = px[idx];
        if (p < P - 1)
            for (int t = 0; t < T; t++) dist[t] = fmn(dist[t], dist_sq(centers[p], px[t]));
    }
    uint32_t assign[MAX_TEXELS];
    for (int it = 0; it < 4; it++) {
        // pass002_assign_kmeans.wgsl:193-251
        uint32_t counts[4] = {0, 0, 0, 0};
        for (int t = 0; t < T; t++) {
            float best = 1e30f; uint32_t bp = 0;
            for (int p = 0; p < P; p++) { float d = dist_sq(px[t], centers[p]); if (d < best) { best = d; bp = p; } }
            assign[t] = bp; counts[bp]++;
        }
        bool problem = false;
        for (int p = 0; p < P; p++) if (counts[p] == 0) problem = true;
        if (problem) for (int p = 0; p < P; p++) assign[p] = p;
        // pass003_update_kmeans.wgsl:52-112
        uint32_t sums[4][4] = {{0}}, cnt[4] = {0, 0, 0, 0};
        for (int t = 0; t < T; t++) {
            uint32_t p = assign[t];
            for (int c = 0; c < 4; c++) sums[p][c] += f2u(compc(px[t], c));
            cnt[p]++;
        }
        for (int p = 0; p < P; p++) {
            v4 nc = V(0.0f);
            if (cnt[p] > 0) {
                float fc = (float)cnt[p];
                nc = {(float)sums[p][0] / fc, (float)sums[p][1] / fc, (float)sums[p][2] / fc, (float)sums[p][3] / fc};
            }
            centers[p] = nc;
        }
    }
    // pass004_count_partition_mismatch.wgsl:90-186
    uint64_t km[4] = {0, 0, 0, 0};
    for (int i = 0; i < 64; i++) km[assign[f.kmeans[i]]] |= 1ULL << i;
    const unsigned sel = f.count_selected[P - 1];
    std::vector<uint32_t> mismatch(1024, 0);
    const uint64_t* cov = f.cov[P].data();
    auto pc64 = [](uint64_t v) { return (uint32_t)__builtin_popcountll(v); };
    for (unsigned i = 0; i < sel; i++) {
        uint32_t m;
        if (P == 2) {
            uint64_t b0 = cov[2 * i], b1 = cov[2 * i + 1];
            uint32_t v1 = pc64(km[0] ^ b0) + pc64(km[1] ^ b1), v2 = pc64(km[0] ^ b1) + pc64(km[1] ^ b0);
            m = std::min(v1, v2) / 2;
        } else if (P == 3) {
            const uint64_t* b = &cov[3 * i];
            uint32_t p[3][3];
            for (int a = 0; a < 3; a++) for (int c = 0; c < 3; c++) p[a][c] = pc64(km[a] ^ b[c]);
            uint32_t v0 = std::min(p[1][1] + p[2][2], p[1][2] + p[2][1]) + p[0][0];
            uint32_t v1 = std::min(p[1][0] + p[2][2], p[1][2] + p[2][0]) + p[0][1];
            uint32_t v2 = std::min(p[1][0] + p[2][1], p[1][1] + p[2][0]) + p[0][2];
            m = std::min(v0, std::min(v1, v2)) / 2;
        } else {
            const uint64_t* b = &cov[4 * i];
            uint32_t p[4][4];
            for (int a = 0; a < 4; a++) for (int c = 0; c < 4; c++) p[a][c] = pc64(km[a] ^ b[c]);
            uint32_t mx23 = std::min(p[2][2] + p[3][3], p[2][3] + p[3][2]);
            uint32_t mx13 = std::min(p[2][1] + p[3][3], p[2][3] + p[3][1]);
            uint32_t mx12 = std::min(p[2][1] + p[3][2], p[2][2] + p[3][1]);
            uint32_t mx03 = std::min(p[2][0] + p[3][3], p[2][3] + p[3][0]);
            uint32_t mx02 = std::min(p[2][0] + p[3][2], p[2][2] + p[3][0]);
            uint32_t mx01 = std::min(p[2][1] + p[3][0], p[2][0] + p[3][1]);
            uint32_t v0 = p[0][0] + std::min(p[1][1] + mx23, std::min(p[1][2] + mx13, p[1][3] + mx12));
            uint32_t v1 = p[0][1] + std::min(p[1][0] + mx23, std::min(p[1][2] + mx03, p[1][3] + mx02));
            uint32_t v2 = p[0][2] + std::min(p[1][1] + mx03, std::min(p[1][0] + mx13, p[1][3] + mx01));
            uint32_t v3 = p[0][3] + std::min(p[1][1] + mx02, std::min(p[1][2] + mx01, p[1][0] + mx12));
            m = std::min(v0, std::min(v1, std::min(v2, v3))) / 2;
        }
        mismatch[i] = m;  // S9: block*1024 + i
    }
    // pass005_partition_ordering.wgsl:35-94 (partial bitonic network, 256 invocations)
    uint32_t score[1024], index[1024];
    for (unsigned i = 0; i < 1024; i++) { index[i] = i; score[i] = i < sel ? mismatch[i] : 0xFFFFFFFFu; }
    if (g_fixed) {  // F1: the full ascending (score, index) order
        std::vector<uint64_t> kv(1024);
        for (unsigned i = 0; i < 1024; i++) kv[i] = (uint64_t)score[i] << 32 | i;
        std::sort(kv.begin(), kv.end());
        for (unsigned i = 0; i < 1024; i++) { score[i] = (uint32_t)(kv[i] >> 32); index[i] = (uint32_t)kv[i]; }
    }
    for (unsigned k = 2; k <= 1024 && !g_fixed; k *= 2)
        for (unsigned j = k / 2; j > 0; j /= 2)
            for (unsigned l = 0; l < 256; l++) {
                unsigned partner = l ^ j;
                if (partner > l) {
                    bool asc = (l & k) == 0;
                    bool sw = (score[l] > score[partner]) || (score[l] == score[partner] && index[l] > index[partner]);
                    if (sw == asc) { std::swap(score[l], score[partner]); std::swap(index[l], index[partner]); }
                }
            }
    if (mismatch_out) for (unsigned i = 0; i < 1024; i++) mismatch_out[i] = i < sel ? mismatch[i] : 0xFFFFFFFFu;
    if (order_out) for (int i = 0; i < PART_CAND_LIMIT; i++) order_out[i] = index[i];
    // pass006_evaluate_partition_candidates.wgsl:73-296
    float err_u[PART_CAND_LIMIT], err_s[PART_CAND_LIMIT];
    float wie = T <= 20 ? 0.03f : T <= 31 ? 0.04f : T <= 41 ? 0.05f : 0.055f;
    wie = wie * wie;
    for (int cand = 0; cand < PART_CAND_LIMIT; cand++) {
        const PartInfo& pi = f.pinfo[(P - 2) * 1024 + index[cand]];
        uint32_t cnt[4] = {0, 0, 0, 0}, sums[4][4] = {{0}};
        for (int t = 0; t < T; t++) {
            uint32_t p = pi.of_texel[t]; cnt[p]++;
            for (int c = 0; c < 4; c++) sums[p][c] += f2u(compc(px[t], c));
        }
        v4 tavg[4];
        for (int p = 0; p < 4; p++) tavg[p] = V(0.0f);
        for (int p = 0; p < P; p++) {
            float c = (float)cnt[p];
            if (c > 0.0f) tavg[p] = {(float)sums[p][0] / c, (float)sums[p][1] / c, (float)sums[p][2] / c, (float)sums[p][3] / c};
        }
        // per-invocation view (S11): invocation t sees avg[q] only for q == t < P
        // (FIXED, F4: every texel sees its partition's average and direction)
        auto own = [&](int t, uint32_t p) { return g_fixed || (t < P && (int)p == t); };
        int32_t axis[4][4][4] = {{{0}}};
        for (int t = 0; t < T; t++) {
            uint32_t p = pi.of_texel[t];
            v4 a = own(t, p) ? tavg[p] : V(0.0f);
            v4 d = px[t] - a;
            int32_t di[4] = {f2i(d.x), f2i(d.y), f2i(d.z), f2i(d.w)};
            for (int ax = 0; ax < 4; ax++)
                if (compc(d, ax) > 0.0f)
                    for (int c = 0; c < 4; c++) axis[p][ax][c] = (int32_t)((uint32_t)axis[p][ax][c] + (uint32_t)di[c]);
        }
        v4 tdir[4];
        for (int p = 0; p < 4; p++) tdir[p] = V(0.0f);
        for (int p = 0; p < P; p++) {
            v4 s[4];
            for (int ax = 0; ax < 4; ax++) s[ax] = {(float)axis[p][ax][0], (float)axis[p][ax][1], (float)axis[p][ax][2], (float)axis[p][ax][3]};
            v4 best = s[0]; float mp = dot4(s[0], s[0]);
            for (int ax = 1; ax < 4; ax++) { float pr = dot4(s[ax], s[ax]); if (pr > mp) { mp = pr; best = s[ax]; } }
            tdir[p] = normalize4(best);
        }
        uint32_t usum = 0, ssum = 0;
        int32_t lmin[4], lmax[4];
        for (int p = 0; p < P; p++) { lmin[p] = 2147483647; lmax[p] = -2147483647; }
        for (int t = 0; t < T; t++) {
            uint32_t p = pi.of_texel[t];
            bool o = own(t, p);
            v4 a = o ? tavg[p] : V(0.0f), ud = o ? tdir[p] : V(0.0f);
            v4 x = px[t];
            float up = dot4(x, ud);
            v4 uproj = a + ud * dot4(x - a, ud);
            v4 udiff = x - uproj;
            float ud2 = dot4(udiff * udiff, CWV);
            v4 sd = normalize4(a);
            v4 sproj = sd * dot4(x, sd);
            v4 sdiff = x - sproj;
            float sd2 = dot4(sdiff * sdiff, CWV);
            usum += f2u(ud2); ssum += f2u(sd2);
            int32_t upi = f2i(up * 4096.0f);
            lmin[p] = std::min(lmin[p], upi); lmax[p] = std::max(lmax[p], upi);
        }
        float tu = (float)usum, ts = (float)ssum;
        for (int p = 0; p < P; p++) {
            float mn = (float)lmin[p] / 4096.0f, mx = (float)lmax[p] / 4096.0f;
            float ll = fmx(mx - mn, 1e-7f);
            float tpp = (float)pi.texel_count[p];
            float ew = tpp * wie;
            tu = tu + ew * (ll * ll);
            v4 a0 = (p == 0 || g_fixed) ? tavg[p] : V(0.0f);  // invocation 0's private avg array (F4: all)
            ts = ts + ew * dot4(a0, a0);
        }
        err_u[cand] = tu; err_s[cand] = ts;
    }
    // pass007_prepare_partitioned_blocks.wgsl:50-174
    const int req = 4;
    struct BC { uint32_t idx; float err; };
    BC bu[8], bs[8];
    for (int i = 0; i < 8; i++) { bu[i] = {0, 1e30f}; bs[i] = {0, 1e30f}; }
    for (int i = 0; i < PART_CAND_LIMIT; i++) {
        if (err_u[i] < bu[req - 1].err) {
            bu[req - 1] = {(uint32_t)i, err_u[i]};
            for (int j = req - 1; j > 0; j--) if (bu[j].err < bu[j - 1].err) std::swap(bu[j], bu[j - 1]);
        }
        if (err_s[i] < bs[req - 1].err) {
            bs[req - 1] = {(uint32_t)i, err_s[i]};
            for (int j = req - 1; j > 0; j--) if (bs[j].err < bs[j - 1].err) std::swap(bs[j], bs[j - 1]);
        }
    }
    uint32_t inter[8], fin[4] = {0, 0, 0, 0}; int emitted = 0;
    for (int i = 0; i < req; i++) { inter[2 * i] = bu[i].idx; inter[2 * i + 1] = bs[i].idx; }
    for (int i = 0; i < req * 2; i++) {
        uint32_t idx = inter[i]; bool written = false;
        for (int j = 0; j < emitted; j++) if (fin[j] == idx) { written = true; break; }
        if (!written) { fin[emitted++] = idx; if (emitted >= req) break; }
    }
    for (int i = 0; i < emitted; i++) {
        // REF-BUG-4: rank used as table index (FIXED, F2: the ordered entry)
        const uint32_t entry = g_fixed ? index[fin[i]] : fin[i];
        make_pb(f, blk, P, (int)entry, out[i]);
        if (entries_out) entries_out[i] = (P - 2) * 1024 + entry;
    }
    return emitted;
}

// ---------------------------------------------------------------- passes 01-18 for one partitioned block
struct PBWork {
    IdealEW ei;
    float dec[MAX_DMS][MAX_WEIGHTS];
    float ang[MAX_DMS][16];
    LHW lh[MAX_DMS][16];
    float lowv[MAX_DMS][13], highv[MAX_DMS][13];
    std::vector<QuantRes> qr;
    ECE ece[4];
    float cerr[4][21][4];
    uint32_t cfmt[4][21][4];
    Combo combo[21][13];
    std::vector<CCR> ccr;
    Cand cand[NUM_CAND], top[NUM_CAND];
    int ncand;  // pass12's candidates (cand[0..ncand); slots whose error is ERR_DEFAULT stay inert)
    v4 rgbs[NUM_CAND][4];
    int32_t ue0[NUM_CAND][4][4], ue1[NUM_CAND][4][4];
};

// pass01_ideal_endpoints_and_weights.wgsl:56-206
void pass01(const Footprint& f, const InputBlock& b, IdealEW& o) {
    const int T = f.T;
    const float ew = (((CW[0] + CW[1]) + CW[2]) + CW[3]) / 4.0f;
    bool is_const = true;
    v4 sum[4]; float cnt[4];
    for (int i = 0; i < 4; i++) { sum[i] = V(0.0f); cnt[i] = 0.0f; }
    for (int i = 0; i < T; i++) { uint32_t p = b.tp[i]; if (p < 4) { sum[p] = sum[p] + b.px[i]; cnt[p] = cnt[p] + 1.0f; } }
    v4 avg[4];
    for (int p = 0; p < 4; p++) { avg[p] = cnt[p] > 0.0f ? sum[p] / V(cnt[p]) : V(0.0f); o.part[p].avg = avg[p]; }
    v4 dir[4]; float mn[4], mx[4];
    for (int p = 0; p < 4; p++) { dir[p] = V(0.0f); mn[p] = 1e10f; mx[p] = -1e10f; }
    for (int i = 0; i < T; i++) {
        uint32_t p = b.tp[i];
        if (p < 4) { v4 d = b.px[i] - avg[p]; v4 pd = vmax(d, V(0.0f)); dir[p] = dir[p] + pd * pd; }
    }
    for (int p = 0; p < 4; p++) { dir[p] = normalize4(dir[p]); o.part[p].dir = dir[p]; }
    for (int i = 0; i < T; i++) {
        uint32_t p = b.tp[i];
        if (p < 4) { float pr = dot4(b.px[i] - avg[p], dir[p]); mn[p] = fmn(mn[p], pr); mx[p] = fmx(mx[p], pr); }
    }
    float p0len = 0.0f, lsq[4];
    for (int p = 0; p < 4; p++) {
        v4 d = dir[p];
        if (mn[p] >= mx[p]) { mn[p] = 0.0f; mx[p] = 1e-7f; }
        float len = mx[p] - mn[p], l2 = len * len;
        lsq[p] = l2;
        if (d.x == 0.0f && d.y == 0.0f && d.z == 0.0f && d.w == 0.0f) { o.part[p].ep0 = avg[p]; o.part[p].ep1 = avg[p]; }
        else { o.part[p].ep0 = avg[p] + d * mn[p]; o.part[p].ep1 = avg[p] + d * mx[p]; }
        if (p == 0) p0len = l2; else is_const = is_const && l2 == p0len;
    }
    for (int i = 0; i < MAX_TEXELS; i++) { o.w[i] = 0.0f; o.wes[i] = 0.0f; }
    for (int i = 0; i < T; i++) {
        uint32_t p = b.tp[i];
        if (p < 4) {
            float pr = dot4(b.px[i] - avg[p], dir[p]);
            float span = fmx(mx[p] - mn[p], 1e-6f);
            o.w[i] = clampf((pr - mn[p]) / span, 0.0f, 1.0f);
            o.wes[i] = lsq[p] * ew;
        }
    }
    o.is_const = is_const ? 1 : 0;
    v4 me = V(10.0f);
    for (int p = 0; p < 4; p++) {
        v4 e0 = o.part[p].ep0, e1 = o.part[p].ep1;
        v4 ep = (V(1.0f) - e0) / ((e1 - e0) + V(1e-9f));
        for (int c = 0; c < 4; c++) if (compc(ep, c) > 0.5f && compc(ep, c) < compc(me, c)) comp(me, c) = compc(ep, c);
    }
    o.min_cutoff = fmn(me.x, fmn(me.y, fmn(me.z, me.w)));
}

// pass02_decimated_weights.wgsl:95-273
void pass02(const Footprint& f, const DecInfo& di, const IdealEW& ei, float* out) {
    auto es = [&](uint32_t t) { return ei.wes[ei.is_const == 0 ? t : 0]; };
    if (di.T == di.W) { for (uint32_t i = 0; i < di.W; i++) out[i] = ei.w[i]; return; }
    float dw[MAX_WEIGHTS], inf[MAX_TEXELS];
    for (uint32_t w = 0; w < di.W; w++) {
        uint32_t n = di.wt_count[w];
        if (n == 0) { dw[w] = 0.0f; continue; }
        float ws = 0.0f, tc = 1e-10f;
        for (uint32_t j = 0; j < n; j++) {
            uint32_t k = di.wt_off[w] + j, t = f.w2t_idx[k];
            float c = f.w2t_c[k], cwt = c * es(t);
            ws = ws + ei.w[t] * cwt; tc = tc + cwt;
        }
        dw[w] = ws / tc;
    }
    for (uint32_t i = 0; i < di.T; i++) {
        float v = 0.0f;
        for (uint32_t j = 0; j < di.tw_count[i]; j++) { uint32_t k = di.tw_off[i] + j; v = v + dw[f.t2w_idx[k]] * f.t2w_c[k]; }
        inf[i] = v;
    }
    for (uint32_t w = 0; w < di.W; w++) {
        float e0 = 1e-10f, e1 = 0.0f;
        for (uint32_t j = 0; j < di.wt_count[w]; j++) {
            uint32_t k = di.wt_off[w] + j, t = f.w2t_idx[k];
            float c = f.w2t_c[k];
            float sc = es(t) * c;
            e0 = e0 + c * sc;
            e1 = e1 + (inf[t] - ei.w[t]) * sc;
        }
        float step = (e1 * -16.0f) / e0;
        dw[w] = dw[w] + clampf(step, -0.25f, 0.25f);
    }
    for (uint32_t w = 0; w < di.W; w++) out[w] = dw[w];
}

// pass03_compute_angular_offsets.wgsl:64-117
void pass03(const Footprint& f, const DecInfo& di, const float* dec, float* ang) {
    uint32_t smp[MAX_WEIGHTS];
    for (uint32_t i = 0; i < di.W; i++) smp[i] = f2u(rne(clampf(dec[i], 0.0f, 1.0f) * (1024.0f - 1.0f)));
    const float inv2pi = 1.0f / (2.0f * 3.14159265358979323846f);
    for (int s = 0; s < 16; s++) {
        float ax = 0.0f, ay = 0.0f;
        for (uint32_t j = 0; j < di.W; j++) { uint32_t k = smp[j] * 16 + s; ax = ax + f.cos_t[k]; ay = ay + f.sin_t[k]; }
        ang[s] = atan2_ref(ay, ax) * inv2pi;
    }
}

// pass04_lowest_and_highest_weight.wgsl:117-227
void pass04(const DecInfo& di, const float* dec, const float* ang, LHW* lh) {
    float mnw = 3.4e38f, mxw = -3.4e38f;
    for (uint32_t i = 0; i < di.W; i++) { if (dec[i] < mnw) mnw = dec[i]; if (dec[i] > mxw) mxw = dec[i]; }
    for (uint32_t sp = 0; sp < di.max_angular_steps; sp++) {
        float rcp = (float)(sp + 1), off = ang[sp];
        float minidx = rne(mnw * rcp - off), maxidx = rne(mxw * rcp - off);
        float ev = 0.0f, cl = 0.0f, ch = 0.0f;
        for (uint32_t j = 0; j < di.W; j++) {
            float sv = dec[j] * rcp - off, r = rne(sv), d = sv - r;
            ev = ev + d * d;
            cl = cl + (r == minidx ? 1.0f - (2.0f * d) : 0.0f);
            ch = ch + (r == maxidx ? 1.0f + (2.0f * d) : 0.0f);
        }
        int32_t span = f2i((maxidx - minidx) + 1.0f);
        int32_t hi = (int32_t)(di.max_quant_steps + 3);
        int32_t cs = std::min(std::max(span, 2), hi);
        float ss = 1.0f / rcp, esc = ss * ss;
        lh[sp] = {minidx, cs, ev * esc, cl * esc, ch * esc};
    }
}

// pass05_best_values_for_quant_levels.wgsl:60-174
void pass05(const DecInfo& di, const LHW* lh, const float* ang, float* lowv, float* highv) {
    struct R { float e, idx, cut; } best[36];
    for (uint32_t i = 0; i < di.max_quant_steps + 4 && i < 36; i++) best[i] = {1e37f, -1.0f, 0.0f};
    for (uint32_t i = 0; i < di.max_angular_steps; i++) {
        float fi = (float)i;
        int32_t s = lh[i].span;
        float e = lh[i].err, cl = lh[i].cl, ch = lh[i].ch;
        float ecl = e + cl, ech = e + ch, eclh = (e + cl) + ch;
        if (e < best[s].e) best[s] = {e, fi, 0.0f};
        if (ecl < best[s - 1].e) best[s - 1] = {ecl, fi, 1.0f};
        if (ech < best[s - 1].e) best[s - 1] = {ech, fi, 0.0f};
        if (eclh < best[s - 2].e) best[s - 2] = {eclh, fi, 1.0f};
    }
    for (int q = 0; q < 13; q++) { lowv[q] = 0.0f; highv[q] = 0.0f; }
    for (uint32_t q = 0; q <= di.max_quant_level; q++) {
        int qs = STEPS_FOR_QUANT[q];
        R w = best[qs];
        int32_t bsi = std::max(f2i(w.idx), 0);
        float lwi = lh[bsi].lowest + w.cut;
        float hwi = (lwi + (float)qs) - 1.0f;
        float step = 1.0f / (1.0f + (float)bsi);
        float off = ang[bsi];
        lowv[q] = (off + lwi) * step;
        highv[q] = (off + hwi) * step;
    }
}

// pass06_remap_low_and_high_values.wgsl + pass07_weights_and_error_for_bm.wgsl:129-331
void pass07(const Footprint& f, const InputBlock& b, PBWork& w, int P, uint32_t bmi) {
    const ConstTables& ct = CT();
    QuantRes& r = w.qr[bmi];
    const BlockMode& bm = f.bms[f.valid_bms[bmi].first];
    uint32_t dml = f.valid_bms[bmi].second;
    std::memset(r.qw, 0, sizeof(r.qw));
    if (bm.quant > 11) { r.error = 1e38f; r.bitcount = 0; return; }
    int bc = FREE_BITS[P - 1] - (int)bm.weight_bits;
    if (bc <= 0) { r.error = 1e38f; r.bitcount = 0; return; }
    const DecInfo& di = f.dis[bm.dm];
    const IdealEW& ei = w.ei;
    float low = w.lowv[dml][bm.quant], high = w.highv[dml][bm.quant];  // pass06 (quant <= 12)
    if (high > 1.02f * ei.min_cutoff) high = 1.0f;
    if (high <= low) { low = 0.0f; high = 1.0f; }
    const float* dec = w.dec[dml];
    float qlm1 = (float)(LEVELS[bm.quant] - 1);
    float rscale = high - low;
    float scale = 1.0f / rscale;
    float slb = low * scale;
    rscale = rscale / 64.0f;
    float qf[MAX_WEIGHTS]; uint32_t qi[MAX_WEIGHTS];
    int off = ct.q2u_off[bm.quant];
    for (uint32_t i = 0; i < di.W; i++) {
        float ix = clampf(dec[i] * scale - slb, 0.0f, 1.0f);
        float ix1 = ix * qlm1;
        uint32_t wl = f2u(ix1), wh = std::min(wl + 1, f2u(qlm1));
        uint32_t li = ct.q2u[off + wl], hi = ct.q2u[off + wh];
        bool uh = ((float)li + (float)hi) < (128.0f * ix);
        qi[i] = uh ? hi : li;
        qf[i] = (float)(uh ? hi : li) * rscale + low;
    }
    float err = 0.0f;
    for (uint32_t t = 0; t < di.T; t++) {
        float v = 0.0f;
        for (uint32_t j = 0; j < di.tw_count[t]; j++) { uint32_t k = di.tw_off[t] + j; v = v + qf[f.t2w_idx[k]] * f.t2w_c[k]; }
        float d = v - ei.w[t];
        float es = ei.wes[ei.is_const == 0 ? t : 0];
        err = err + (d * d) * es;
    }
    r.error = err; r.bitcount = bc;
    uint32_t nw = g_fixed ? di.W : (di.W / 4) * 4;  // REF-BUG-6 (FIXED, F3: every weight)
    for (uint32_t i = 0; i < nw; i++) r.qw[i] = qi[i];
}

// pass08_compute_encoding_choice_errors.wgsl:82-325
void pass08(const Footprint& f, const InputBlock& b, const IdealEW& ei, int P, ECE* out) {
    v4 sxp[4], syp[4], szp[4];
    for (int p = 0; p < 4; p++) sxp[p] = syp[p] = szp[p] = V(0.0f);
    for (int t = 0; t < f.T; t++) {
        uint32_t p = b.tp[t];
        if ((int)p < P) {
            v4 d = b.px[t] - ei.part[p].avg; d.w = 0.0f;
            if (d.x > 0.0f) sxp[p] = sxp[p] + d;
            if (d.y > 0.0f) syp[p] = syp[p] + d;
            if (d.z > 0.0f) szp[p] = szp[p] + d;
        }
    }
    v4 ua[4], ub[4], sb[4], la[4], lb[4], nb[4];
    const v4 luma = normalize4({1.0f, 1.0f, 1.0f, 0.0f});
    for (int p = 0; p < P; p++) {
        float px_ = dot4(sxp[p], sxp[p]), py_ = dot4(syp[p], syp[p]), pz_ = dot4(szp[p], szp[p]);
        v4 bv = sxp[p]; float bs = px_;
        if (py_ > bs) { bv = syp[p]; bs = py_; }
        if (pz_ > bs) { bv = szp[p]; bs = pz_; }
        v4 avg = ei.part[p].avg; avg.w = 0.0f;
        ub[p] = normalize4(bv); ua[p] = avg - ub[p] * dot4(avg, ub[p]);
        sb[p] = normalize4(avg);
        lb[p] = luma; la[p] = avg - lb[p] * dot4(avg, lb[p]);
        nb[p] = luma;
    }
    float acc[4][5] = {{0}};
    for (int t = 0; t < f.T; t++) {
        uint32_t p = b.tp[t];
        if ((int)p < P) {
            v4 rgb = b.px[t]; rgb.w = 0.0f;
            float ad = b.px[t].w - 65536.0f;
            acc[p][0] = acc[p][0] + (ad * ad) * CW[3];
            v4 du = (ua[p] + ub[p] * dot3(rgb, ub[p])) - rgb;
            acc[p][1] = acc[p][1] + dot3(du * du, CWV);
            v4 ds = sb[p] * dot3(rgb, sb[p]) - rgb;
            acc[p][2] = acc[p][2] + dot3(ds * ds, CWV);
            v4 dl = (la[p] + lb[p] * dot3(rgb, lb[p])) - rgb;
            acc[p][3] = acc[p][3] + dot3(dl * dl, CWV);
            v4 dn = nb[p] * dot3(rgb, nb[p]) - rgb;
            acc[p][4] = acc[p][4] + dot3(dn * dn, CWV);
        }
    }
    for (int p = 0; p < P; p++) {
        v4 e0 = ei.part[p].ep0, e1 = ei.part[p].ep1;
        const float lim = 0.12f * 65536.0f;
        bool co = std::fabs(e1.x - e0.x) < lim && std::fabs(e1.y - e0.y) < lim && std::fabs(e1.z - e0.z) < lim;
        out[p].can_offset = co ? 1 : 0;
        out[p].can_bc = (b.gray == 1 && b.calpha == 1) ? 0 : 1;
        out[p].rgb_scale = (acc[p][2] - acc[p][1]) * 0.7f;
        out[p].rgb_luma = (acc[p][3] - acc[p][1]) * 1.5f;
        out[p].lum = (acc[p][4] - acc[p][1]) * 3.0f;
        out[p].alpha_drop = acc[p][0] * 3.0f;
    }
}

// pass09_compute_color_error.wgsl:118-267
void pass09(const InputBlock& b, const IdealEW& ei, const ECE* ece, int P, float cerr[4][21][4], uint32_t cfmt[4][21][4]) {
    const ConstTables& ct = CT();
    float rre[4], are[4], brgb[4], ba[4], bcrgba[4], oergba[4], bcrgb[4], oergb[4];
    for (int p = 0; p < P; p++) {
        v4 e0 = ei.part[p].ep0, e1 = ei.part[p].ep1;
        float ps = (float)b.pcount[p];
        v4 e0h = vmax(e0 - V(65535.0f), V(0.0f)), e1h = vmax(e1 - V(65535.0f), V(0.0f));
        v4 e0l = vmin(e0, V(0.0f)), e1l = vmin(e1, V(0.0f));
        v4 sre = ((e0l * e0l + e1l * e1l) + e0h * e0h) + e1h * e1h;
        rre[p] = (dot3(sre, CWV) * 0.5f) * ps;
        are[p] = ((sre.w * CW[3]) * 0.5f) * ps;
        brgb[p] = ((CW[0] + CW[1]) + CW[2]) * ps;
        ba[p] = CW[3] * ps;
        bcrgba[p] = ece[p].can_bc == 1 ? 0.625f : 1.0f;
        oergba[p] = ece[p].can_offset == 1 ? 0.5f : 1.0f;
        bcrgb[p] = ece[p].can_bc == 1 ? 0.5f : 1.0f;
        oergb[p] = ece[p].can_offset == 1 ? 0.25f : 1.0f;
        for (int q = 0; q < 4; q++) {
            for (int j = 0; j < 4; j++) cerr[p][q][j] = ERR_DEFAULT;
            cfmt[p][q][3] = FMT_RGBA; cfmt[p][q][2] = FMT_RGB; cfmt[p][q][1] = FMT_RGB_SCALE; cfmt[p][q][0] = FMT_LUMINANCE;
        }
    }
    for (int i = 0; i < 17; i++) {
        int q = i + 4;
        for (int p = 0; p < P; p++) {
            const ECE& e = ece[p];
            float orgba = oergba[p], orgb = oergb[p];
            if (q >= 19) { orgba = 1.0f; orgb = 1.0f; }
            float bq = ct.bqe[i];
            float qrgb = brgb[p] * bq, qrgba = (brgb[p] + ba[p]) * bq;
            cerr[p][q][3] = (((qrgba * bcrgba[p]) * orgba) + rre[p]) + are[p]; cfmt[p][q][3] = FMT_RGBA;
            float full = (((qrgb * bcrgb[p]) * orgb) + rre[p]) + e.alpha_drop;
            float rgbsa = ((qrgba + e.rgb_scale) + rre[p]) + are[p];
            if (rgbsa < full) { cerr[p][q][2] = rgbsa; cfmt[p][q][2] = FMT_RGB_SCALE_ALPHA; }
            else { cerr[p][q][2] = full; cfmt[p][q][2] = FMT_RGB; }
            float lrgbs = ((qrgb + rre[p]) + e.alpha_drop) + e.rgb_scale;
            float la = ((qrgba + rre[p]) + are[p]) + e.lum;
            if (lrgbs < la) { cerr[p][q][1] = lrgbs; cfmt[p][q][1] = FMT_RGB_SCALE; }
            else { cerr[p][q][1] = la; cfmt[p][q][1] = FMT_LUMINANCE_ALPHA; }
            cerr[p][q][0] = ((qrgb + rre[p]) + e.alpha_drop) + e.lum; cfmt[p][q][0] = FMT_LUMINANCE;
        }
    }
}

// pass10_color_combinations_for_quant_{2,3,4}part.wgsl
void pass10(int P, const float cerr[4][21][4], const uint32_t cfmt[4][21][4], Combo combo[21][13]) {
    const int NC = P == 2 ? 7 : P == 3 ? 10 : 13;
    for (int q = 0; q < 21; q++) for (int c = 0; c < NC; c++) combo[q][c].error = ERR_DEFAULT;
    for (int q = 4; q < 21; q++) {
        auto consider = [&](int total, float e, const uint32_t* fm) {
            Combo& o = combo[q][total];
            if (e < o.error) { o.error = e; for (int k = 0; k < 4; k++) o.fmt[k] = fm[k]; }
        };
        for (int i = 0; i < 4; i++)
            for (int j = 0; j < 4; j++) {
                int lo2 = std::min(i, j), hi2 = std::max(i, j);
                if (hi2 - lo2 > 1) continue;
                if (P == 2) {
                    float e = fmn(cerr[0][q][i] + cerr[1][q][j], 1e10f);
                    uint32_t fm[4] = {cfmt[0][q][i], cfmt[1][q][j], 0, 0};
                    consider(i + j, e, fm);
                    continue;
                }
                for (int k = 0; k < 4; k++) {
                    int lo3 = std::min(k, lo2), hi3 = std::max(k, hi2);
                    if (hi3 - lo3 > 1) continue;
                    if (P == 3) {
                        float e = fmn((cerr[0][q][i] + cerr[1][q][j]) + cerr[2][q][k], 1e10f);
                        uint32_t fm[4] = {cfmt[0][q][i], cfmt[1][q][j], cfmt[2][q][k], 0};
                        consider(i + j + k, e, fm);
                        continue;
                    }
                    for (int l = 0; l < 4; l++) {
                        int lo4 = std::min(l, lo3), hi4 = std::max(l, hi3);
                        if (hi4 - lo4 > 1) continue;
                        float e = fmn(((cerr[0][q][i] + cerr[1][q][j]) + cerr[2][q][k]) + cerr[3][q][l], 1e10f);
                        uint32_t fm[4] = {cfmt[0][q][i], cfmt[1][q][j], cfmt[2][q][k], cfmt[3][q][l]};
                        consider(i + j + k + l, e, fm);
                    }
                }
            }
    }
}

// pass11_best_color_combination_for_mode_{1,2,3,4}part.wgsl
void pass11(const Footprint& f, PBWork& w, int P, uint32_t bmi) {
    const ConstTables& ct = CT();
    const QuantRes& r = w.qr[bmi];
    CCR& o = w.ccr[bmi];
    if (r.error >= ERR_DEFAULT) { o.total = ERR_DEFAULT; o.ql = o.qlm = 0; for (int k = 0; k < 4; k++) o.fmt[k] = 0; return; }
    uint32_t bits = (uint32_t)r.bitcount;
    if (P == 1) {
        uint32_t best_i = 0; float best_e = ERR_DEFAULT;
        for (uint32_t ic = 1; ic <= 4; ic++) {
            int ql = ct.qmt[ic][bits];
            if (ql < 4) continue;
            float e = w.cerr[0][ql][ic - 1];
            if (e < best_e) { best_e = e; best_i = ic; }
        }
        int fql = ct.qmt[best_i][bits];
        uint32_t fmt = FMT_LUMINANCE;
        if (fql >= 4) fmt = w.cfmt[0][fql][best_i - 1];
        o.total = best_e + r.error;
        o.ql = (uint32_t)fql; o.qlm = (uint32_t)fql;
        o.fmt[0] = fmt; o.fmt[1] = o.fmt[2] = o.fmt[3] = 0;
        return;
    }
    const int lo = P, hi = P == 2 ? 8 : 9, modb = P == 2 ? 2 : P == 3 ? 5 : 8;
    uint32_t best_i = 0; float best_e = ERR_DEFAULT;
    for (int ic = lo; ic <= hi; ic++) {
        int ql = ct.qmt[ic][bits];
        if (ql < 4) break;
        float e = w.combo[ql][ic - P].error;
        if (e < best_e) { best_e = e; best_i = ic; }
    }
    int fql = ct.qmt[best_i][bits], fqlm = ct.qmt[best_i][bits + modb];
    uint32_t fm[4] = {0, 0, 0, 0};
    if (fql >= 4) for (int k = 0; k < 4; k++) fm[k] = w.combo[fql][best_i - P].fmt[k];
    o.total = best_e + r.error;
    o.ql = (uint32_t)fql; o.qlm = (uint32_t)fqlm;
    for (int k = 0; k < 4; k++) o.fmt[k] = fm[k];
}

// ---- pass14 helpers (pass14_pack_color_endpoints.wgsl:320-1250)
struct i4 { int32_t x, y, z, w; };
inline int32_t& ic(i4& v, int c) { return (&v.x)[c]; }
inline int32_t icc(const i4& v, int c) { return (&v.x)[c]; }
inline i4 ivec(v4 v) { return {f2i(v.x), f2i(v.y), f2i(v.z), f2i(v.w)}; }
inline v4 rnev(v4 v) { return {rne(v.x), rne(v.y), rne(v.z), rne(v.w)}; }

struct Packer {
    const int32_t (*cu2u)[512];
    Packer() : cu2u(CT().cu2u) {}
    int32_t tab(uint32_t q, int32_t idx) const { return cu2u[(int)q - 4][idx]; }
    float enc_err(v4 u0, v4 u1, i4 q0, i4 q1) const {
        v4 e0 = u0 - v4{(float)q0.x, (float)q0.y, (float)q0.z, (float)q0.w};
        v4 e1 = u1 - v4{(float)q1.x, (float)q1.y, (float)q1.z, (float)q1.w};
        v4 e = e0 * e0 + e1 * e1;
        return ((e.x + e.y) + e.z) + e.w;
    }
    i4 q3int(uint32_t q, i4 v) const { return {tab(q, v.x * 2 + 1), tab(q, v.y * 2 + 1), tab(q, v.z * 2 + 1), 0}; }
    i4 q3flt(uint32_t q, i4 v, v4 vf) const {
        i4 r; for (int c = 0; c < 3; c++) { int32_t idx = icc(v, c) * 2; if (compc(vf, c) - (float)icc(v, c) >= -0.1f) idx += 1; ic(r, c) = tab(q, idx); }
        r.w = 0; return r;
    }
    uint32_t qint(uint32_t q, int32_t v) const { return (uint32_t)tab(q, v * 2 + 1); }
    uint32_t qflt(uint32_t q, int32_t v, float vf) const { int32_t idx = v * 2; if (vf - (float)v >= -0.1f) idx += 1; return (uint32_t)tab(q, idx); }
    static void bts(i4& a, i4& b) {  // bit_transfer_signed(input0=a, input1=b)
        for (int c = 0; c < 4; c++) {
            uint32_t a0 = (uint32_t)icc(a, c), b0 = (uint32_t)icc(b, c);
            int32_t nb = (int32_t)((b0 >> 1) | (a0 & 0x80));
            int32_t na = (int32_t)((a0 >> 1) & 0x3F);
            if (na & 0x20) na -= 0x40;
            ic(a, c) = na; ic(b, c) = nb;
        }
    }
    static i4 uncontract(i4 v) { return {(v.x + v.z) >> 1, (v.y + v.z) >> 1, v.z, v.w}; }
    static void delta_unpack(i4 i0, i4 i1, i4& o0, i4& o1) {
        bts(i1, i0);
        int32_t s = i1.x + i1.y + i1.z;
        i1 = {i1.x + i0.x, i1.y + i0.y, i1.z + i0.z, i1.w + i0.w};
        if (s < 0) { i0 = uncontract(i0); i1 = uncontract(i1); std::swap(i0, i1); }
        for (int c = 0; c < 4; c++) { ic(o0, c) = std::min(std::max(icc(i0, c), 0), 255); ic(o1, c) = std::min(std::max(icc(i1, c), 0), 255); }
    }
    static void rgba_unpack(i4 i0, i4 i1, i4& o0, i4& o1) {
        if ((i0.x + i0.y + i0.z) > (i1.x + i1.y + i1.z)) { i0 = uncontract(i0); i1 = uncontract(i1); std::swap(i0, i1); }
        o0 = i0; o1 = i1;
    }
    static bool out_of_range(v4 c) {
        for (int k = 0; k < 4; k++) if (compc(c, k) < 0.0f || compc(c, k) > 255.0f) return true;
        return false;
    }
    static v4 inv_bc(v4 c) { return {(c.x + c.x) - c.z, (c.y + c.y) - c.z, (c.z + c.z) - c.z, (c.w + c.w) - c.w}; }
    bool rgb_delta_common(v4 c0, v4 c1, i4& o0, i4& o1, uint32_t q, bool want_bc) const {
        i4 c0a = ivec(rnev(c0));
        for (int k = 0; k < 4; k++) ic(c0a, k) = (int32_t)((uint32_t)icc(c0a, k) << 1);
        i4 c0b = {c0a.x & 0xFF, c0a.y & 0xFF, c0a.z & 0xFF, c0a.w & 0xFF};
        i4 c0be = q3int(q, c0b);
        for (int k = 0; k < 4; k++) ic(c0b, k) = icc(c0be, k) | (icc(c0a, k) & 0x100);
        i4 c1d = ivec(rnev(c1));
        for (int k = 0; k < 4; k++) ic(c1d, k) = (int32_t)((uint32_t)icc(c1d, k) << 1);
        for (int k = 0; k < 4; k++) ic(c1d, k) = icc(c1d, k) - icc(c0b, k);
        c1d.w = 0;
        for (int k = 0; k < 4; k++) if (icc(c1d, k) > 63 || icc(c1d, k) < -64) return false;
        for (int k = 0; k < 4; k++) ic(c1d, k) = (icc(c1d, k) & 0x7F) | ((icc(c0b, k) & 0x100) >> 1);
        i4 c1de = q3int(q, c1d);
        i4 fl; for (int k = 0; k < 4; k++) ic(fl, k) = (icc(c1d, k) ^ icc(c1de, k)) & 0xC0;
        fl.w = 0;
        if (fl.x || fl.y || fl.z || fl.w) return false;
        i4 e0 = c0be, e1 = c1de;
        bts(e1, e0);
        int32_t s = e1.x + e1.y + e1.z;
        if (want_bc ? (s >= 0) : (s < 0)) return false;
        for (int k = 0; k < 4; k++) ic(e0, k) = icc(e0, k) + icc(e1, k);
        for (int k = 0; k < 4; k++) if (icc(e0, k) < 0 || icc(e0, k) > 0xFF) return false;
        o0 = c0be; o1 = c1de;
        return true;
    }
    bool try_rgb_delta_bc(v4 color0, v4 color1, i4& o0, i4& o1, uint32_t q) const {
        v4 c0 = inv_bc(color1), c1 = inv_bc(color0);
        if (out_of_range(c0) || out_of_range(c1)) return false;
        return rgb_delta_common(c0, c1, o0, o1, q, true);
    }
    bool try_rgb_delta(v4 color0, v4 color1, i4& o0, i4& o1, uint32_t q) const {
        return rgb_delta_common(color0, color1, o0, o1, q, false);
    }
    bool try_rgb_bc(v4 color0, v4 color1, i4& o0, i4& o1, uint32_t q) const {
        v4 c0 = inv_bc(color0), c1 = inv_bc(color1);
        if (out_of_range(c0) || out_of_range(c1)) return false;
        i4 c0i = q3flt(q, ivec(rnev(c0)), c0), c1i = q3flt(q, ivec(rnev(c1)), c1);
        if ((c1i.x + c1i.y + c1i.z) <= (c0i.x + c0i.y + c0i.z)) return false;
        o0 = c1i; o1 = c0i;
        return true;
    }
    void quant_rgb(v4 color0, v4 color1, i4& o0, i4& o1, uint32_t q) const {
        v4 c0 = color0, c1 = color1; i4 c0i, c1i;
        const v4 nudge = V(0.2f);
        for (;;) {
            i4 c0q = ivec(rnev(c0)); for (int k = 0; k < 4; k++) ic(c0q, k) = std::max(icc(c0q, k), 0);
            c0i = q3flt(q, c0q, c0);
            c0 = c0 - nudge;
            i4 c1q = ivec(rnev(c1)); for (int k = 0; k < 4; k++) ic(c1q, k) = std::min(icc(c1q, k), 255);
            c1i = q3flt(q, c1q, c1);
            c1 = c1 + nudge;
            if ((c0i.x + c0i.y + c0i.z) <= (c1i.x + c1i.y + c1i.z)) break;
        }
        o0 = c0i; o1 = c1i;
    }
    bool try_alpha_delta(v4 color0, v4 color1, i4& o0, i4& o1, uint32_t q) const {
        float a0 = color0.w, a1 = color1.w;
        int32_t a0a = (int32_t)((uint32_t)f2i(rne(a0)) << 1);
        int32_t a0b = a0a & 0xFF;
        int32_t a0be = (int32_t)qint(q, a0b);
        a0b = a0be | (a0a & 0x100);
        int32_t a1d = (int32_t)((uint32_t)f2i(rne(a1)) << 1);
        a1d = a1d - a0b;
        if (a1d > 63 || a1d < -64) return false;
        a1d = a1d & 0x7F;
        a1d = a1d | ((a0b & 0x100) >> 1);
        int32_t a1de = (int32_t)qint(q, a1d);
        int32_t a1du = a1de;
        if (((a1d ^ a1du) & 0xC0) != 0) return false;
        a1du = a1du & 0x7F;
        if ((a1du & 0x40) != 0) a1du = a1du - 0x80;
        a1du = a1du + a0b;
        if (a1du < 0 || a1du > 0x1FF) return false;
        o0.w = a0be; o1.w = a1de;
        return true;
    }
    bool try_rgba_delta_bc(v4 c0, v4 c1, i4& o0, i4& o1, uint32_t q) const {
        return try_rgb_delta_bc(c0, c1, o0, o1, q) && try_alpha_delta(c1, c0, o0, o1, q);
    }
    bool try_rgba_delta(v4 c0, v4 c1, i4& o0, i4& o1, uint32_t q) const {
        return try_rgb_delta(c0, c1, o0, o1, q) && try_alpha_delta(c0, c1, o0, o1, q);
    }
    bool try_rgba_bc(v4 c0, v4 c1, i4& o0, i4& o1, uint32_t q) const {
        if (try_rgb_bc(c0, c1, o0, o1, q)) {
            o0.w = (int32_t)qflt(q, f2i(rne(c1.w)), c1.w);
            o1.w = (int32_t)qflt(q, f2i(rne(c0.w)), c0.w);
            return true;
        }
        return false;
    }
    void quant_rgba(v4 c0, v4 c1, i4& o0, i4& o1, uint32_t q) const {
        quant_rgb(c0, c1, o0, o1, q);
        o0.w = (int32_t)qflt(q, f2i(rne(c0.w)), c0.w);
        o1.w = (int32_t)qflt(q, f2i(rne(c1.w)), c1.w);
    }
    void quant_rgbs(v4 color, uint32_t* out, uint32_t q) const {
        const float scale = 1.0f / 257.0f;
        float r = clampf(color.x * scale, 0.0f, 255.0f), g = clampf(color.y * scale, 0.0f, 255.0f), b = clampf(color.z * scale, 0.0f, 255.0f);
        uint32_t ri = qflt(q, f2i(rne(r)), r), gi = qflt(q, f2i(rne(g)), g), bi = qflt(q, f2i(rne(b)), b);
        float oldsum = ((color.x + color.y) + color.z) * scale;
        float newsum = (float)(ri + gi + bi);
        float sa = clampf((color.w * (oldsum + 1e-10f)) / (newsum + 1e-10f), 0.0f, 1.0f);
        int32_t si = f2i(rne(sa * 256.0f));
        si = std::min(std::max(si, 0), 255);
        out[0] = ri; out[1] = gi; out[2] = bi; out[3] = qint(q, si);
    }
    void quant_lum(v4 c0, v4 c1, uint32_t* out, uint32_t q) const {
        float l0 = ((c0.x + c0.y) + c0.z) / 3.0f, l1 = ((c1.x + c1.y) + c1.z) / 3.0f;
        if (l0 > l1) { float a = (l0 + l1) * 0.5f; l0 = a; l1 = a; }
        out[0] = qflt(q, f2i(rne(l0)), l0);
        out[1] = qflt(q, f2i(rne(l1)), l1);
    }
    bool try_la_delta(v4 c0, v4 c1, uint32_t* out, uint32_t q) const {
        float l0 = ((c0.x + c0.y) + c0.z) / 3.0f, l1 = ((c1.x + c1.y) + c1.z) / 3.0f;
        float a0 = c0.w, a1 = c1.w;
        int32_t l0a = (int32_t)((uint32_t)f2i(rne(l0)) << 1), a0a = (int32_t)((uint32_t)f2i(rne(a0)) << 1);
        int32_t l0b = l0a & 0xFF, a0b = a0a & 0xFF;
        uint32_t l0be = qint(q, l0b), a0be = qint(q, a0b);
        l0b = (int32_t)l0be | (l0a & 0x100); a0b = (int32_t)a0be | (a0a & 0x100);
        int32_t l1d = (int32_t)((uint32_t)f2i(rne(l1)) << 1), a1d = (int32_t)((uint32_t)f2i(rne(a1)) << 1);
        l1d = l1d - l0b; a1d = a1d - a0b;
        if (l1d > 63 || l1d < -64 || a1d > 63 || a1d < -64) return false;
        l1d = l1d & 0x7F; a1d = a1d & 0x7F;
        l1d = l1d | ((l0b & 0x100) >> 1); a1d = a1d | ((a0b & 0x100) >> 1);
        uint32_t l1de = qint(q, l1d), a1de = qint(q, a1d);
        int32_t l1du = (int32_t)l1de, a1du = (int32_t)a1de;
        if (((l1d ^ l1du) & 0xC0) != 0) return false;
        if (((a1d ^ a1du) & 0xC0) != 0) return false;
        l1du &= 0x7F; a1du &= 0x7F;
        if (l1du & 0x40) l1du -= 0x80;
        if (a1du & 0x40) a1du -= 0x80;
        l1du = l1du + l0b; a1du = a1du + a0b;
        if (l1du < 0 || l1du > 0x1FF || a1du < 0 || a1du > 0x1FF) return false;
        out[0] = l0be; out[1] = l1de; out[2] = a0be; out[3] = a1de;
        return true;
    }
    void quant_la(v4 c0, v4 c1, uint32_t* out, uint32_t q) const {
        float l0 = ((c0.x + c0.y) + c0.z) / 3.0f, l1 = ((c1.x + c1.y) + c1.z) / 3.0f;
        out[0] = qflt(q, f2i(rne(l0)), l0); out[1] = qflt(q, f2i(rne(l1)), l1);
        out[2] = qflt(q, f2i(rne(c0.w)), c0.w); out[3] = qflt(q, f2i(rne(c1.w)), c1.w);
    }
    // pack_color_endpoints_helper
    uint32_t pack(v4 color0, v4 color1, v4 rgbs, uint32_t fmt, uint32_t q, uint32_t* out) const {
        v4 c0 = vmin(vmax(color0, V(0.0f)), V(65535.0f)) / V(257.0f);
        v4 c1 = vmin(vmax(color1, V(0.0f)), V(65535.0f)) / V(257.0f);
        float best = ERR_DEFAULT;
        for (int i = 0; i < 8; i++) out[i] = 0;
        uint32_t bf = FMT_LUMINANCE;
        i4 o0 = {0, 0, 0, 0}, o1 = {0, 0, 0, 0}, p0 = {0, 0, 0, 0}, p1 = {0, 0, 0, 0};
        switch (fmt) {
            case FMT_RGB:
            case FMT_RGBA: {
                const bool rgba = fmt == FMT_RGBA;
                const uint32_t delta_fmt = rgba ? FMT_RGBA_DELTA : FMT_RGB_DELTA;
                if (q <= 18) {
                    if (rgba ? try_rgba_delta_bc(c0, c1, o0, o1, q) : try_rgb_delta_bc(c0, c1, o0, o1, q)) {
                        i4 u0, u1; delta_unpack(o0, o1, u0, u1);
                        bf = delta_fmt; best = enc_err(c0, c1, u0, u1);
                    }
                    if (rgba ? try_rgba_delta(c0, c1, p0, p1, q) : try_rgb_delta(c0, c1, p0, p1, q)) {
                        i4 u0, u1; delta_unpack(p0, p1, u0, u1);
                        float e = enc_err(c0, c1, u0, u1);
                        if (e < best) { best = e; bf = delta_fmt; o0 = p0; o1 = p1; }
                    }
                }
                if (q < 20) {
                    if (rgba ? try_rgba_bc(c0, c1, p0, p1, q) : try_rgb_bc(c0, c1, p0, p1, q)) {
                        i4 u0, u1; rgba_unpack(p0, p1, u0, u1);
                        float e = enc_err(c0, c1, u0, u1);
                        if (e < best) { best = e; bf = fmt; o0 = p0; o1 = p1; }
                    }
                }
                {
                    if (rgba) quant_rgba(c0, c1, p0, p1, q); else quant_rgb(c0, c1, p0, p1, q);
                    i4 u0, u1; rgba_unpack(p0, p1, u0, u1);
                    float e = enc_err(c0, c1, u0, u1);
                    if (e < best) { best = e; bf = fmt; o0 = p0; o1 = p1; }
                }
                out[0] = (uint32_t)o0.x; out[1] = (uint32_t)o1.x; out[2] = (uint32_t)o0.y;
                out[3] = (uint32_t)o1.y; out[4] = (uint32_t)o0.z; out[5] = (uint32_t)o1.z;
                if (rgba) { out[6] = (uint32_t)o0.w; out[7] = (uint32_t)o1.w; }
                break;
            }
            case FMT_RGB_SCALE: quant_rgbs(rgbs, out, q); bf = FMT_RGB_SCALE; break;
            case FMT_RGB_SCALE_ALPHA:
                out[4] = qflt(q, f2i(rne(c0.w)), c0.w); out[5] = qflt(q, f2i(rne(c1.w)), c1.w);
                quant_rgbs(rgbs, out, q); bf = FMT_RGB_SCALE_ALPHA; break;
            case FMT_LUMINANCE: quant_lum(c0, c1, out, q); bf = FMT_LUMINANCE; break;
            case FMT_LUMINANCE_ALPHA:
                if (q <= 18 && try_la_delta(c0, c1, out, q)) { bf = FMT_LUMINANCE_ALPHA_DELTA; break; }
                quant_la(c0, c1, out, q); bf = FMT_LUMINANCE_ALPHA; break;
            default: bf = FMT_LUMINANCE; quant_lum(c0, c1, out, q); break;
        }
        return bf;
    }
};

// pass13_recompute_ideal_endpoints.wgsl:142-392
void pass13(const Footprint& f, const InputBlock& b, int P, Cand& c, v4* rgbs) {
    const DecInfo& di = f.dis[f.bms[c.bm].dm];
    float dw[MAX_WEIGHTS], uw[MAX_TEXELS];
    for (uint32_t i = 0; i < di.W; i++) dw[i] = (float)c.qw[i] / 64.0f;
    for (uint32_t t = 0; t < di.T; t++) {
        if (di.T == di.W) uw[t] = dw[t];
        else {
            float v = 0.0f;
            for (uint32_t j = 0; j < di.tw_count[t]; j++) { uint32_t k = di.tw_off[t] + j; v = v + dw[f.t2w_idx[k]] * f.t2w_c[k]; }
            uw[t] = v;
        }
    }
    float wmin[4], wmax[4], ls[4], ms[4], rs[4], smin[4], smax[4];
    v4 cx[4], cy[4], sdir[4]; float sv0[4], sv1[4];
    for (int p = 0; p < P; p++) {
        wmin[p] = 1.0f; wmax[p] = 0.0f; ls[p] = ms[p] = rs[p] = 0.0f; smin[p] = 1e10f; smax[p] = 0.0f;
        cx[p] = cy[p] = V(0.0f); sv0[p] = sv1[p] = 0.0f;
        float ps = (float)b.pcount[p];
        v4 rsum = (c.part[p].avg * ps) * CWV;
        v4 rws = vmax(CWV * ps, V(1e-17f));
        v4 q = rsum / rws; q.w = 0.0f;
        sdir[p] = normalize4(q);
    }
    const float lsw = (CW[0] + CW[1]) + CW[2];
    for (uint32_t t = 0; t < di.T; t++) {
        uint32_t p = b.tp[t];
        v4 rgba = b.px[t]; float w = uw[t];
        if (w < wmin[p]) wmin[p] = w;
        if (w > wmax[p]) wmax[p] = w;
        float sc = dot3(rgba, sdir[p]);
        if (sc < smin[p]) smin[p] = sc;
        if (sc > smax[p]) smax[p] = sc;
        float om = 1.0f - w;
        ls[p] = ls[p] + om * om; ms[p] = ms[p] + om * w; rs[p] = rs[p] + w * w;
        v4 cyc = rgba * w;
        cy[p] = cy[p] + cyc;
        cx[p] = cx[p] + (rgba - cyc);
        sv0[p] = sv0[p] + (om * sc) * lsw;
        sv1[p] = sv1[p] + (w * sc) * lsw;
    }
    for (int p = 0; p < P; p++) {
        v4 colx = cx[p] * CWV, coly = cy[p] * CWV;
        v4 lv = V(ls[p]) * CWV, mv = V(ms[p]) * CWV, rv = V(rs[p]) * CWV;
        float lx = ls[p] * lsw, my = ms[p] * lsw, rz = rs[p] * lsw;
        float scalediv = clampf(smin[p] / fmx(smax[p], 1e-10f), 0.0f, 1.0f);
        v4 sds = sdir[p] * smax[p];
        rgbs[p] = {sds.x, sds.y, sds.z, scalediv};
        PartEW& pt = c.part[p];
        if (wmin[p] >= wmax[p] * 0.999f) {
            float ps = (float)b.pcount[p];
            v4 rws = vmax(CWV * ps, V(1e-17f));
            v4 ac = (colx + coly) / rws;
            for (int k = 0; k < 4; k++) if (compc(ac, k) == compc(ac, k)) { comp(pt.ep0, k) = compc(ac, k); comp(pt.ep1, k) = compc(ac, k); }
            rgbs[p] = {sds.x, sds.y, sds.z, 1.0f};
        } else {
            v4 det = (lv * rv) - (mv * mv);
            v4 rdet = V(1.0f) / det;
            float lsdet = (lx * rz) - (my * my), lsrdet = 1.0f / lsdet;
            v4 mss = ((lv * lv) + V(2.0f) * (mv * mv)) + (rv * rv);
            float lsmss = ((lx * lx) + 2.0f * (my * my)) + (rz * rz);
            v4 e0 = ((rv * colx) - (mv * coly)) * rdet;
            v4 e1 = ((lv * coly) - (mv * colx)) * rdet;
            for (int k = 0; k < 4; k++) {
                bool dm = std::fabs(compc(det, k)) > (compc(mss, k) * 1e-4f);
                bool nn = (compc(e0, k) == compc(e0, k)) && (compc(e1, k) == compc(e1, k));
                if (dm && nn) { comp(pt.ep0, k) = compc(e0, k); comp(pt.ep1, k) = compc(e1, k); }
            }
            float se0 = ((rz * sv0[p]) - (my * sv1[p])) * lsrdet;
            float se1 = ((lx * sv1[p]) - (my * sv0[p])) * lsrdet;
            if ((std::fabs(lsdet) > (lsmss * 1e-4f)) && se0 == se0 && se1 == se1 && se0 < se1) {
                float sd2 = se0 / se1; v4 sdsm = sdir[p] * se1;
                rgbs[p] = {sdsm.x, sdsm.y, sdsm.z, sd2};
            }
        }
    }
}

// pass14_pack_color_endpoints.wgsl:1252-1304
void pass14(int P, Cand& c, const v4* rgbs) {
    static const Packer pk;
    bool all_same = c.ql != c.qlm;
    uint32_t fn[4] = {0, 0, 0, 0}, vn[32] = {0};
    for (int p = 0; p < P; p++) {
        uint32_t v[8];
        uint32_t fm = pk.pack(c.part[p].ep0, c.part[p].ep1, rgbs[p], c.fmt[p], c.ql, v);
        fn[p] = fm;
        for (int i = 0; i < 8; i++) vn[p * 8 + i] = v[i];
        if (p > 0) all_same = all_same && (fm == fn[0]);
    }
    bool matched = false;
    if (P >= 2 && all_same) {
        uint32_t fmod[4] = {0, 0, 0, 0}, vmod[32] = {0};
        bool same_mod = true;
        for (int p = 0; p < P; p++) {
            uint32_t v[8];
            uint32_t fm = pk.pack(c.part[p].ep0, c.part[p].ep1, rgbs[p], c.fmt[p], c.qlm, v);
            fmod[p] = fm;
            for (int i = 0; i < 8; i++) vmod[p * 8 + i] = v[i];
            if (p > 0 && fm != fmod[0]) { same_mod = false; break; }
        }
        if (same_mod) { matched = true; std::memcpy(fn, fmod, sizeof(fn)); std::memcpy(vn, vmod, sizeof(vn)); }
    }
    c.matched = matched ? 1 : 0;
    c.final_q = matched ? c.qlm : c.ql;
    std::memcpy(c.ffmt, fn, sizeof(fn));
    std::memcpy(c.packed, vn, sizeof(vn));
}

// pass15_unpack_color_endpoints.wgsl:292-391
void pass15(int P, const Cand& c, int32_t e0[4][4], int32_t e1[4][4]) {
    for (int p = 0; p < P; p++) {
        const uint32_t* v = &c.packed[p * 8];
        i4 o0, o1;
        auto I = [&](int k) { return (int32_t)v[k]; };
        switch (c.ffmt[p]) {
            case FMT_LUMINANCE: default: o0 = {I(0), I(0), I(0), 255}; o1 = {I(1), I(1), I(1), 255}; break;
            case FMT_LUMINANCE_DELTA: {
                int32_t l0 = (I(0) >> 2) | (I(1) & 0xC0), l1 = std::min(l0 + (I(1) & 0x3F), 255);
                o0 = {l0, l0, l0, 255}; o1 = {l1, l1, l1, 255}; break;
            }
            case FMT_LUMINANCE_ALPHA: o0 = {I(0), I(0), I(0), I(2)}; o1 = {I(1), I(1), I(1), I(3)}; break;
            case FMT_LUMINANCE_ALPHA_DELTA: {
                int32_t l0 = I(0), l1 = I(1), a0 = I(2), a1 = I(3);
                l0 = l0 | ((l1 & 0x80) << 1); a0 = a0 | ((a1 & 0x80) << 1);
                l1 &= 0x7F; a1 &= 0x7F;
                if (l1 & 0x40) l1 -= 0x80;
                if (a1 & 0x40) a1 -= 0x80;
                l0 >>= 1; l1 >>= 1; a0 >>= 1; a1 >>= 1;
                l1 = l0 + l1; a1 = a0 + a1;
                l1 = std::min(std::max(l1, 0), 255); a1 = std::min(std::max(a1, 0), 255);
                o0 = {l0, l0, l0, a0}; o1 = {l1, l1, l1, a1}; break;
            }
            case FMT_RGB_SCALE: {
                i4 in0 = {I(0), I(1), I(2), 255}; int32_t s = I(3);
                o1 = in0;
                o0 = {(in0.x * s) >> 8, (in0.y * s) >> 8, (in0.z * s) >> 8, 255}; break;
            }
            case FMT_RGB_SCALE_ALPHA: {
                i4 in0 = {I(0), I(1), I(2), I(4)}; int32_t s = I(3);
                o1 = {in0.x, in0.y, in0.z, I(5)};
                o0 = {(in0.x * s) >> 8, (in0.y * s) >> 8, (in0.z * s) >> 8, I(4)}; break;
            }
            case FMT_RGB: Packer::rgba_unpack({I(0), I(2), I(4), 0}, {I(1), I(3), I(5), 0}, o0, o1); o0.w = 255; o1.w = 255; break;
            case FMT_RGB_DELTA: Packer::delta_unpack({I(0), I(2), I(4), 0}, {I(1), I(3), I(5), 0}, o0, o1); o0.w = 255; o1.w = 255; break;
            case FMT_RGBA: Packer::rgba_unpack({I(0), I(2), I(4), I(6)}, {I(1), I(3), I(5), I(7)}, o0, o1); break;
            case FMT_RGBA_DELTA: Packer::delta_unpack({I(0), I(2), I(4), I(6)}, {I(1), I(3), I(5), I(7)}, o0, o1); break;
        }
        for (int k = 0; k < 4; k++) { e0[p][k] = icc(o0, k) * 257; e1[p][k] = icc(o1, k) * 257; }
    }
}

// pass16_realign_weights.wgsl:108-367
void pass16(const Footprint& f, const InputBlock& b, int P, Cand& c, const int32_t e0[4][4], const int32_t e1[4][4]) {
    const ConstTables& ct = CT();
    const BlockMode& bm = f.bms[c.bm];
    const DecInfo& di = f.dis[bm.dm];
    v4 base[4], offs[4];
    for (int p = 0; p < P; p++) {
        base[p] = {(float)e0[p][0], (float)e0[p][1], (float)e0[p][2], (float)e0[p][3]};
        v4 d = {(float)(e1[p][0] - e0[p][0]), (float)(e1[p][1] - e0[p][1]), (float)(e1[p][2] - e0[p][2]), (float)(e1[p][3] - e0[p][3])};
        offs[p] = d * (1.0f / 64.0f);
    }
    float uqf[MAX_WEIGHTS];
    for (uint32_t i = 0; i < di.W; i++) uqf[i] = (float)c.qw[i];
    if (di.W == di.T) {
        uint32_t nq[MAX_WEIGHTS];
        for (uint32_t t = 0; t < di.T; t++) {
            int32_t uqw = (int32_t)c.qw[t];
            uint32_t pn = (uint32_t)ct.prev_next[bm.quant][uqw];
            int32_t dn = (int32_t)(pn & 0xFF), up = (int32_t)((pn >> 8) & 0xFF);
            float wb = (float)uqw, wdd = (float)(dn - uqw), wud = (float)(up - uqw);
            uint32_t p = b.tp[t];
            v4 col = base[p] + offs[p] * wb;
            v4 cd = col - b.px[t];
            v4 cdd = cd + offs[p] * wdd, cdu = cd + offs[p] * wud;
            float eb = dot4(cd * cd, CWV), ed = dot4(cdd * cdd, CWV), eu = dot4(cdu * cdu, CWV);
            nq[t] = c.qw[t];
            if ((eu < eb) && (eu < ed) && (uqw < 64)) nq[t] = (uint32_t)up;
            else if ((ed < eb) && (uqw > 0)) nq[t] = (uint32_t)dn;
        }
        for (uint32_t t = 0; t < di.T; t++) c.qw[t] = nq[t];
    } else {
        for (uint32_t we = 0; we < di.W; we++) {
            int32_t uqw = (int32_t)c.qw[we];
            uint32_t pn = (uint32_t)ct.prev_next[bm.quant][uqw];
            float dn = (float)(pn & 0xFF), up = (float)((pn >> 8) & 0xFF), ub = (float)uqw;
            float ddn = dn - ub, dup = up - ub;
            v4 ebv = V(0.0f), edv = V(0.0f), euv = V(0.0f);
            for (uint32_t te = 0; te < di.wt_count[we]; te++) {
                uint32_t t = f.w2t_idx[di.wt_off[we] + te];
                float wbase = 0.0f;
                uint32_t to = di.tw_off[t];
                for (uint32_t j = 0; j < di.tw_count[t]; j++) wbase = wbase + uqf[f.t2w_idx[to + j]] * f.t2w_c[to + j];
                float twb = 0.0f;
                for (uint32_t k = 0; k < di.tw_count[t]; k++) if (f.t2w_idx[to + k] == we) { twb = f.t2w_c[to + k]; break; }
                float wdd = ddn * twb, wud = dup * twb;
                uint32_t p = b.tp[t];
                v4 col = base[p] + offs[p] * wbase;
                v4 cd = col - b.px[t];
                v4 cdd = cd + offs[p] * wdd, cdu = cd + offs[p] * wud;
                ebv = ebv + cd * cd; edv = edv + cdd * cdd; euv = euv + cdu * cdu;
            }
            float eb = dot4(ebv, CWV), ed = dot4(edv, CWV), eu = dot4(euv, CWV);
            if ((eu < eb) && (eu < ed) && (uqw < 64)) { c.qw[we] = (uint32_t)up; uqf[we] = up; }
            else if ((ed < eb) && (uqw > 0)) { c.qw[we] = (uint32_t)dn; uqf[we] = dn; }
        }
    }
}

// pass17_compute_final_error.wgsl:110-230
void pass17(const Footprint& f, const InputBlock& b, int P, Cand& c, Cand& top, const int32_t e0[4][4], const int32_t e1[4][4]) {
    const DecInfo& di = f.dis[f.bms[c.bm].dm];
    float dw[MAX_WEIGHTS], uw[MAX_TEXELS];
    for (uint32_t i = 0; i < di.W; i++) dw[i] = (float)c.qw[i] / 64.0f;
    for (uint32_t t = 0; t < di.T; t++) {
        if (di.T == di.W) uw[t] = dw[t];
        else {
            float v = 0.0f;
            for (uint32_t j = 0; j < di.tw_count[t]; j++) { uint32_t k = di.tw_off[t] + j; v = v + dw[f.t2w_idx[k]] * f.t2w_c[k]; }
            uw[t] = v;
        }
    }
    float total = 0.0f;
    for (uint32_t t = 0; t < di.T; t++) {
        uint32_t p = b.tp[t];
        if ((int)p < P) {
            int32_t w1 = f2i(rne(uw[t] * 64.0f)), w0 = 64 - w1;
            v4 diff;
            for (int k = 0; k < 4; k++) {
                int32_t col = ((e0[p][k] * w0) + (e1[p][k] * w1) + 32) >> 6;
                comp(diff, k) = compc(b.px[t], k) - (float)col;
            }
            diff = vmin({std::fabs(diff.x), std::fabs(diff.y), std::fabs(diff.z), std::fabs(diff.w)}, V(1e15f));
            float e = dot4(diff * diff, CWV);
            total = total + fmn(e, ERR_DEFAULT);
        }
    }
    c.total_error = total;
    if (total < top.total_error) top = c;
}

// mask (optional): the block modes to evaluate, one bit per valid block mode (4 words);
// the others get pass07's "unusable" error and never become candidates.  topn: how many
// of the 8 best trials are refined; iters: refinement iterations (the reference: 8, 6).
Sym process_pb(const Footprint& f, const InputBlock& b, int P, PBWork& w, const uint64_t* mask = nullptr,
               int topn = NUM_CAND, int iters = 6) {
    pass01(f, b, w.ei);
    const int ndm = (int)f.valid_dms.size(), nbm = (int)f.valid_bms.size();
    for (int m = 0; m < ndm; m++) {
        const DecInfo& di = f.dis[f.valid_dms[m]];
        pass02(f, di, w.ei, w.dec[m]);
        pass03(f, di, w.dec[m], w.ang[m]);
        pass04(di, w.dec[m], w.ang[m], w.lh[m]);
        pass05(di, w.lh[m], w.ang[m], w.lowv[m], w.highv[m]);
    }
    w.qr.resize(nbm); w.ccr.resize(nbm);
    for (int i = 0; i < nbm; i++) {
        if (mask && !((mask[i >> 6] >> (i & 63)) & 1)) {
            QuantRes& r = w.qr[i];
            std::memset(r.qw, 0, sizeof(r.qw));
            r.error = 1e38f; r.bitcount = 0;
            continue;
        }
        pass07(f, b, w, P, i);
    }
    pass08(f, b, w.ei, P, w.ece);
    pass09(b, w.ei, w.ece, P, w.cerr, w.cfmt);
    if (P > 1) pass10(P, w.cerr, w.cfmt, w.combo);
    for (int i = 0; i < nbm; i++) pass11(f, w, P, i);
    // pass12_find_top_N_candidates.wgsl:88-190
    struct SI { float e; int i; } tc[NUM_CAND];
    for (int i = 0; i < NUM_CAND; i++) tc[i] = {ERR_DEFAULT, 0};
    for (int i = 0; i < nbm; i++) {
        float e = w.ccr[i].total;
        if (e < tc[NUM_CAND - 1].e) {
            tc[NUM_CAND - 1] = {e, i};
            for (int j = NUM_CAND - 1; j > 0; j--) if (tc[j].e < tc[j - 1].e) std::swap(tc[j], tc[j - 1]);
        }
    }
    int ncand = 0;
    for (int k = 0; k < NUM_CAND; k++) {
        w.top[k].total_error = ERR_DEFAULT;
        if (!(tc[k].e < ERR_DEFAULT)) continue;  // S10: slot stays inert
        Cand& c = w.cand[k];
        std::memset(&c, 0, sizeof(c));
        const CCR& cr = w.ccr[tc[k].i];
        c.bm = f.valid_bms[tc[k].i].first; c.bm_lookup = tc[k].i;
        c.total_error = cr.total; c.ql = cr.ql; c.qlm = cr.qlm;
        for (int q = 0; q < 4; q++) c.fmt[q] = cr.fmt[q];
        for (int q = 0; q < 4; q++) c.part[q] = w.ei.part[q];
        for (int i = 0; i < MAX_WEIGHTS; i++) c.qw[i] = w.qr[tc[k].i].qw[i];
        ncand = k + 1;
    }
    w.ncand = ncand;
    // compression_pipeline.cpp:473-484 refinement loop, one candidate at a time
    for (int k = 0; k < std::min(ncand, topn); k++) {
        Cand& c = w.cand[k];
        for (int a = 0; a < iters; a++) {
            pass13(f, b, P, c, w.rgbs[k]);
            pass14(P, c, w.rgbs[k]);
            pass15(P, c, w.ue0[k], w.ue1[k]);
            if (a == 0) pass17(f, b, P, c, w.top[k], w.ue0[k], w.ue1[k]);
            pass16(f, b, P, c, w.ue0[k], w.ue1[k]);
            pass17(f, b, P, c, w.top[k], w.ue0[k], w.ue1[k]);
        }
    }
    // pass18_pick_best_candidate.wgsl:79-141
    float be = ERR_DEFAULT; int bi = -1;
    for (int k = 0; k < NUM_CAND; k++) if (w.top[k].total_error < be) { be = w.top[k].total_error; bi = k; }
    Sym s; std::memset(&s, 0, sizeof(s));
    s.err = be;
    if (bi >= 0) {
        const Cand& c = w.top[bi];
        s.mode_index = f.bms[c.bm].mode_index; s.pc = P; s.pidx = b.pidx;
        s.quant = c.final_q; s.matched = c.matched;
        for (int q = 0; q < 4; q++) s.fmt[q] = c.ffmt[q];
        for (int i = 0; i < 32; i++) s.packed[i] = c.packed[i];
        for (int i = 0; i < MAX_WEIGHTS; i++) s.qw[i] = c.qw[i];
    }
    return s;
}

// compression_pipeline.cpp:359-519, for one block: P = 1..4, best candidate, best P
// (iters: refinement iterations, 6 in the reference).
Sym encode_block(const Footprint& f, const InputBlock& blk, PBWork& w, int iters = 6) {
    Sym best; std::memset(&best, 0, sizeof(best)); best.err = 1e30f;  // ERROR_CALC_DEFAULT (astc.h:77)
    InputBlock pbs[4];
    for (int P = 1; P <= 4; P++) {
        int n;
        if (P == 1) { pbs[0] = blk; n = 1; }
        else n = partition_search(f, blk, P, pbs, nullptr);
        const Sym* bc = nullptr; Sym cur[4];
        for (int i = 0; i < n; i++) {
            cur[i] = process_pb(f, pbs[i], P, w, nullptr, NUM_CAND, iters);
            if (bc == nullptr || cur[i].err < bc->err) bc = &cur[i];
        }
        if (bc && bc->err < best.err) best = *bc;
    }
    return best;
}

// The search restricted to given candidates (no counterpart in the reference; the
// checker of the learned proposal search): P = 1 unless flags bit 0 is set, then the
// proposed partitionings in the given order, each with its partition count's block-mode
// mask, `topn` trials refined `iters` times; the first minimum over that order wins, and
// only errors below 1e30 count (`found` = 0: none, the block goes to the full search).
Sym encode_block_restricted(const Footprint& f, const InputBlock& blk, PBWork& w, const uint16_t* picks,
                            const uint64_t* masks, int topn, int iters, bool& found) {
    Sym best; std::memset(&best, 0, sizeof(best)); best.err = 1e30f;
    found = false;
    const int n = picks[0], flags = picks[1];
    for (int s = (flags & 1) ? 1 : 0; s <= n; s++) {
        int P = 1;
        InputBlock pb;
        if (s == 0) pb = blk;
        else {
            const int v = picks[2 + s - 1];
            P = 2 + (v >> 10);
            make_pb(f, blk, P, v & 1023, pb);
        }
        const Sym cur = process_pb(f, pb, P, w, masks + (P - 1) * 4, topn, iters);
        if (cur.err < best.err) { best = cur; found = true; }
    }
    return best;
}

// ---------------------------------------------------------------- physical encoding
// code/physical_compression.cpp:641-666 write_bits
void write_bits(unsigned value, unsigned bitcount, unsigned bitoffset, uint8_t* ptr) {
    unsigned mask = (1u << bitcount) - 1;
    value &= mask;
    ptr += bitoffset >> 3;
    bitoffset &= 7;
    value <<= bitoffset; mask <<= bitoffset; mask = ~mask;
    ptr[0] &= mask; ptr[0] |= value;
    ptr[1] &= mask >> 8; ptr[1] |= value >> 8;
}
// code/physical_compression.cpp:672-826 encode_ise
void encode_ise(int q, unsigned n, const uint8_t* in, uint8_t* out, unsigned off) {
    const ConstTables& ct = CT();
    int bits, trits, quints; btq(q, bits, trits, quints);
    unsigned mask = (1u << bits) - 1;
    if (trits) {
        unsigned i = 0, full = n / 5;
        static const uint8_t tb[5] = {2, 2, 1, 2, 1}, ts[5] = {0, 2, 4, 5, 7};
        for (unsigned j = 0; j < full; j++) {
            uint8_t T = ct.trits[in[i + 4] >> bits][in[i + 3] >> bits][in[i + 2] >> bits][in[i + 1] >> bits][in[i] >> bits];
            for (int e = 0; e < 5; e++) {
                uint8_t pack = (uint8_t)((in[i++] & mask) | (((T >> ts[e]) & ((1 << tb[e]) - 1)) << bits));
                write_bits(pack, bits + tb[e], off, out); off += bits + tb[e];
            }
        }
        if (i != n) {
            unsigned i3 = i + 3 >= n ? 0 : in[i + 3] >> bits, i2 = i + 2 >= n ? 0 : in[i + 2] >> bits;
            unsigned i1 = i + 1 >= n ? 0 : in[i + 1] >> bits, i0 = in[i] >> bits;
            uint8_t T = ct.trits[0][i3][i2][i1][i0];
            for (unsigned j = 0; i < n; i++, j++) {
                uint8_t pack = (uint8_t)((in[i] & mask) | (((T >> ts[j]) & ((1 << tb[j]) - 1)) << bits));
                write_bits(pack, bits + tb[j], off, out); off += bits + tb[j];
            }
        }
    } else if (quints) {
        unsigned i = 0, full = n / 3;
        static const uint8_t qb[3] = {3, 2, 2}, qs[3] = {0, 3, 5};
        for (unsigned j = 0; j < full; j++) {
            uint8_t Q = ct.quints[in[i + 2] >> bits][in[i + 1] >> bits][in[i] >> bits];
            for (int e = 0; e < 3; e++) {
                uint8_t pack = (uint8_t)((in[i++] & mask) | (((Q >> qs[e]) & ((1 << qb[e]) - 1)) << bits));
                write_bits(pack, bits + qb[e], off, out); off += bits + qb[e];
            }
        }
        if (i != n) {
            unsigned i1 = i + 1 >= n ? 0 : in[i + 1] >> bits, i0 = in[i] >> bits;
            uint8_t Q = ct.quints[0][i1][i0];
            for (unsigned j = 0; i < n; i++, j++) {
                uint8_t pack = (uint8_t)((in[i] & mask) | (((Q >> qs[j]) & ((1 << qb[j]) - 1)) << bits));
                write_bits(pack, bits + qb[j], off, out); off += bits + qb[j];
            }
        }
    } else {
        for (unsigned i = 0; i < n; i++) { write_bits(in[i], bits, off, out); off += bits; }
    }
}
int bitrev8(int p) {
    p = ((p & 0x0F) << 4) | ((p >> 4) & 0x0F);
    p = ((p & 0x33) << 2) | ((p >> 2) & 0x33);
    p = ((p & 0x55) << 1) | ((p >> 1) & 0x55);
    return p;
}
// code/physical_compression.cpp:843-1003 symbolic_to_physical (single plane)
void sym_to_phys(const Footprint& f, const uint32_t* s, uint8_t* pcb) {
    const ConstTables& ct = CT();
    if (s[7]) {  // extension: LDR void-extent block (mode bits 0x1FC, bits 10-11 set), every
                 // extent coordinate all ones (no extent), then RGBA as 16-bit UNORM (colour x 257)
        const uint8_t head[8] = {0xFC, 0xFD, 0xFF, 0xFF, 0xFF, 0xFF, 0xFF, 0xFF};
        for (int i = 0; i < 8; i++) pcb[i] = head[i];
        for (int c = 0; c < 4; c++) { pcb[8 + 2 * c] = (uint8_t)s[12 + c]; pcb[9 + 2 * c] = (uint8_t)s[12 + c]; }
        return;
    }
    unsigned pc = s[2];
    uint8_t wbuf[16] = {0};
    const BlockMode& bm = f.bms[f.bm_index[s[1]]];
    const DecInfo& di = f.dis[bm.dm];
    int W = di.W, q = bm.quant;
    float levels = (float)LEVELS[q];
    int real_w = bm.dual ? 2 * W : W;
    int bits_w = ise_bitcount(real_w, q);
    uint8_t wts[64];
    for (int i = 0; i < W; i++) {
        float uqw = (float)s[44 + i];
        float qw = (uqw / 64.0f) * (levels - 1.0f);
        int qwi = (int)(qw + 0.5f);
        if (bm.dual) {
            wts[2 * i] = ct.wscr[q][qwi];
            float u2 = (float)s[44 + i + 32];
            float q2 = (u2 / 64.0f) * (levels - 1.0f);
            wts[2 * i + 1] = ct.wscr[q][(int)(q2 + 0.5f)];
        } else wts[i] = ct.wscr[q][qwi];
    }
    encode_ise(q, real_w, wts, wbuf, 0);
    for (int i = 0; i < 16; i++) pcb[i] = (uint8_t)bitrev8(wbuf[15 - i]);
    write_bits(s[1] & 0xFFFF, 11, 0, pcb);
    write_bits(pc - 1, 2, 11, pcb);
    if (pc > 1) {
        write_bits(s[3], 6, 13, pcb);
        write_bits(s[3] >> 6, 4, 19, pcb);
        if (s[4]) write_bits(s[8] << 2, 6, 23, pcb);
        else {
            int low = 4;
            for (unsigned i = 0; i < pc; i++) low = std::min((int)(s[8 + i] >> 2), low);
            if (low == 3) low = 2;
            int et = low + 1, bp = 2;
            for (unsigned i = 0; i < pc; i++) { et |= ((int)(s[8 + i] >> 2) - low) << bp; bp++; }
            for (unsigned i = 0; i < pc; i++) { et |= (int)(s[8 + i] & 3) << bp; bp += 2; }
            int hs = 3 * pc - 4;
            write_bits(et & 0x3F, 6, 23, pcb);
            write_bits(et >> 6, hs, 128 - bits_w - hs, pcb);
        }
    } else {
        write_bits((uint8_t)s[8], 4, 13, pcb);
    }
    // extension: the plane-2 component of a dual-plane block (the reference leaves it
    // out, physical_compression.cpp:967-971); single partition only
    if (bm.dual && pc == 1) write_bits(s[6] - 1, 2, 128 - bits_w - 2, pcb);
    uint8_t vals[32]; int nv = 0;
    const uint8_t* tab = ct.cscr[s[5] - 4];
    for (unsigned i = 0; i < pc; i++) {
        int n = 2 * (s[8 + i] >> 2) + 2;
        for (int j = 0; j < n; j++) vals[nv + j] = tab[s[12 + i * 8 + j]];
        nv += n;
    }
    encode_ise((int)s[5], nv, vals, pcb, pc == 1 ? 17 : 29);
}

void sym_to_words(const Sym& s, uint32_t* o) {
    std::memset(o, 0, ORC_SYMBOLIC_WORDS * 4);
    std::memcpy(&o[0], &s.err, 4);
    o[1] = s.mode_index; o[2] = s.pc; o[3] = s.pidx; o[4] = s.matched; o[5] = s.quant;
    for (int i = 0; i < 4; i++) o[8 + i] = s.fmt[i];
    for (int i = 0; i < 32; i++) o[12 + i] = s.packed[i];
    for (int i = 0; i < 64; i++) o[44 + i] = s.qw[i];
}


// ---------------------------------------------------------------- extension (no reference counterpart)
// Opt-in encodings the reference never emits (orc_set_extensions): an LDR void-extent block
// for a block whose texels are all equal, and single-partition dual-plane blocks, tried after
// the search and kept when their decoded error is lower.  Errors here are exact decoded
// errors: integer texels against the 8-bit texels a decoder produces (weights infilled with
// the specification's integer weights, endpoints x257, integer interpolation, 16-bit to 8-bit
// rounding), weighted by the channel weights x 10^4 in 64-bit integers.
// Symbolic words of these blocks: [6] = 1 + plane-2 component (dual plane), [7] = 1 (void
// extent, colour in [12..15]); dual plane: plane-1 weights [44..], plane-2 weights [76..].
int g_ext = 0;  // bit 0: void extent, bit 1: dual plane
const int64_t CWI[4] = {6750, 13275, 2475, 10000};

inline int dec8(int32_t v16) { return (int)(((uint32_t)v16 * 255u + 32767u) / 65535u); }
inline int32_t lerp16(int32_t e0, int32_t e1, int32_t w) { return (e0 * (64 - w) + e1 * w + 32) >> 6; }

// Integer infill of texel t from 0..64 grid weights (the specification's weights / 16).
int32_t infill_int(const Footprint& f, const DecInfo& di, const uint32_t* qw, int t) {
    if (di.W == di.T) return (int32_t)qw[t];
    int32_t s = 0;
    for (uint32_t j = 0; j < di.tw_count[t]; j++) {
        const uint32_t k = di.tw_off[t] + j;
        s += (int32_t)(f.t2w_c[k] * 16.0f) * (int32_t)qw[f.t2w_idx[k]];
    }
    return (s + 8) >> 4;
}

// LDR endpoint decoding of the ASTC specification ("LDR Endpoint Decoding": bit transfer,
// blue contraction, clamping) for the endpoint modes the encoder emits; 0..255 values.
void spec_endpoints(uint32_t cem, const uint32_t* v, int32_t* e0, int32_t* e1) {
    auto bts = [](int32_t& a, int32_t& b) {  // bit_transfer_signed(a, b)
        b = (b >> 1) | (a & 0x80);
        a = (a >> 1) & 0x3F;
        if (a & 0x20) a -= 0x40;
    };
    auto clamp255 = [](int32_t x) { return std::min(255, std::max(0, x)); };
    auto set = [](int32_t* e, int32_t r, int32_t g, int32_t b, int32_t a) { e[0] = r; e[1] = g; e[2] = b; e[3] = a; };
    int32_t x[8];
    for (int i = 0; i < 8; i++) x[i] = (int32_t)v[i];
    switch (cem) {
        case FMT_LUMINANCE: default: set(e0, x[0], x[0], x[0], 255); set(e1, x[1], x[1], x[1], 255); break;
        case FMT_LUMINANCE_DELTA: {
            const int32_t l0 = (x[0] >> 2) | (x[1] & 0xC0), l1 = std::min(l0 + (x[1] & 0x3F), 255);
            set(e0, l0, l0, l0, 255); set(e1, l1, l1, l1, 255); break;
        }
        case FMT_LUMINANCE_ALPHA: set(e0, x[0], x[0], x[0], x[2]); set(e1, x[1], x[1], x[1], x[3]); break;
        case FMT_LUMINANCE_ALPHA_DELTA: {
            bts(x[1], x[0]); bts(x[3], x[2]);
            set(e0, clamp255(x[0]), clamp255(x[0]), clamp255(x[0]), clamp255(x[2]));
            const int32_t l = clamp255(x[0] + x[1]), a = clamp255(x[2] + x[3]);
            set(e1, l, l, l, a); break;
        }
        case FMT_RGB_SCALE: case FMT_RGB_SCALE_ALPHA: {
            const int32_t a0 = cem == FMT_RGB_SCALE ? 255 : x[4], a1 = cem == FMT_RGB_SCALE ? 255 : x[5];
            set(e0, (x[0] * x[3]) >> 8, (x[1] * x[3]) >> 8, (x[2] * x[3]) >> 8, a0);
            set(e1, x[0], x[1], x[2], a1); break;
        }
        case FMT_RGB: case FMT_RGBA: {
            const int32_t a0 = cem == FMT_RGB ? 255 : x[6], a1 = cem == FMT_RGB ? 255 : x[7];
            if (x[1] + x[3] + x[5] >= x[0] + x[2] + x[4]) { set(e0, x[0], x[2], x[4], a0); set(e1, x[1], x[3], x[5], a1); }
            else {
                set(e0, (x[1] + x[5]) >> 1, (x[3] + x[5]) >> 1, x[5], a1);
                set(e1, (x[0] + x[4]) >> 1, (x[2] + x[4]) >> 1, x[4], a0);
            }
            break;
        }
        case FMT_RGB_DELTA: case FMT_RGBA_DELTA: {
            bts(x[1], x[0]); bts(x[3], x[2]); bts(x[5], x[4]);
            int32_t b3 = 0, a3 = 255;
            if (cem == FMT_RGBA_DELTA) { bts(x[7], x[6]); b3 = x[7]; a3 = x[6]; }
            int32_t c0[4] = {x[0], x[2], x[4], a3}, c1[4] = {x[0] + x[1], x[2] + x[3], x[4] + x[5], a3 + b3};
            if (x[1] + x[3] + x[5] < 0) {
                const int32_t t0[4] = {(c1[0] + c1[2]) >> 1, (c1[1] + c1[2]) >> 1, c1[2], c1[3]};
                const int32_t t1[4] = {(c0[0] + c0[2]) >> 1, (c0[1] + c0[2]) >> 1, c0[2], c0[3]};
                for (int k = 0; k < 4; k++) { c0[k] = t0[k]; c1[k] = t1[k]; }
            }
            for (int k = 0; k < 4; k++) { e0[k] = clamp255(c0[k]); e1[k] = clamp255(c1[k]); }
            break;
        }
    }
}

// Exact decoded error of a single-plane symbolic block (words) against 8-bit texels c8.
int64_t exact_error_single(const Footprint& f, const uint32_t* s, const uint8_t (*c8)[4]) {
    const BlockMode& bm = f.bms[f.bm_index[s[1] & 2047]];
    const DecInfo& di = f.dis[bm.dm];
    const int P = (int)s[2];
    int32_t e0[4][4], e1[4][4];
    for (int p = 0; p < P; p++) {
        spec_endpoints(s[8 + p], &s[12 + p * 8], e0[p], e1[p]);
        for (int k = 0; k < 4; k++) { e0[p][k] *= 257; e1[p][k] *= 257; }
    }
    const PartInfo* pi = P > 1 ? &f.pinfo[(P - 2) * 1024 + f.packed_index[P - 2][s[3]]] : nullptr;
    int64_t err = 0;
    for (int t = 0; t < f.T; t++) {
        const int p = pi ? (int)pi->of_texel[t] : 0;
        const int32_t w = infill_int(f, di, &s[44], t);
        for (int ch = 0; ch < 4; ch++) {
            const int d = (int)c8[t][ch] - dec8(lerp16(e0[p][ch], e1[p][ch], w));
            err += CWI[ch] * (int64_t)(d * d);
        }
    }
    return err;
}

// Dual-plane search of one block (single partition): plane-2 component c = 0..3 (3 only when
// alpha varies), every dual-plane block mode of the footprint whose grid is a trial
// decimation mode, in block-mode order; the first minimum of the exact error wins.
// Returns the error (INT64_MAX if no candidate fits) and its symbolic words in `o`.
int64_t dual_plane_search(const Footprint& f, const uint8_t (*c8)[4], uint32_t* o) {
    const ConstTables& ct = CT();
    const int T = f.T;
    bool calpha = true;
    int sum[4] = {0, 0, 0, 0};
    for (int t = 0; t < T; t++) { calpha = calpha && c8[t][3] == 255; for (int ch = 0; ch < 4; ch++) sum[ch] += c8[t][ch]; }
    bool const_a = true;
    for (int t = 0; t < T; t++) const_a = const_a && c8[t][3] == c8[0][3];
    std::vector<uint32_t> lookup(f.dis.size(), 0xFFFF);
    for (uint32_t d = 0; d < f.valid_dms.size(); d++) lookup[f.valid_dms[d]] = d;
    int64_t best = INT64_MAX;
    float w1[MAX_TEXELS], w2[MAX_TEXELS];
    for (int ccs = 0; ccs < 4; ccs++) {
        if (ccs == 3 && const_a) continue;
        // plane 1: the other channels' line through the mean, direction by positive-deviation sums
        float mu[4];
        for (int ch = 0; ch < 4; ch++) mu[ch] = (float)sum[ch] / (float)T;
        float S[4][4] = {{0}};
        for (int t = 0; t < T; t++) {
            float d[4];
            for (int ch = 0; ch < 4; ch++) d[ch] = ch == ccs ? 0.0f : (float)c8[t][ch] - mu[ch];
            for (int ax = 0; ax < 4; ax++)
                if (ax != ccs && d[ax] > 0.0f)
                    for (int ch = 0; ch < 4; ch++) S[ax][ch] = S[ax][ch] + d[ch];
        }
        int bax = -1; float bl = 0.0f;
        for (int ax = 0; ax < 4; ax++) {
            if (ax == ccs) continue;
            float l = S[ax][0] * S[ax][0]; l = l + S[ax][1] * S[ax][1]; l = l + S[ax][2] * S[ax][2]; l = l + S[ax][3] * S[ax][3];
            if (l > bl) { bl = l; bax = ax; }
        }
        float dir[4] = {0, 0, 0, 0};
        if (bax >= 0) { const float len = std::sqrt(bl); for (int ch = 0; ch < 4; ch++) dir[ch] = S[bax][ch] / len; }
        float pmin = 1e30f, pmax = -1e30f, prm[MAX_TEXELS];
        for (int t = 0; t < T; t++) {
            float d[4];
            for (int ch = 0; ch < 4; ch++) d[ch] = ch == ccs ? 0.0f : (float)c8[t][ch] - mu[ch];
            float v = d[0] * dir[0]; v = v + d[1] * dir[1]; v = v + d[2] * dir[2]; v = v + d[3] * dir[3];
            prm[t] = v; pmin = fmn(pmin, v); pmax = fmx(pmax, v);
        }
        int vmin = 255, vmax = 0;
        for (int t = 0; t < T; t++) { vmin = std::min(vmin, (int)c8[t][ccs]); vmax = std::max(vmax, (int)c8[t][ccs]); }
        for (int t = 0; t < T; t++) {
            w1[t] = pmax > pmin ? (prm[t] - pmin) / (pmax - pmin) : 0.0f;
            w2[t] = vmax > vmin ? (float)(c8[t][ccs] - vmin) / (float)(vmax - vmin) : 0.0f;
        }
        const bool rgb_only = calpha && ccs != 3;
        const int cem = rgb_only ? FMT_RGB : FMT_RGBA, nint = rgb_only ? 6 : 8;
        for (uint32_t m = 0; m < 2048; m++) {
            const uint32_t bi = f.bm_index[m];
            if (bi == 0xFFFF) continue;
            const BlockMode& bm = f.bms[bi];
            if (!bm.dual || lookup[bm.dm] == 0xFFFF) continue;
            const DecInfo& di = f.dis[bm.dm];
            const int avail = 109 - (int)bm.weight_bits;
            int qc = -1;
            for (int q = 20; q >= 4; q--) if ((int)ise_bitcount(nint, q) <= avail) { qc = q; break; }
            if (qc < 0) continue;
            // decimate, quantise (pass07's rule over [0, 1]) both planes
            uint32_t qw[2][MAX_WEIGHTS];
            const float qlm1 = (float)(LEVELS[bm.quant] - 1);
            const int off = ct.q2u_off[bm.quant];
            for (int pl = 0; pl < 2; pl++) {
                const float* wv = pl ? w2 : w1;
                for (uint32_t i = 0; i < di.W; i++) {
                    float dw;
                    if (di.W == di.T) dw = wv[i];
                    else {
                        float num = 0.0f, den = 0.0f;
                        for (uint32_t j = 0; j < di.wt_count[i]; j++) {
                            const uint32_t k = di.wt_off[i] + j;
                            num = num + f.w2t_c[k] * wv[f.w2t_idx[k]];
                            den = den + f.w2t_c[k];
                        }
                        dw = num / den;
                    }
                    const float ix = clampf(dw, 0.0f, 1.0f), ix1 = ix * qlm1;
                    const uint32_t wl = f2u(ix1), wh = std::min(wl + 1, f2u(qlm1));
                    const uint32_t li = ct.q2u[off + wl], hi = ct.q2u[off + wh];
                    qw[pl][i] = ((float)li + (float)hi) < (128.0f * ix) ? hi : li;
                }
            }
            // endpoints per channel by least squares on the channel's plane
            int32_t wt[2][MAX_TEXELS];
            for (int t = 0; t < T; t++) { wt[0][t] = infill_int(f, di, qw[0], t); wt[1][t] = infill_int(f, di, qw[1], t); }
            int ue[2][4];
            for (int ch = 0; ch < 4; ch++) {
                const int32_t* wp = wt[ch == ccs ? 1 : 0];
                float a = 0.0f, b = 0.0f, cc = 0.0f, s0 = 0.0f, s1 = 0.0f;
                for (int t = 0; t < T; t++) {
                    const float w = (float)wp[t] / 64.0f, om = 1.0f - w, x = (float)c8[t][ch];
                    a = a + om * om; b = b + om * w; cc = cc + w * w; s0 = s0 + om * x; s1 = s1 + w * x;
                }
                const float det = a * cc - b * b;
                float e0, e1;
                if (det > 0.0001f * (a * cc)) { e0 = (cc * s0 - b * s1) / det; e1 = (a * s1 - b * s0) / det; }
                else { e0 = e1 = (float)sum[ch] / (float)T; }
                e0 = clampf(e0, 0.0f, 255.0f); e1 = clampf(e1, 0.0f, 255.0f);
                ue[0][ch] = ct.cu2u[qc - 4][(int)rne(e0) * 2 + 1];
                ue[1][ch] = ct.cu2u[qc - 4][(int)rne(e1) * 2 + 1];
            }
            if (rgb_only) { ue[0][3] = 255; ue[1][3] = 255; }
            // the decoder swaps RGB(A) direct endpoints whose second sum is the smaller
            if (ue[1][0] + ue[1][1] + ue[1][2] < ue[0][0] + ue[0][1] + ue[0][2]) {
                for (int ch = 0; ch < 4; ch++) std::swap(ue[0][ch], ue[1][ch]);
                for (int pl = 0; pl < 2; pl++)
                    for (uint32_t i = 0; i < di.W; i++) qw[pl][i] = 64 - qw[pl][i];
                for (int t = 0; t < T; t++) { wt[0][t] = infill_int(f, di, qw[0], t); wt[1][t] = infill_int(f, di, qw[1], t); }
            }
            int64_t err = 0;
            for (int t = 0; t < T; t++)
                for (int ch = 0; ch < 4; ch++) {
                    const int d = (int)c8[t][ch] - dec8(lerp16(ue[0][ch] * 257, ue[1][ch] * 257, wt[ch == ccs ? 1 : 0][t]));
                    err += CWI[ch] * (int64_t)(d * d);
                }
            if (err < best) {
                best = err;
                std::memset(o, 0, ORC_SYMBOLIC_WORDS * 4);
                const float fe = (float)err * 1e-4f;
                std::memcpy(&o[0], &fe, 4);
                o[1] = m; o[2] = 1; o[5] = (uint32_t)qc; o[6] = 1 + ccs; o[8] = (uint32_t)cem;
                for (int ch = 0; ch < nint / 2; ch++) { o[12 + 2 * ch] = (uint32_t)ue[0][ch]; o[12 + 2 * ch + 1] = (uint32_t)ue[1][ch]; }
                for (uint32_t i = 0; i < di.W; i++) { o[44 + i] = qw[0][i]; o[76 + i] = qw[1][i]; }
            }
        }
    }
    return best;
}

// Applies the enabled extensions to one block's symbolic words (c8: its edge-clamped texels).
void apply_extensions(const Footprint& f, const uint8_t (*c8)[4], uint32_t* s) {
    if (!g_ext) return;
    const int T = f.T;
    bool constant = true;
    for (int t = 1; t < T && constant; t++)
        for (int ch = 0; ch < 4; ch++) constant = constant && c8[t][ch] == c8[0][ch];
    if ((g_ext & 1) && constant) {
        std::memset(s, 0, ORC_SYMBOLIC_WORDS * 4);
        s[2] = 1; s[7] = 1;
        for (int ch = 0; ch < 4; ch++) s[12 + ch] = c8[0][ch];
        return;
    }
    if (!(g_ext & 2)) return;
    const int64_t es = exact_error_single(f, s, c8);
    uint32_t o[ORC_SYMBOLIC_WORDS];
    const int64_t ed = dual_plane_search(f, c8, o);
    if (ed < es) std::memcpy(s, o, sizeof(o));
}

void block_c8(const uint8_t* img, int w, int h, int bx, int by, int bxi, int byi, uint8_t (*c8)[4]) {
    int t = 0;
    for (int dy = 0; dy < by; dy++) {
        const int y = std::min(byi * by + dy, h - 1);
        for (int dx = 0; dx < bx; dx++, t++) {
            const int x = std::min(bxi * bx + dx, w - 1);
            for (int c = 0; c < 4; c++) c8[t][c] = img[((size_t)y * w + x) * 4 + c];
        }
    }
}

template <class F>
void run_parallel(int n, int threads, F fn) {
#ifdef _OPENMP
    int nt = threads > 0 ? threads : omp_get_max_threads();
#pragma omp parallel num_threads(nt)
    {
        std::unique_ptr<PBWork> w(new PBWork());
#pragma omp for schedule(static)
        for (int i = 0; i < n; i++) fn(i, *w);
    }
#else
    (void)threads;
    std::unique_ptr<PBWork> w(new PBWork());
    for (int i = 0; i < n; i++) fn(i, *w);
#endif
}

}  // namespace

extern "C" {

int orc_set_extensions(int flags) {
    const int prev = g_ext;
    g_ext = flags & 3;
    return prev;
}

int orc_set_semantics(int fixed) {
    const int prev = g_fixed;
    g_fixed = fixed ? 1 : 0;
    return prev;
}

int orc_encode(const uint8_t* rgba, int width, int height, int bx, int by, int threads,
               uint8_t* out_blocks, uint32_t* symbolic) {
    if (!rgba || width <= 0 || height <= 0 || !valid_footprint(bx, by) || !out_blocks) return -1;
    const Footprint& f = *get_fp(bx, by);
    CT();
    int nbx = (width + bx - 1) / bx, nby = (height + by - 1) / by, n = nbx * nby;
    run_parallel(n, threads, [&](int i, PBWork& w) {
        InputBlock b; make_block(rgba, width, height, bx, by, i % nbx, i / nbx, b);
        Sym s = encode_block(f, b, w);
        uint32_t words[ORC_SYMBOLIC_WORDS]; sym_to_words(s, words);
        if (g_ext) { uint8_t c8[MAX_TEXELS][4]; block_c8(rgba, width, height, bx, by, i % nbx, i / nbx, c8); apply_extensions(f, c8, words); }
        if (symbolic) std::memcpy(symbolic + (size_t)i * ORC_SYMBOLIC_WORDS, words, sizeof(words));
        sym_to_phys(f, words, out_blocks + (size_t)i * 16);
    });
    return 0;
}

int orc_encode_iters(const uint8_t* rgba, int width, int height, int bx, int by, int threads, int refine_iters,
                     uint8_t* out_blocks, uint32_t* symbolic) {
    if (!rgba || width <= 0 || height <= 0 || !valid_footprint(bx, by) || !out_blocks || refine_iters < 1) return -1;
    const Footprint& f = *get_fp(bx, by);
    CT();
    int nbx = (width + bx - 1) / bx, nby = (height + by - 1) / by, n = nbx * nby;
    run_parallel(n, threads, [&](int i, PBWork& w) {
        InputBlock b; make_block(rgba, width, height, bx, by, i % nbx, i / nbx, b);
        Sym s = encode_block(f, b, w, refine_iters);
        uint32_t words[ORC_SYMBOLIC_WORDS]; sym_to_words(s, words);
        if (g_ext) { uint8_t c8[MAX_TEXELS][4]; block_c8(rgba, width, height, bx, by, i % nbx, i / nbx, c8); apply_extensions(f, c8, words); }
        if (symbolic) std::memcpy(symbolic + (size_t)i * ORC_SYMBOLIC_WORDS, words, sizeof(words));
        sym_to_phys(f, words, out_blocks + (size_t)i * 16);
    });
    return 0;
}

int orc_encode_blocks(const float* texels, int nblocks, int bx, int by, int threads, uint32_t* symbolic, uint8_t* out_blocks) {
    if (!texels || nblocks < 0 || !valid_footprint(bx, by)) return -1;
    const Footprint& f = *get_fp(bx, by);
    CT();
    const int T = bx * by;
    run_parallel(nblocks, threads, [&](int i, PBWork& w) {
        InputBlock b; std::memset(&b, 0, sizeof(b));
        for (int t = 0; t < T; t++) for (int c = 0; c < 4; c++) comp(b.px[t], c) = texels[((size_t)i * T + t) * 4 + c];
        flags_from_texels(b, T);
        Sym s = encode_block(f, b, w);
        uint32_t words[ORC_SYMBOLIC_WORDS]; sym_to_words(s, words);
        if (symbolic) std::memcpy(symbolic + (size_t)i * ORC_SYMBOLIC_WORDS, words, sizeof(words));
        if (out_blocks) sym_to_phys(f, words, out_blocks + (size_t)i * 16);
    });
    return 0;
}

int orc_encode_restricted(const uint8_t* rgba, int width, int height, int bx, int by, int threads,
                          const uint16_t* picks, const uint64_t* masks, int topn, int refine_iters,
                          uint8_t* out_blocks, uint32_t* symbolic, uint8_t* found) {
    if (!rgba || width <= 0 || height <= 0 || !valid_footprint(bx, by) || !picks || !masks || !found ||
        topn < 1 || topn > NUM_CAND || refine_iters < 1)
        return -1;
    const Footprint& f = *get_fp(bx, by);
    if (f.valid_bms.size() > 256) return -1;  // masks hold 256 block modes
    CT();
    int nbx = (width + bx - 1) / bx, nby = (height + by - 1) / by, n = nbx * nby;
    for (int i = 0; i < n; i++) {
        const uint16_t* pk = picks + (size_t)i * ORC_PICK_WORDS;
        if (pk[0] > 16) return -1;
        for (int j = 0; j < pk[0]; j++) {
            const int P = 2 + (pk[2 + j] >> 10), e = pk[2 + j] & 1023;
            if (P > 4 || e >= (int)f.count_selected[P - 1]) return -1;
        }
    }
    run_parallel(n, threads, [&](int i, PBWork& w) {
        InputBlock b; make_block(rgba, width, height, bx, by, i % nbx, i / nbx, b);
        bool ok = false;
        Sym s = encode_block_restricted(f, b, w, picks + (size_t)i * ORC_PICK_WORDS, masks + (size_t)i * 16, topn,
                                        refine_iters, ok);
        found[i] = ok ? 1 : 0;
        uint32_t words[ORC_SYMBOLIC_WORDS];
        if (ok) sym_to_words(s, words);
        else std::memset(words, 0, sizeof(words));  // no block to describe
        if (ok && g_ext) { uint8_t c8[MAX_TEXELS][4]; block_c8(rgba, width, height, bx, by, i % nbx, i / nbx, c8); apply_extensions(f, c8, words); }
        if (symbolic) std::memcpy(symbolic + (size_t)i * ORC_SYMBOLIC_WORDS, words, sizeof(words));
        if (out_blocks) {
            if (ok) sym_to_phys(f, words, out_blocks + (size_t)i * 16);
            else std::memset(out_blocks + (size_t)i * 16, 0, 16);
        }
    });
    return 0;
}

int orc_symbolic_to_physical(int bx, int by, const uint32_t* symbolic, uint8_t* out16) {
    if (!valid_footprint(bx, by)) return -1;
    sym_to_phys(*get_fp(bx, by), symbolic, out16);
    return 0;
}

int orc_counts(int bx, int by, uint32_t* c) {
    if (!valid_footprint(bx, by)) return -1;
    const Footprint& f = *get_fp(bx, by);
    c[0] = f.T; c[1] = (uint32_t)f.bms.size(); c[2] = (uint32_t)f.dis.size();
    c[3] = (uint32_t)f.t2w_idx.size(); c[4] = (uint32_t)f.w2t_idx.size();
    for (int i = 0; i < 4; i++) { c[5 + i] = f.count_selected[i]; c[9 + i] = f.count_all[i]; }
    return 0;
}
int orc_block_modes(int bx, int by, uint32_t* bm_index, uint32_t* bms) {
    if (!valid_footprint(bx, by)) return -1;
    const Footprint& f = *get_fp(bx, by);
    std::memcpy(bm_index, f.bm_index, sizeof(f.bm_index));
    for (size_t i = 0; i < f.bms.size(); i++) {
        const BlockMode& b = f.bms[i];
        uint32_t* o = bms + i * 5; o[0] = b.mode_index; o[1] = b.dm; o[2] = b.quant; o[3] = b.weight_bits; o[4] = b.dual;
    }
    return 0;
}
int orc_decimation(int bx, int by, uint32_t* dmodes, uint32_t* dinfo) {
    if (!valid_footprint(bx, by)) return -1;
    const Footprint& f = *get_fp(bx, by);
    for (size_t i = 0; i < f.dis.size(); i++) {
        const DecMode& m = f.dms[i];
        dmodes[i * 4 + 0] = m.maxprec1; dmodes[i * 4 + 1] = m.maxprec2; dmodes[i * 4 + 2] = m.refprec1; dmodes[i * 4 + 3] = m.refprec2;
        const DecInfo& d = f.dis[i];
        uint32_t* o = dinfo + i * 424;
        o[0] = d.T; o[1] = d.W; o[2] = d.wx; o[3] = d.wy; o[4] = d.max_quant_level; o[5] = d.max_angular_steps; o[6] = d.max_quant_steps; o[7] = 0;
        for (int t = 0; t < 144; t++) { o[8 + t] = d.tw_count[t]; o[152 + t] = d.tw_off[t]; }
        for (int w = 0; w < 64; w++) { o[296 + w] = d.wt_count[w]; o[360 + w] = d.wt_off[w]; }
    }
    return 0;
}
int orc_maps(int bx, int by, uint32_t* ti, float* tc, uint32_t* wi, float* wc) {
    if (!valid_footprint(bx, by)) return -1;
    const Footprint& f = *get_fp(bx, by);
    for (size_t i = 0; i < f.t2w_idx.size(); i++) { ti[i] = f.t2w_idx[i]; tc[i] = f.t2w_c[i]; }
    for (size_t i = 0; i < f.w2t_idx.size(); i++) { wi[i] = f.w2t_idx[i]; wc[i] = f.w2t_c[i]; }
    return 0;
}
int orc_partitions(int bx, int by, uint32_t* pinfo, uint64_t* cov2, uint64_t* cov3, uint64_t* cov4, uint32_t* km, uint16_t* pidx) {
    if (!valid_footprint(bx, by)) return -1;
    const Footprint& f = *get_fp(bx, by);
    for (int i = 0; i < 3073; i++) {
        const PartInfo& p = f.pinfo[i];
        uint32_t* o = pinfo + (size_t)i * 150;
        o[0] = p.count; o[1] = p.index;
        for (int k = 0; k < 4; k++) o[2 + k] = p.texel_count[k];
        for (int t = 0; t < 144; t++) o[6 + t] = p.of_texel[t];
    }
    std::memcpy(cov2, f.cov[2].data(), 1024 * 2 * 8);
    std::memcpy(cov3, f.cov[3].data(), 1024 * 3 * 8);
    std::memcpy(cov4, f.cov[4].data(), 1024 * 4 * 8);
    std::memcpy(km, f.kmeans, sizeof(f.kmeans));
    std::memcpy(pidx, f.packed_index, sizeof(f.packed_index));
    return 0;
}
int orc_angular(float* s, float* c) {
    const Footprint& f = *get_fp(4, 4);
    std::memcpy(s, f.sin_t.data(), 16384 * 4);
    std::memcpy(c, f.cos_t.data(), 16384 * 4);
    return 16384;
}
int orc_trial_modes(int bx, int by, uint32_t* n_dm, uint32_t* vdm, uint32_t* n_bm, uint32_t* vbm) {
    if (!valid_footprint(bx, by)) return -1;
    const Footprint& f = *get_fp(bx, by);
    *n_dm = (uint32_t)f.valid_dms.size(); *n_bm = (uint32_t)f.valid_bms.size();
    if (vdm) for (size_t i = 0; i < f.valid_dms.size(); i++) vdm[i] = f.valid_dms[i];
    if (vbm) for (size_t i = 0; i < f.valid_bms.size(); i++) { vbm[2 * i] = f.valid_bms[i].first; vbm[2 * i + 1] = f.valid_bms[i].second; }
    return 0;
}
int orc_const_tables(int32_t* q2u, int32_t* qmt, int32_t* cu2u, int32_t* pn, float* bqe, uint8_t* trits, uint8_t* quints, uint8_t* wscr, uint8_t* cscr) {
    const ConstTables& t = CT();
    std::memcpy(q2u, t.q2u, sizeof(t.q2u)); std::memcpy(qmt, t.qmt, sizeof(t.qmt));
    std::memcpy(cu2u, t.cu2u, sizeof(t.cu2u)); std::memcpy(pn, t.prev_next, sizeof(t.prev_next));
    std::memcpy(bqe, t.bqe, sizeof(t.bqe)); std::memcpy(trits, t.trits, sizeof(t.trits));
    std::memcpy(quints, t.quints, sizeof(t.quints)); std::memcpy(wscr, t.wscr, sizeof(t.wscr));
    std::memcpy(cscr, t.cscr, sizeof(t.cscr));
    return 0;
}
int orc_partition_search(int bx, int by, const float* texels, int P, uint32_t* entries) {
    if (!valid_footprint(bx, by) || P < 2 || P > 4) return -1;
    const Footprint& f = *get_fp(bx, by);
    InputBlock b; std::memset(&b, 0, sizeof(b));
    for (int t = 0; t < f.T; t++) for (int c = 0; c < 4; c++) comp(b.px[t], c) = texels[t * 4 + c];
    flags_from_texels(b, f.T);
    std::unique_ptr<InputBlock[]> out(new InputBlock[4]);
    return partition_search(f, b, P, out.get(), entries);
}
int orc_front_candidates(int bx, int by, const float* texels, int P, int entry, float* ep, uint32_t* cands) {
    if (!valid_footprint(bx, by) || P < 1 || P > 4 || entry < 0 || entry > 1023 || !ep || !cands) return -1;
    const Footprint& f = *get_fp(bx, by);
    InputBlock b; std::memset(&b, 0, sizeof(b));
    for (int t = 0; t < f.T; t++) for (int c = 0; c < 4; c++) comp(b.px[t], c) = texels[t * 4 + c];
    flags_from_texels(b, f.T);
    InputBlock pb = b;
    if (P > 1) make_pb(f, b, P, entry, pb);
    std::unique_ptr<PBWork> w(new PBWork());
    process_pb(f, pb, P, *w, nullptr, NUM_CAND, 0);  // passes 01-12, no refinement
    for (int q = 0; q < 4; q++)
        for (int c = 0; c < 4; c++) {
            ep[q * 12 + c] = compc(w->ei.part[q].avg, c);
            ep[q * 12 + 4 + c] = compc(w->ei.part[q].ep0, c);
            ep[q * 12 + 8 + c] = compc(w->ei.part[q].ep1, c);
        }
    std::memset(cands, 0, sizeof(uint32_t) * NUM_CAND * 71);
    for (int k = 0; k < w->ncand; k++) {
        const Cand& c = w->cand[k];
        uint32_t* o = cands + k * 71;
        o[0] = c.bm_lookup; o[1] = c.ql; o[2] = c.qlm;
        for (int q = 0; q < 4; q++) o[3 + q] = c.fmt[q];
        for (int i = 0; i < 64; i++) o[7 + i] = i < MAX_WEIGHTS ? c.qw[i] : 0;
    }
    return w->ncand;
}
int orc_refined_candidates(int bx, int by, const float* texels, int P, int entry, int iters, uint32_t* out) {
    if (!valid_footprint(bx, by) || P < 1 || P > 4 || entry < 0 || entry > 1023 || iters < 1 || iters > 6 || !out) return -1;
    const Footprint& f = *get_fp(bx, by);
    InputBlock b; std::memset(&b, 0, sizeof(b));
    for (int t = 0; t < f.T; t++) for (int c = 0; c < 4; c++) comp(b.px[t], c) = texels[t * 4 + c];
    flags_from_texels(b, f.T);
    InputBlock pb = b;
    if (P > 1) make_pb(f, b, P, entry, pb);
    std::unique_ptr<PBWork> w(new PBWork());
    process_pb(f, pb, P, *w, nullptr, NUM_CAND, iters);
    std::memset(out, 0, sizeof(uint32_t) * NUM_CAND * 104);
    for (int k = 0; k < NUM_CAND; k++) {
        const Cand& c = w->top[k];
        uint32_t* o = out + k * 104;
        std::memcpy(&o[0], &c.total_error, 4);
        if (!(c.total_error < ERR_DEFAULT)) continue;
        o[1] = c.bm_lookup; o[2] = c.final_q; o[3] = c.matched;
        for (int q = 0; q < 4; q++) o[4 + q] = c.ffmt[q];
        for (int i = 0; i < 32; i++) o[8 + i] = c.packed[i];
        for (int i = 0; i < 64; i++) o[40 + i] = c.qw[i];
    }
    return w->ncand;
}
int orc_partition_order(int bx, int by, const float* texels, int P, uint32_t* mismatch, uint32_t* order) {
    if (!valid_footprint(bx, by) || P < 2 || P > 4 || !mismatch || !order) return -1;
    const Footprint& f = *get_fp(bx, by);
    InputBlock b; std::memset(&b, 0, sizeof(b));
    for (int t = 0; t < f.T; t++) for (int c = 0; c < 4; c++) comp(b.px[t], c) = texels[t * 4 + c];
    flags_from_texels(b, f.T);
    std::unique_ptr<InputBlock[]> out(new InputBlock[4]);
    uint32_t entries[4];
    partition_search(f, b, P, out.get(), entries, mismatch, order);
    return (int)f.count_selected[P - 1];
}

}  // extern "C"
