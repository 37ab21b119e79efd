// Host construction of the search tables (see tables.h for the reference map).
#include "tables.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>

namespace astcb200 {

namespace {

const int kLevels[21] = {2, 3, 4, 5, 6, 8, 10, 12, 16, 20, 24, 32, 40, 48, 64, 80, 96, 128, 160, 192, 256};
const int kStepsForQuant[12] = {2, 3, 4, 5, 6, 8, 10, 12, 16, 20, 24, 32};  // astc.h:157

// Bits / trits / quints of a quant method (ASTC integer sequence encoding).
struct Btq { int bits, trits, quints; };
Btq btq(int q) {
    int L = kLevels[q];
    Btq r{0, 0, 0};
    if (L % 3 == 0) { r.trits = 1; L /= 3; }
    else if (L % 5 == 0) { r.quints = 1; L /= 5; }
    while ((1 << r.bits) < L) r.bits++;
    return r;
}

unsigned ise_bits(unsigned count, int q) {  // physical_compression.cpp:625-639
    if (q < 0 || q > 20) return 1024;
    Btq b = btq(q);
    if (b.trits) return (count * (8 + 5 * b.bits) + 4) / 5;
    if (b.quints) return (count * (7 + 3 * b.bits) + 2) / 3;
    return count * b.bits;
}

// Replicates the low `bits` bits of v until `width` bits are filled.
int replicate(int v, int bits, int width) {
    int out = 0, have = 0;
    while (have < width) { out = (out << bits) | v; have += bits; }
    return out >> (have - width);
}

// ASTC weight unquantisation to 0..64 for the ISE value v of method q.
int weight_unquant(int q, int v) {
    Btq b = btq(q);
    int r;
    if (!b.trits && !b.quints) {
        r = replicate(v, b.bits, 6);
    } else {
        const int D = v >> b.bits, m = v & ((1 << b.bits) - 1);
        const int A = (m & 1) ? 0x7F : 0, b1 = (m >> 1) & 1, b2 = (m >> 2) & 1;
        if (b.bits == 0) {
            static const int t0[3] = {0, 32, 63}, q0[5] = {0, 16, 32, 47, 63};
            r = b.trits ? t0[D] : q0[D];
        } else {
            int B, C;
            if (b.trits) {
                C = b.bits == 1 ? 50 : b.bits == 2 ? 23 : 11;
                B = b.bits == 1 ? 0 : b.bits == 2 ? (b1 * 0x45) : (b2 * 0x42 + b1 * 0x21);
            } else {
                C = b.bits == 1 ? 28 : 13;
                B = b.bits == 1 ? 0 : b1 * 0x42;
            }
            r = (A & 0x20) | (((D * C + B) ^ A) >> 2);
        }
    }
    return r > 32 ? r + 1 : r;
}

// ASTC colour endpoint unquantisation to 0..255 for the ISE value v of method q.
int color_unquant(int q, int v) {
    Btq b = btq(q);
    if (!b.trits && !b.quints) return replicate(v, b.bits, 8);
    const int D = v >> b.bits, m = v & ((1 << b.bits) - 1);
    const int A = (m & 1) ? 0x1FF : 0;
    auto bit = [m](int i) { return (m >> i) & 1; };
    int B = 0, C;
    if (b.trits) {
        static const int kC[7] = {0, 204, 93, 44, 22, 11, 5};
        C = kC[b.bits];
        switch (b.bits) {
            case 2: B = bit(1) * 0x116; break;                                       // b000b0bb0
            case 3: B = bit(2) * 0x10A + bit(1) * 0x85; break;                       // cb000cbcb
            case 4: B = bit(3) * 0x104 + bit(2) * 0x82 + bit(1) * 0x41; break;       // dcb000dcb
            case 5: B = bit(4) * 0x102 + bit(3) * 0x81 + bit(2) * 0x40 + bit(1) * 0x20; break;  // edcb000ed
            case 6: B = bit(5) * 0x101 + bit(4) * 0x80 + bit(3) * 0x40 + bit(2) * 0x20 + bit(1) * 0x10; break;  // fedcb000f
            default: break;
        }
    } else {
        static const int kC[6] = {0, 113, 54, 26, 13, 6};
        C = kC[b.bits];
        switch (b.bits) {
            case 2: B = bit(1) * 0x10C; break;                                       // b0000bb00
            case 3: B = bit(2) * 0x105 + bit(1) * 0x82; break;                       // cb0000cbc
            case 4: B = bit(3) * 0x102 + bit(2) * 0x81 + bit(1) * 0x40; break;       // dcb0000dc
            case 5: B = bit(4) * 0x101 + bit(3) * 0x80 + bit(2) * 0x40 + bit(1) * 0x20; break;  // edcb0000e
            default: break;
        }
    }
    return (A & 0x80) | (((D * C + B) ^ A) >> 2);
}

// ASTC trit / quint block decoding; the encoder tables keep, for each digit
// tuple, the largest code that decodes to it.
void trits_of(int T, int t[5]) {
    auto bit = [](int x, int i) { return (x >> i) & 1; };
    int C;
    if (((T >> 2) & 7) == 7) { C = (((T >> 5) & 7) << 2) | (T & 3); t[4] = 2; t[3] = 2; }
    else {
        C = T & 31;
        if (((T >> 5) & 3) == 3) { t[4] = 2; t[3] = bit(T, 7); } else { t[4] = bit(T, 7); t[3] = (T >> 5) & 3; }
    }
    if ((C & 3) == 3) { t[2] = 2; t[1] = bit(C, 4); t[0] = (bit(C, 3) << 1) | (bit(C, 2) & ~bit(C, 3) & 1); }
    else if (((C >> 2) & 3) == 3) { t[2] = 2; t[1] = 2; t[0] = C & 3; }
    else { t[2] = bit(C, 4); t[1] = (C >> 2) & 3; t[0] = (bit(C, 1) << 1) | (bit(C, 0) & ~bit(C, 1) & 1); }
}
void quints_of(int Q, int q[3]) {
    auto bit = [](int x, int i) { return (x >> i) & 1; };
    if (((Q >> 1) & 3) == 3 && ((Q >> 5) & 3) == 0) {
        const int b0 = bit(Q, 0);
        q[2] = (b0 << 2) | ((bit(Q, 4) & (1 - b0)) << 1) | (bit(Q, 3) & (1 - b0));
        q[1] = 4; q[0] = 4;
        return;
    }
    int C;
    if (((Q >> 1) & 3) == 3) { q[2] = 4; C = (((Q >> 3) & 3) << 3) | (((~Q >> 5) & 3) << 1) | (Q & 1); }
    else { q[2] = (Q >> 5) & 3; C = Q & 31; }
    if ((C & 7) == 5) { q[1] = 4; q[0] = (C >> 3) & 3; } else { q[1] = (C >> 3) & 3; q[0] = C & 7; }
}

struct ConstTables {
    uint8_t q2u[142], q2u_start[12];
    int8_t qmt[10][128];
    uint8_t cu2u[17][512];
    uint16_t prev_next[12][65];
    float bqe[17];
    uint8_t wscr[12][32], cscr[17][256], trits[243], quints[125];
};

ConstTables make_const_tables() {
    ConstTables c;
    std::memset(&c, 0, sizeof(c));
    int pos = 0;
    for (int q = 0; q < 12; q++) {
        const int L = kLevels[q];
        std::vector<std::pair<int, int>> v;  // (unquantised value, ISE value)
        for (int i = 0; i < L; i++) v.emplace_back(weight_unquant(q, i), i);
        std::sort(v.begin(), v.end());
        c.q2u_start[q] = (uint8_t)pos;
        for (int k = 0; k < L; k++) {
            c.q2u[pos + k] = (uint8_t)v[k].first;
            c.wscr[q][k] = (uint8_t)v[k].second;
            const int lo = v[std::max(k - 1, 0)].first, hi = v[std::min(k + 1, L - 1)].first;
            c.prev_next[q][v[k].first] = (uint16_t)(lo | (hi << 8));
        }
        pos += L;
    }
    int qmt[10][128];
    for (auto& row : qmt) for (int& x : row) x = -1;
    for (int q = 0; q < 21; q++)
        for (int n = 1; n <= 9; n++) { unsigned b = ise_bits(2 * n, q); if (b < 128) qmt[n][b] = q; }
    for (int n = 0; n < 10; n++) {
        int best = -1;
        for (int b = 0; b < 128; b++) { best = std::max(best, qmt[n][b]); c.qmt[n][b] = (int8_t)best; }
    }
    for (int k = 0; k < 17; k++) {
        const int q = k + 4, L = kLevels[q];
        std::vector<int> val(L);
        for (int i = 0; i < L; i++) val[i] = color_unquant(q, i);
        for (int idx = 0; idx < 512; idx++) {  // nearest to idx/2; even idx ties down, odd up
            const int v = idx >> 1;
            int bd = 1 << 30, bu = 0;
            for (int u : val) {
                const int d = std::abs(u - v);
                if (d < bd || (d == bd && ((idx & 1) ? u > bu : u < bu))) { bd = d; bu = u; }
            }
            c.cu2u[k][idx] = (uint8_t)bu;
        }
        for (int v = 0; v < 256; v++) {  // nearest representable value; ties to the higher code
            int bd = 1 << 30, be = 0;
            for (int e = 0; e < L; e++) { const int d = std::abs(val[e] - v); if (d <= bd) { bd = d; be = e; } }
            c.cscr[k][v] = (uint8_t)be;
        }
    }
    static const int div[17] = {5, 7, 9, 11, 15, 19, 23, 31, 39, 47, 63, 79, 95, 127, 159, 191, 255};
    const float base = (65536.0f * 65536.0f) / 18.0f;
    for (int i = 0; i < 17; i++) c.bqe[i] = base / (float)(div[i] * div[i]);
    for (int T = 0; T < 256; T++) { int t[5]; trits_of(T, t); c.trits[(((t[4] * 3 + t[3]) * 3 + t[2]) * 3 + t[1]) * 3 + t[0]] = (uint8_t)T; }
    for (int Q = 0; Q < 128; Q++) { int q[3]; quints_of(Q, q); c.quints[(q[2] * 5 + q[1]) * 5 + q[0]] = (uint8_t)Q; }
    return c;
}

const ConstTables& const_tables() {
    static const ConstTables c = make_const_tables();
    return c;
}

// ------------------------------------------------------------ block modes
struct ModeDecode { unsigned xw, yw, quant, weight_bits; bool dual; };

// ASTC 2D block mode field decode (metadata_structures.cpp:72-173).
bool decode_mode(unsigned m, ModeDecode& o) {
    unsigned q = (m >> 4) & 1, H = (m >> 9) & 1, D = (m >> 10) & 1, A = (m >> 5) & 3;
    if (m & 3) {
        q |= (m & 3) << 1;
        unsigned B = (m >> 7) & 3;
        switch ((m >> 2) & 3) {
            case 0: o.xw = B + 4; o.yw = A + 2; break;
            case 1: o.xw = B + 8; o.yw = A + 2; break;
            case 2: o.xw = A + 2; o.yw = B + 8; break;
            default:
                B &= 1;
                if (m & 0x100) { o.xw = B + 2; o.yw = A + 2; } else { o.xw = A + 2; o.yw = B + 6; }
        }
    } else {
        q |= ((m >> 2) & 3) << 1;
        if (((m >> 2) & 3) == 0) return false;
        unsigned B = (m >> 9) & 3;
        switch ((m >> 7) & 3) {
            case 0: o.xw = 12; o.yw = A + 2; break;
            case 1: o.xw = A + 2; o.yw = 12; break;
            case 2: o.xw = A + 6; o.yw = B + 6; D = 0; H = 0; break;
            default:
                if (((m >> 5) & 3) == 0) { o.xw = 6; o.yw = 10; }
                else if (((m >> 5) & 3) == 1) { o.xw = 10; o.yw = 6; }
                else return false;
        }
    }
    const unsigned n = o.xw * o.yw * (D + 1);
    o.quant = (q - 2) + 6 * H;
    o.dual = D != 0;
    o.weight_bits = ise_bits(n, (int)o.quant);
    return n <= 64 && o.weight_bits >= 24 && o.weight_bits <= 96;
}

}  // namespace

// ------------------------------------------------------------ reference-layout host tables
struct HostTables {
    int bx, by, T;
    uint32_t bm_index[2048];
    struct Bm { uint32_t mode, dm, quant, bits, dual; };
    std::vector<Bm> bms;
    struct Dm {
        uint32_t maxprec1, maxprec2, ref1, ref2;
        uint32_t W, wx, wy, maxq, steps, qsteps;
        uint32_t tw_count[kMaxTexels], tw_off[kMaxTexels], wt_count[kMaxWeights], wt_off[kMaxWeights];
    };
    std::vector<Dm> dms;
    std::vector<uint32_t> t2w_w, w2t_t;
    std::vector<uint8_t> t2w_k, w2t_k;   // contribution in 1/16 units
    struct Part { uint32_t count, seed, tcount[4]; uint8_t of[kMaxTexels]; };
    std::vector<Part> parts;               // [3*1024 + 1], P=2..4 then P=1
    uint32_t sel[4], all[4];
    std::vector<uint64_t> cov[5];
    uint32_t kmeans[64];
    uint16_t packed_index[3][1024];
    std::vector<uint32_t> valid_dms;
    std::vector<std::pair<uint32_t, uint32_t>> valid_bms;
    std::vector<float> sin_t, cos_t;
};

namespace {

// Bilinear texel<->weight maps of one weight grid (metadata_structures.cpp:176-275).
void add_grid(HostTables& h, unsigned xw, unsigned yw, HostTables::Dm& d) {
    const unsigned X = h.bx, Y = h.by, T = X * Y, W = xw * yw;
    std::vector<std::vector<std::pair<uint8_t, uint8_t>>> of_texel(T), of_weight(W);
    for (unsigned y = 0; y < Y; y++)
        for (unsigned x = 0; x < X; x++) {
            const unsigned t = y * X + x;
            const unsigned fx = (((1024 + X / 2) / (X - 1)) * x * (xw - 1) + 32) >> 6;
            const unsigned fy = (((1024 + Y / 2) / (Y - 1)) * y * (yw - 1) + 32) >> 6;
            const unsigned xf = fx & 15, yf = fy & 15, w00 = (fx >> 4) + (fy >> 4) * xw;
            const unsigned idx[4] = {w00, w00 + 1, w00 + xw, w00 + xw + 1};
            unsigned k[4];
            k[3] = (xf * yf + 8) >> 4; k[1] = xf - k[3]; k[2] = yf - k[3]; k[0] = 16 - xf - yf + k[3];
            for (int i = 0; i < 4; i++)
                if (k[i]) { of_texel[t].emplace_back(idx[i], k[i]); of_weight[idx[i]].emplace_back(t, k[i]); }
        }
    std::memset(d.tw_count, 0, sizeof(d.tw_count)); std::memset(d.tw_off, 0, sizeof(d.tw_off));
    std::memset(d.wt_count, 0, sizeof(d.wt_count)); std::memset(d.wt_off, 0, sizeof(d.wt_off));
    for (unsigned t = 0; t < T; t++) {
        d.tw_off[t] = (uint32_t)h.t2w_w.size(); d.tw_count[t] = (uint32_t)of_texel[t].size();
        for (auto& e : of_texel[t]) { h.t2w_w.push_back(e.first); h.t2w_k.push_back(e.second); }
    }
    for (unsigned w = 0; w < W; w++) {
        d.wt_off[w] = (uint32_t)h.w2t_t.size(); d.wt_count[w] = (uint32_t)of_weight[w].size();
        for (auto& e : of_weight[w]) { h.w2t_t.push_back(e.first); h.w2t_k.push_back(e.second); }
    }
    d.W = W; d.wx = xw; d.wy = yw;
}

uint32_t hash52(uint32_t v) {  // partition_tables.cpp:92-106
    v ^= v >> 15; v *= 0xEEDE0891; v ^= v >> 5; v += v << 16;
    v ^= v >> 7; v ^= v >> 3; v ^= v << 6; v ^= v >> 17;
    return v;
}

// ASTC partition-pattern function for 2D blocks (partition_tables.cpp:120-241).
int partition_of(int seed, int x, int y, int pc, bool small) {
    if (small) { x <<= 1; y <<= 1; }
    seed += (pc - 1) * 1024;
    const uint32_t r = hash52((uint32_t)seed);
    uint8_t s[12];
    const int shifts[12] = {0, 4, 8, 12, 16, 20, 24, 28, 18, 22, 26, 30};
    for (int i = 0; i < 12; i++) {
        uint32_t v = i == 11 ? ((r >> 30) | (r << 2)) : (r >> shifts[i]);
        s[i] = (uint8_t)((v & 0xF) * (v & 0xF));
    }
    int sh1, sh2;
    if (seed & 1) { sh1 = (seed & 2) ? 4 : 5; sh2 = pc == 3 ? 6 : 5; }
    else { sh1 = pc == 3 ? 6 : 5; sh2 = (seed & 2) ? 4 : 5; }
    const int sh3 = (seed & 0x10) ? sh1 : sh2;
    for (int i = 0; i < 8; i++) s[i] >>= (i & 1) ? sh2 : sh1;
    for (int i = 8; i < 12; i++) s[i] >>= sh3;
    int a = (s[0] * x + s[1] * y + (r >> 14)) & 0x3F;   // z = 0 for 2D blocks
    int b = (s[2] * x + s[3] * y + (r >> 10)) & 0x3F;
    int c = (s[4] * x + s[5] * y + (r >> 6)) & 0x3F;
    int d = (s[6] * x + s[7] * y + (r >> 2)) & 0x3F;
    if (pc <= 3) d = 0;
    if (pc <= 2) c = 0;
    if (pc <= 1) b = 0;
    if (a >= b && a >= c && a >= d) return 0;
    if (b >= c && b >= d) return 1;
    return c >= d ? 2 : 3;
}

std::unique_ptr<HostTables> make_host_tables(int bx, int by) {
    std::unique_ptr<HostTables> hp(new HostTables());
    HostTables& h = *hp;
    h.bx = bx; h.by = by; h.T = bx * by;
    const int T = h.T;
    // block modes and decimation modes, in block-mode order
    int grid_dm[16 * 16];
    for (int& g : grid_dm) g = -1;
    for (unsigned m = 0; m < 2048; m++) {
        ModeDecode md;
        if (!decode_mode(m, md) || md.xw > (unsigned)bx || md.yw > (unsigned)by ||
            (int)((md.dual ? 109 : 111) - md.weight_bits) <= 0) { h.bm_index[m] = 0xFFFF; continue; }
        int& dm = grid_dm[md.yw * 16 + md.xw];
        if (dm < 0) {
            HostTables::Dm d;
            add_grid(h, md.xw, md.yw, d);
            int p1 = -1, p2 = -1;
            for (int q = 0; q < 12; q++) {
                const unsigned b1 = ise_bits(d.W, q), b2 = ise_bits(2 * d.W, q);
                if (b1 >= 24 && b1 <= 96) p1 = q;
                if (2 * d.W <= 64 && b2 >= 24 && b2 <= 96) p2 = q;
            }
            d.maxprec1 = (uint32_t)p1; d.maxprec2 = (uint32_t)p2; d.ref1 = d.ref2 = 0;
            const int mp = p1 < 0 ? -1 : std::min(p1, 7);  // angular quant cap QUANT_12 (astc.h:146,152)
            d.maxq = mp < 0 ? 0 : mp;
            d.steps = d.qsteps = mp < 0 ? 0 : kStepsForQuant[mp];
            dm = (int)h.dms.size();
            h.dms.push_back(d);
        }
        if (md.dual) h.dms[dm].ref2 |= 1u << md.quant; else h.dms[dm].ref1 |= 1u << md.quant;
        h.bm_index[m] = (uint32_t)h.bms.size();
        h.bms.push_back({m, (uint32_t)dm, md.quant, md.weight_bits, md.dual ? 1u : 0u});
    }
    // k-means texel subset (metadata_structures.cpp:33-70)
    std::memset(h.kmeans, 0, sizeof(h.kmeans));
    if (T <= 64) { for (int i = 0; i < T; i++) h.kmeans[i] = i; }
    else {
        uint64_t s0 = 0xfaf9e171cea1ec6bULL, s1 = 0xf1b318cc06af5d71ULL;
        bool seen[kMaxTexels] = {};
        for (int n = 0; n < 64;) {
            const uint64_t res = s0 + s1, x = s1 ^ s0;
            s0 = ((s0 << 24) | (s0 >> 40)) ^ x ^ (x << 16);
            s1 = (x << 37) | (x >> 27);
            const int t = (uint8_t)res % T;
            if (!seen[t]) { seen[t] = true; h.kmeans[n++] = t; }
        }
    }
    // partition tables: selected (valid, canonically distinct) entries first
    h.parts.assign(3 * 1024 + 1, HostTables::Part());
    std::memset(h.packed_index, 0, sizeof(h.packed_index));
    const bool small = T < 32;
    auto make_part = [&](int pc, int seed, HostTables::Part& p) {
        std::memset(&p, 0, sizeof(p));
        int n = 0;
        for (int y = 0; y < by; y++)
            for (int x = 0; x < bx; x++) { int q = partition_of(seed, x, y, pc, small); p.of[n++] = (uint8_t)q; p.tcount[q]++; }
        p.count = !p.tcount[0] ? 0 : !p.tcount[1] ? 1 : !p.tcount[2] ? 2 : !p.tcount[3] ? 3 : 4;
        p.seed = seed;
    };
    make_part(1, 0, h.parts[3 * 1024]);
    h.sel[0] = h.all[0] = 1;
    for (int pc = 2; pc <= 4; pc++) {
        HostTables::Part* tab = &h.parts[(pc - 2) * 1024];
        // Canonical pattern of the first 32 texels only: the reference's dedupe
        // compares one 64-bit word (partition_tables.cpp:59-83).
        auto canon32 = [&](const HostTables::Part& p) {
            int map[4] = {-1, -1, -1, -1}, next = 0;
            uint64_t w = 0;
            for (int t = 0; t < std::min(T, 32); t++) {
                if (map[p.of[t]] < 0) map[p.of[t]] = next++;
                w |= (uint64_t)map[p.of[t]] << (2 * t);
            }
            return w;
        };
        std::vector<uint64_t> pattern;
        std::vector<uint8_t> taken(1024, 0);
        h.sel[pc - 1] = h.all[pc - 1] = 0;
        for (int pass = 0; pass < 2; pass++)
            for (int seed = 0; seed < 1024; seed++) {
                if (pass == 1 && taken[seed]) continue;
                HostTables::Part p; make_part(pc, seed, p);
                const bool useful = (int)p.count == pc;
                if (pass == 0 && !useful) continue;
                const uint64_t c = canon32(p);
                const bool dup = std::find(pattern.begin(), pattern.end(), c) != pattern.end();
                if (pass == 0 && dup) continue;
                const unsigned at = (unsigned)pattern.size();
                pattern.push_back(c);
                tab[at] = p;
                h.packed_index[pc - 2][seed] = (uint16_t)at;
                if (pass == 0) { taken[seed] = 1; h.sel[pc - 1]++; }
                h.all[pc - 1]++;
            }
        h.cov[pc].assign((size_t)1024 * pc, 0);
        for (int e = 0; e < 1024; e++)
            for (int i = 0; i < std::min(T, 64); i++) h.cov[pc][(size_t)e * pc + tab[e].of[h.kmeans[i]]] |= 1ULL << i;
    }
    // trial modes: decimation modes used by a single-plane mode up to QUANT_12,
    // then single-plane block modes on those (compression_pipeline.cpp:146-198)
    std::vector<uint32_t> lookup(h.dms.size(), 0xFFFF);
    for (uint32_t d = 0; d < h.dms.size(); d++)
        if (h.dms[d].ref1 & 0xFF) { lookup[d] = (uint32_t)h.valid_dms.size(); h.valid_dms.push_back(d); }
    for (uint32_t m = 0; m < 2048; m++) {
        const uint32_t b = h.bm_index[m];
        if (b == 0xFFFF || h.bms[b].dual || lookup[h.bms[b].dm] == 0xFFFF) continue;
        h.valid_bms.emplace_back(b, lookup[h.bms[b].dm]);
    }
    // sin / cos of (2 pi / 1023) * (i+1) * j (metadata_structures.cpp:463-481)
    h.sin_t.resize(1024 * 16); h.cos_t.resize(1024 * 16);
    const float pi = 3.14159265358979323846f;
    for (unsigned i = 0; i < 16; i++)
        for (unsigned j = 0; j < 1024; j++) {
            const float a = (2.0f * pi / 1023.0f) * (float)(i + 1) * (float)j;
            h.sin_t[j * 16 + i] = std::sin(a);
            h.cos_t[j * 16 + i] = std::cos(a);
        }
    return hp;
}

template <class T>
uint32_t put(std::vector<uint8_t>& blob, const T* data, size_t n) {
    size_t off = (blob.size() + 15) & ~size_t(15);
    blob.resize(off + n * sizeof(T));
    if (n) std::memcpy(blob.data() + off, data, n * sizeof(T));
    return (uint32_t)off;
}

}  // namespace

bool valid_footprint(int bx, int by) {
    static const int v[14][2] = {{4, 4}, {5, 4}, {5, 5}, {6, 5}, {6, 6}, {8, 5}, {8, 6},
                                 {10, 5}, {10, 6}, {8, 8}, {10, 8}, {10, 10}, {12, 10}, {12, 12}};
    for (auto& p : v) if (p[0] == bx && p[1] == by) return true;
    return false;
}

const HostTables* host_tables(int bx, int by) {
    if (!valid_footprint(bx, by)) return nullptr;
    static std::mutex mu;
    static std::map<int, std::unique_ptr<HostTables>> cache;
    std::lock_guard<std::mutex> g(mu);
    auto& slot = cache[bx * 256 + by];
    if (!slot) slot = make_host_tables(bx, by);
    return slot.get();
}

bool build_tables(int bx, int by, TableLayout& L, std::vector<uint8_t>& blob) {
    const HostTables* hp = host_tables(bx, by);
    if (!hp) return false;
    const HostTables& h = *hp;
    const ConstTables& c = const_tables();
    // the refinement's endpoint quantisation search relies on each level's colour table
    // being non-decreasing in its index (true by construction: nearest values of idx / 2)
    for (int k = 0; k < 17; k++)
        for (int i = 1; i < 512; i++)
            if (c.cu2u[k][i] < c.cu2u[k][i - 1]) return false;
    std::memset(&L, 0, sizeof(L));
    blob.clear();
    L.bx = bx; L.by = by; L.T = h.T;
    L.ndm = (int)h.valid_dms.size(); L.nbm = (int)h.valid_bms.size();
    for (int i = 0; i < 4; i++) L.count_selected[i] = h.sel[i];
    std::memcpy(L.kmeans, h.kmeans, sizeof(L.kmeans));
    const int T = h.T, ndm = L.ndm;
    std::vector<DevDm> dms(ndm);
    std::vector<uint8_t> twc((size_t)ndm * T, 0), wtc((size_t)ndm * 64, 0);
    std::vector<uint16_t> tws((size_t)ndm * T, 0), wts((size_t)ndm * 64, 0), t2w, w2t;
    for (int m = 0; m < ndm; m++) {
        const HostTables::Dm& d = h.dms[h.valid_dms[m]];
        DevDm& o = dms[m];
        o.W = (uint8_t)d.W; o.wx = (uint8_t)d.wx; o.wy = (uint8_t)d.wy; o.max_quant_level = (uint8_t)d.maxq;
        o.max_angular_steps = (uint8_t)d.steps; o.max_quant_steps = (uint8_t)d.qsteps; o.pad0 = o.pad1 = 0;
        o.tw_base = (uint16_t)t2w.size(); o.wt_base = (uint16_t)w2t.size();
        for (int t = 0; t < T; t++) {
            twc[(size_t)m * T + t] = (uint8_t)d.tw_count[t];
            tws[(size_t)m * T + t] = (uint16_t)(t2w.size() - o.tw_base);
            for (uint32_t j = 0; j < d.tw_count[t]; j++) {
                const uint32_t e = d.tw_off[t] + j;
                t2w.push_back((uint16_t)(h.t2w_w[e] | (h.t2w_k[e] << 8)));
            }
        }
        for (uint32_t w = 0; w < d.W; w++) {
            wtc[(size_t)m * 64 + w] = (uint8_t)d.wt_count[w];
            wts[(size_t)m * 64 + w] = (uint16_t)(w2t.size() - o.wt_base);
            for (uint32_t j = 0; j < d.wt_count[w]; j++) {
                const uint32_t e = d.wt_off[w] + j;
                w2t.push_back((uint16_t)(h.w2t_t[e] | (h.w2t_k[e] << 8)));
            }
        }
    }
    std::vector<uint64_t> tw4((size_t)ndm * T, 0);
    for (int m = 0; m < ndm; m++)
        for (int t = 0; t < T; t++) {
            uint64_t v = 0;
            const int n = twc[(size_t)m * T + t], base = dms[m].tw_base + tws[(size_t)m * T + t];
            for (int j = 0; j < n; j++) v |= (uint64_t)t2w[base + j] << (16 * j);
            tw4[(size_t)m * T + t] = v;
        }
    L.max_w = 0;
    for (int m = 0; m < ndm; m++) L.max_w = std::max<int>(L.max_w, dms[m].W);
    std::vector<DevBm> bms(L.nbm);
    for (int i = 0; i < L.nbm; i++) {
        const HostTables::Bm& b = h.bms[h.valid_bms[i].first];
        bms[i] = DevBm{(uint16_t)b.mode, (uint8_t)h.valid_bms[i].second, (uint8_t)b.quant, (uint8_t)b.bits, {0, 0, 0}};
    }
    std::vector<uint8_t> ptex((size_t)3 * 1024 * T), pcnt((size_t)3 * 1024 * 4);
    std::vector<uint32_t> pinfo(3 * 1024);
    std::vector<uint64_t> cov((size_t)3 * 1024 * 4, 0);
    for (int pc = 2; pc <= 4; pc++)
        for (int e = 0; e < 1024; e++) {
            const HostTables::Part& p = h.parts[(pc - 2) * 1024 + e];
            const size_t k = (size_t)(pc - 2) * 1024 + e;
            std::memcpy(&ptex[k * T], p.of, T);
            for (int q = 0; q < 4; q++) pcnt[k * 4 + q] = (uint8_t)p.tcount[q];
            pinfo[k] = p.seed;
            for (int q = 0; q < pc; q++) cov[k * 4 + q] = h.cov[pc][(size_t)e * pc + q];
        }
    std::vector<DevBm> dual;  // dual-plane block modes whose grid is a trial decimation mode
    {
        std::vector<uint32_t> lookup(h.dms.size(), 0xFFFF);
        for (uint32_t d = 0; d < h.valid_dms.size(); d++) lookup[h.valid_dms[d]] = d;
        for (const HostTables::Bm& b : h.bms)
            if (b.dual && lookup[b.dm] != 0xFFFF)
                dual.push_back(DevBm{(uint16_t)b.mode, (uint8_t)lookup[b.dm], (uint8_t)b.quant, (uint8_t)b.bits, {0, 0, 0}});
    }
    L.ndual = (int)dual.size();
    std::vector<uint16_t> order(L.nbm);
    for (int i = 0; i < L.nbm; i++) order[i] = (uint16_t)i;
    std::stable_sort(order.begin(), order.end(), [&](uint16_t x, uint16_t y) { return bms[x].dm < bms[y].dm; });
    L.off_dm = put(blob, dms.data(), dms.size());
    L.off_bm = put(blob, bms.data(), bms.size());
    L.off_tw_count = put(blob, twc.data(), twc.size());
    L.off_tw_start = put(blob, tws.data(), tws.size());
    L.off_wt_count = put(blob, wtc.data(), wtc.size());
    L.off_wt_start = put(blob, wts.data(), wts.size());
    L.off_t2w = put(blob, t2w.data(), t2w.size());
    L.off_w2t = put(blob, w2t.data(), w2t.size());
    L.off_tw4 = put(blob, tw4.data(), tw4.size());
    L.off_bm_order = put(blob, order.data(), order.size());
    L.off_dual = put(blob, dual.data(), dual.size());
    L.off_part_texel = put(blob, ptex.data(), ptex.size());
    L.off_part_info = put(blob, pinfo.data(), pinfo.size());
    L.off_part_counts = put(blob, pcnt.data(), pcnt.size());
    L.off_cov = put(blob, cov.data(), cov.size());
    L.off_sin = put(blob, h.sin_t.data(), h.sin_t.size());
    L.off_cos = put(blob, h.cos_t.data(), h.cos_t.size());
    L.off_q2u = put(blob, c.q2u, 142);
    L.off_q2u_start = put(blob, c.q2u_start, 12);
    L.off_qmt = put(blob, &c.qmt[0][0], 1280);
    L.off_cu2u = put(blob, &c.cu2u[0][0], 17 * 512);
    L.off_prev_next = put(blob, &c.prev_next[0][0], 12 * 65);
    L.off_bqe = put(blob, c.bqe, 17);
    L.off_wscr = put(blob, &c.wscr[0][0], 12 * 32);
    L.off_cscr = put(blob, &c.cscr[0][0], 17 * 256);
    L.off_trits = put(blob, c.trits, 243);
    L.off_quints = put(blob, c.quints, 125);
    blob.resize((blob.size() + 15) & ~size_t(15));
    L.total_bytes = (uint32_t)blob.size();
    return true;
}

}  // namespace astcb200

// ------------------------------------------------------------ table dumps (C ABI, tests only)
using astcb200::HostTables;

extern "C" {

int astcb200_tables_counts(int bx, int by, uint32_t* c) {
    const HostTables* h = astcb200::host_tables(bx, by);
    if (!h) return -1;
    size_t nt = h->t2w_w.size(), nw = h->w2t_t.size();
    c[0] = h->T; c[1] = (uint32_t)h->bms.size(); c[2] = (uint32_t)h->dms.size(); c[3] = (uint32_t)nt; c[4] = (uint32_t)nw;
    for (int i = 0; i < 4; i++) { c[5 + i] = h->sel[i]; c[9 + i] = h->all[i]; }
    return 0;
}
int astcb200_tables_block_modes(int bx, int by, uint32_t* bm_index, uint32_t* bms) {
    const HostTables* h = astcb200::host_tables(bx, by);
    if (!h) return -1;
    std::memcpy(bm_index, h->bm_index, sizeof(h->bm_index));
    for (size_t i = 0; i < h->bms.size(); i++) {
        const auto& b = h->bms[i];
        uint32_t* o = bms + i * 5; o[0] = b.mode; o[1] = b.dm; o[2] = b.quant; o[3] = b.bits; o[4] = b.dual;
    }
    return 0;
}
int astcb200_tables_decimation(int bx, int by, uint32_t* dmodes, uint32_t* dinfo) {
    const HostTables* h = astcb200::host_tables(bx, by);
    if (!h) return -1;
    for (size_t i = 0; i < h->dms.size(); i++) {
        const auto& d = h->dms[i];
        dmodes[i * 4] = d.maxprec1; dmodes[i * 4 + 1] = d.maxprec2; dmodes[i * 4 + 2] = d.ref1; dmodes[i * 4 + 3] = d.ref2;
        uint32_t* o = dinfo + i * 424;
        o[0] = h->T; o[1] = d.W; o[2] = d.wx; o[3] = d.wy; o[4] = d.maxq; o[5] = d.steps; o[6] = d.qsteps; o[7] = 0;
        for (int t = 0; t < 144; t++) { o[8 + t] = d.tw_count[t]; o[152 + t] = d.tw_off[t]; }
        for (int w = 0; w < 64; w++) { o[296 + w] = d.wt_count[w]; o[360 + w] = d.wt_off[w]; }
    }
    return 0;
}
int astcb200_tables_maps(int bx, int by, uint32_t* ti, float* tc, uint32_t* wi, float* wc) {
    const HostTables* h = astcb200::host_tables(bx, by);
    if (!h) return -1;
    for (size_t i = 0; i < h->t2w_w.size(); i++) { ti[i] = h->t2w_w[i]; tc[i] = (float)h->t2w_k[i] * (1.0f / 16.0f); }
    for (size_t i = 0; i < h->w2t_t.size(); i++) { wi[i] = h->w2t_t[i]; wc[i] = (float)h->w2t_k[i] * (1.0f / 16.0f); }
    return 0;
}
int astcb200_tables_partitions(int bx, int by, uint32_t* pinfo, uint64_t* cov2, uint64_t* cov3, uint64_t* cov4,
                               uint32_t* km, uint16_t* pidx) {
    const HostTables* h = astcb200::host_tables(bx, by);
    if (!h) return -1;
    for (int i = 0; i < 3073; i++) {
        const auto& p = h->parts[i];
        uint32_t* o = pinfo + (size_t)i * 150;
        o[0] = p.count; o[1] = p.seed;
        for (int k = 0; k < 4; k++) o[2 + k] = p.tcount[k];
        for (int t = 0; t < 144; t++) o[6 + t] = t < h->T ? p.of[t] : 0;
    }
    std::memcpy(cov2, h->cov[2].data(), 1024 * 2 * 8);
    std::memcpy(cov3, h->cov[3].data(), 1024 * 3 * 8);
    std::memcpy(cov4, h->cov[4].data(), 1024 * 4 * 8);
    std::memcpy(km, h->kmeans, sizeof(h->kmeans));
    std::memcpy(pidx, h->packed_index, sizeof(h->packed_index));
    return 0;
}
// Block mode (11-bit ASTC mode) of every trial block mode, in trial order.
int astcb200_tables_trial_modes(int bx, int by, uint32_t* n_bm, uint16_t* mode_index) {
    const HostTables* h = astcb200::host_tables(bx, by);
    if (!h || !n_bm) return -1;
    *n_bm = (uint32_t)h->valid_bms.size();
    if (mode_index)
        for (size_t i = 0; i < h->valid_bms.size(); i++) mode_index[i] = (uint16_t)h->bms[h->valid_bms[i].first].mode;
    return 0;
}
int astcb200_tables_angular(float* s, float* c) {
    const HostTables* h = astcb200::host_tables(4, 4);
    std::memcpy(s, h->sin_t.data(), 16384 * 4);
    std::memcpy(c, h->cos_t.data(), 16384 * 4);
    return 16384;
}

}  // extern "C"
