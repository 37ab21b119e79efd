// ASTC LDR block decoding, written from the ASTC specification, shared by the host
// decoder (decoder.cpp) and the device decoder (decoder_gpu.cu) so that both produce
// the same texels.  A block is parsed once (parse_block: block mode, partitioning,
// endpoint formats, integer-sequence-encoded colour values and weights, unquantised)
// and then any texel of it can be evaluated (texel16: weight infill, endpoint
// interpolation, 16-bit result; to_unorm8 gives the 8-bit texel).  Blocks that are
// not valid LDR blocks (reserved modes, HDR endpoints, too many colour values) decode
// to the error colour (magenta, opaque).
#pragma once
#include <stdint.h>

#ifdef __CUDACC__
#define ASTC_HD __host__ __device__ __forceinline__
// The unquantisation functions stay out of line in device code: inlined into
// parse_block, the optimised device build decoded some weights wrongly (found by the
// device-against-host decoder tests; the debug build and the out-of-line build agree
// with the host on every block).
#define ASTC_HD_CALL static __host__ __device__ __noinline__
#else
#define ASTC_HD inline
#define ASTC_HD_CALL inline
#endif

namespace astcb200 {
namespace dec {

struct Bits {
    const uint8_t* p;
    ASTC_HD uint32_t get(int off, int n) const {
        uint32_t v = 0;
        for (int i = 0; i < n; i++) v |= (uint32_t)((p[(off + i) >> 3] >> ((off + i) & 7)) & 1) << i;
        return v;
    }
};

ASTC_HD int level_count(int q) {
    const int L[21] = {2, 3, 4, 5, 6, 8, 10, 12, 16, 20, 24, 32, 40, 48, 64, 80, 96, 128, 160, 192, 256};
    return L[q];
}
// bits, trits, quints of quantisation method q
ASTC_HD void btq(int q, int& bits, int& trits, int& quints) {
    int L = level_count(q);
    trits = quints = 0;
    if (L % 3 == 0) { trits = 1; L /= 3; } else if (L % 5 == 0) { quints = 1; L /= 5; }
    bits = 0;
    while ((1 << bits) < L) bits++;
}
ASTC_HD int ise_bits(int n, int q) {
    int b, t, qu;
    btq(q, b, t, qu);
    if (t) return (n * (8 + 5 * b) + 4) / 5;
    if (qu) return (n * (7 + 3 * b) + 2) / 3;
    return n * b;
}
ASTC_HD int bit_of(int x, int i) { return (x >> i) & 1; }
// the five trits packed in the 8-bit value T
ASTC_HD void trit_digits(int T, int t[5]) {
    int C;
    if (((T >> 2) & 7) == 7) { C = (((T >> 5) & 7) << 2) | (T & 3); t[4] = 2; t[3] = 2; }
    else {
        C = T & 31;
        if (((T >> 5) & 3) == 3) { t[4] = 2; t[3] = bit_of(T, 7); } else { t[4] = bit_of(T, 7); t[3] = (T >> 5) & 3; }
    }
    if ((C & 3) == 3) { t[2] = 2; t[1] = bit_of(C, 4); t[0] = (bit_of(C, 3) << 1) | (bit_of(C, 2) & ~bit_of(C, 3) & 1); }
    else if (((C >> 2) & 3) == 3) { t[2] = 2; t[1] = 2; t[0] = C & 3; }
    else { t[2] = bit_of(C, 4); t[1] = (C >> 2) & 3; t[0] = (bit_of(C, 1) << 1) | (bit_of(C, 0) & ~bit_of(C, 1) & 1); }
}
// the three quints packed in the 7-bit value Q
ASTC_HD void quint_digits(int Q, int q[3]) {
    if (((Q >> 1) & 3) == 3 && ((Q >> 5) & 3) == 0) {
        const int b0 = bit_of(Q, 0);
        q[2] = (b0 << 2) | ((bit_of(Q, 4) & (1 - b0)) << 1) | (bit_of(Q, 3) & (1 - b0));
        q[1] = 4; q[0] = 4;
        return;
    }
    int C;
    if (((Q >> 1) & 3) == 3) { q[2] = 4; C = (((Q >> 3) & 3) << 3) | (((~Q >> 5) & 3) << 1) | (Q & 1); }
    else { q[2] = (Q >> 5) & 3; C = Q & 31; }
    if ((C & 7) == 5) { q[1] = 4; q[0] = (C >> 3) & 3; } else { q[1] = (C >> 3) & 3; q[0] = C & 7; }
}
// Integer-sequence decode of n values of method q starting at bit `off`.
ASTC_HD void decode_ise(const Bits& b, int off, int n, int q, int* out) {
    int bits, trits, quints;
    btq(q, bits, trits, quints);
    if (trits) {
        for (int i = 0; i < n; i += 5) {
            int m[5] = {0, 0, 0, 0, 0}, T = 0, sh = 0;
            for (int e = 0; e < 5 && i + e < n; e++) {  // absent digits of a partial group read as 0
                const int tb = (e == 2 || e == 4) ? 1 : 2;
                m[e] = (int)b.get(off, bits); off += bits;
                T |= (int)b.get(off, tb) << sh; off += tb; sh += tb;
            }
            int d[5];
            trit_digits(T, d);
            for (int e = 0; e < 5 && i + e < n; e++) out[i + e] = (d[e] << bits) | m[e];
        }
    } else if (quints) {
        for (int i = 0; i < n; i += 3) {
            int m[3] = {0, 0, 0}, Q = 0, sh = 0;
            for (int e = 0; e < 3 && i + e < n; e++) {
                const int qb = e == 0 ? 3 : 2;
                m[e] = (int)b.get(off, bits); off += bits;
                Q |= (int)b.get(off, qb) << sh; off += qb; sh += qb;
            }
            int d[3];
            quint_digits(Q, d);
            for (int e = 0; e < 3 && i + e < n; e++) out[i + e] = (d[e] << bits) | m[e];
        }
    } else {
        for (int i = 0; i < n; i++) { out[i] = (int)b.get(off, bits); off += bits; }
    }
}
// v (bits bits, 1..8) repeated from the top until width bits are filled.  The loop has a
// fixed bound: an unbounded one (endless for bits = 0, which never occurs) lets a compiler
// draw conclusions about callers that miscompile the weight and colour unquantisation.
ASTC_HD int replicate(int v, int bits, int width) {
    if (bits <= 0) return 0;
    int out = 0, have = 0;
    for (int i = 0; i < 8 && have < width; i++) { out = (out << bits) | v; have += bits; }
    return out >> (have - width);
}
ASTC_HD_CALL int unq_color(int q, int v) {
    int bits, trits, quints;
    btq(q, bits, trits, quints);
    if (!trits && !quints) return replicate(v, bits, 8);
    const int D = v >> bits, m = v & ((1 << bits) - 1), A = (m & 1) ? 0x1FF : 0;
    // C of trits (bits 0..6) and of quints (bits 0..5) in one table (see unq_weight)
    const int kC[13] = {0, 204, 93, 44, 22, 11, 5, 0, 113, 54, 26, 13, 6};
    const int C = kC[trits ? bits : 7 + bits];
    int B = 0;
    if (trits) {
        if (bits == 2) B = bit_of(m, 1) * 0x116;
        else if (bits == 3) B = bit_of(m, 2) * 0x10A + bit_of(m, 1) * 0x85;
        else if (bits == 4) B = bit_of(m, 3) * 0x104 + bit_of(m, 2) * 0x82 + bit_of(m, 1) * 0x41;
        else if (bits == 5) B = bit_of(m, 4) * 0x102 + bit_of(m, 3) * 0x81 + bit_of(m, 2) * 0x40 + bit_of(m, 1) * 0x20;
        else if (bits == 6) B = bit_of(m, 5) * 0x101 + bit_of(m, 4) * 0x80 + bit_of(m, 3) * 0x40 + bit_of(m, 2) * 0x20 + bit_of(m, 1) * 0x10;
    } else {
        if (bits == 2) B = bit_of(m, 1) * 0x10C;
        else if (bits == 3) B = bit_of(m, 2) * 0x105 + bit_of(m, 1) * 0x82;
        else if (bits == 4) B = bit_of(m, 3) * 0x102 + bit_of(m, 2) * 0x81 + bit_of(m, 1) * 0x40;
        else if (bits == 5) B = bit_of(m, 4) * 0x101 + bit_of(m, 3) * 0x80 + bit_of(m, 2) * 0x40 + bit_of(m, 1) * 0x20;
    }
    return (A & 0x80) | (((D * C + B) ^ A) >> 2);
}
ASTC_HD_CALL int unq_weight(int q, int v) {
    int bits, trits, quints;
    btq(q, bits, trits, quints);
    int r;
    if (!trits && !quints) r = replicate(v, bits, 6);
    else {
        const int D = v >> bits, m = v & ((1 << bits) - 1), A = (m & 1) ? 0x7F : 0, b1 = (m >> 1) & 1, b2 = (m >> 2) & 1;
        if (bits == 0) {
            // trits {0, 32, 63}, quints {0, 16, 32, 47, 63}: one table, so that no index of
            // either can run past its array (an out-of-range read, even on the branch not
            // taken, lets a compiler assume the index is small and decode wrong values)
            const int tq[8] = {0, 32, 63, 0, 16, 32, 47, 63};
            r = tq[trits ? D : 3 + D];
        } else {
            int B, C;
            if (trits) { C = bits == 1 ? 50 : bits == 2 ? 23 : 11; B = bits == 1 ? 0 : bits == 2 ? b1 * 0x45 : b2 * 0x42 + b1 * 0x21; }
            else { C = bits == 1 ? 28 : 13; B = bits == 1 ? 0 : b1 * 0x42; }
            r = (A & 0x20) | (((D * C + B) ^ A) >> 2);
        }
    }
    return r > 32 ? r + 1 : r;
}
struct Mode { int xw, yw, q; bool dual; };
// Weight grid, weight quantisation and dual-plane flag of the 11-bit block mode m;
// false for reserved modes and grids whose weights do not fit the spec's limits.
ASTC_HD bool decode_mode(int m, Mode& o) {
    int q = (m >> 4) & 1, H = (m >> 9) & 1, D = (m >> 10) & 1;
    const int A = (m >> 5) & 3;
    if (m & 3) {
        q |= (m & 3) << 1;
        int B = (m >> 7) & 3;
        switch ((m >> 2) & 3) {
            case 0: o.xw = B + 4; o.yw = A + 2; break;
            case 1: o.xw = B + 8; o.yw = A + 2; break;
            case 2: o.xw = A + 2; o.yw = B + 8; break;
            default: B &= 1; if (m & 0x100) { o.xw = B + 2; o.yw = A + 2; } else { o.xw = A + 2; o.yw = B + 6; }
        }
    } else {
        q |= ((m >> 2) & 3) << 1;
        if (((m >> 2) & 3) == 0) return false;
        const int B = (m >> 9) & 3;
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
    o.q = (q - 2) + 6 * H;
    o.dual = D != 0;
    const int n = o.xw * o.yw * (D + 1);
    return n <= 64 && ise_bits(n, o.q) >= 24 && ise_bits(n, o.q) <= 96;
}
ASTC_HD uint32_t hash52(uint32_t v) {
    v ^= v >> 15; v *= 0xEEDE0891u; v ^= v >> 5; v += v << 16;
    v ^= v >> 7; v ^= v >> 3; v ^= v << 6; v ^= v >> 17;
    return v;
}
// Partition of texel (x, y) for partitioning `seed` of pc partitions.
ASTC_HD int select_partition(int seed, int x, int y, int pc, bool small) {
    if (small) { x <<= 1; y <<= 1; }
    seed += (pc - 1) * 1024;
    const uint32_t r = hash52((uint32_t)seed);
    uint32_t s[8];
    for (int i = 0; i < 8; i++) { const uint32_t v = (r >> (4 * i)) & 0xF; s[i] = v * v; }
    int sh1, sh2;
    if (seed & 1) { sh1 = (seed & 2) ? 4 : 5; sh2 = pc == 3 ? 6 : 5; } else { sh1 = pc == 3 ? 6 : 5; sh2 = (seed & 2) ? 4 : 5; }
    for (int i = 0; i < 8; i++) s[i] >>= (i & 1) ? sh2 : sh1;
    int a = (int)((s[0] * x + s[1] * y + (r >> 14)) & 0x3F), b = (int)((s[2] * x + s[3] * y + (r >> 10)) & 0x3F);
    int c = (int)((s[4] * x + s[5] * y + (r >> 6)) & 0x3F), d = (int)((s[6] * x + s[7] * y + (r >> 2)) & 0x3F);
    if (pc <= 3) d = 0;
    if (pc <= 2) c = 0;
    if (pc <= 1) b = 0;
    if (a >= b && a >= c && a >= d) return 0;
    if (b >= c && b >= d) return 1;
    return c >= d ? 2 : 3;
}
ASTC_HD void bts(int& a, int& b) {  // bit_transfer_signed(a, b)
    b >>= 1; b |= a & 0x80; a >>= 1; a &= 0x3F;
    if (a & 0x20) a -= 0x40;
}
ASTC_HD int c255(int v) { return v < 0 ? 0 : v > 255 ? 255 : v; }
ASTC_HD void set4(int* e, int r, int g, int b, int a) { e[0] = r; e[1] = g; e[2] = b; e[3] = a; }
ASTC_HD void blue_contract(int* e) { e[0] = (e[0] + e[2]) >> 1; e[1] = (e[1] + e[2]) >> 1; }
// LDR endpoint decode of colour endpoint mode cem; false for HDR modes.
ASTC_HD bool decode_endpoints(int cem, const int* v, int* e0, int* e1) {
    switch (cem) {
        case 0: set4(e0, v[0], v[0], v[0], 255); set4(e1, v[1], v[1], v[1], 255); return true;
        case 1: {
            const int l0 = (v[0] >> 2) | (v[1] & 0xC0), l1 = c255(l0 + (v[1] & 0x3F));
            set4(e0, l0, l0, l0, 255); set4(e1, l1, l1, l1, 255);
            return true;
        }
        case 4: set4(e0, v[0], v[0], v[0], v[2]); set4(e1, v[1], v[1], v[1], v[3]); return true;
        case 5: {
            int a0 = v[0], b0 = v[1], a1 = v[2], b1 = v[3];
            bts(b0, a0); bts(b1, a1);
            set4(e0, a0, a0, a0, a1);
            set4(e1, c255(a0 + b0), c255(a0 + b0), c255(a0 + b0), c255(a1 + b1));
            return true;
        }
        case 6: set4(e0, (v[0] * v[3]) >> 8, (v[1] * v[3]) >> 8, (v[2] * v[3]) >> 8, 255); set4(e1, v[0], v[1], v[2], 255); return true;
        case 8: case 12: {
            const int a0 = cem == 12 ? v[6] : 255, a1 = cem == 12 ? v[7] : 255;
            if (v[1] + v[3] + v[5] >= v[0] + v[2] + v[4]) { set4(e0, v[0], v[2], v[4], a0); set4(e1, v[1], v[3], v[5], a1); }
            else { set4(e0, v[1], v[3], v[5], a1); set4(e1, v[0], v[2], v[4], a0); blue_contract(e0); blue_contract(e1); }
            return true;
        }
        case 9: case 13: {
            int x[8];
            for (int i = 0; i < 8; i++) x[i] = v[i];
            bts(x[1], x[0]); bts(x[3], x[2]); bts(x[5], x[4]);
            if (cem == 13) bts(x[7], x[6]);
            const int a0 = cem == 13 ? x[6] : 255, a1 = cem == 13 ? x[6] + x[7] : 255;
            if (x[1] + x[3] + x[5] >= 0) { set4(e0, x[0], x[2], x[4], a0); set4(e1, x[0] + x[1], x[2] + x[3], x[4] + x[5], a1); }
            else { set4(e0, x[0] + x[1], x[2] + x[3], x[4] + x[5], a1); set4(e1, x[0], x[2], x[4], a0); blue_contract(e0); blue_contract(e1); }
            for (int i = 0; i < 4; i++) { e0[i] = c255(e0[i]); e1[i] = c255(e1[i]); }
            return true;
        }
        case 10: set4(e0, (v[0] * v[3]) >> 8, (v[1] * v[3]) >> 8, (v[2] * v[3]) >> 8, v[4]); set4(e1, v[0], v[1], v[2], v[5]); return true;
        default: return false;
    }
}

// A parsed block.  kind: 0 error (decodes to the error colour), 1 void extent (constant
// 16-bit colour vc), 2 a weighted block.
struct Block {
    int kind, xw, yw, dual, ccs, pc, seed;
    uint8_t e0[4][4], e1[4][4];  // endpoints per partition (0..255)
    uint8_t w[64];               // unquantised weights 0..64, planes interleaved when dual
    uint16_t vc[4];
};

ASTC_HD void parse_block(const uint8_t* blk, int bx, int by, Block& o) {
    const Bits b{blk};
    const int T = bx * by;
    o.kind = 0;
    const int mode = (int)b.get(0, 11);
    if ((mode & 0x1FF) == 0x1FC) {  // void extent
        if (mode & 0x200) return;    // HDR
        for (int i = 0; i < 4; i++) o.vc[i] = (uint16_t)b.get(64 + 16 * i, 16);
        o.kind = 1;
        return;
    }
    Mode m;
    if (!decode_mode(mode, m) || m.xw > bx || m.yw > by) return;
    const int pc = (int)b.get(11, 2) + 1;
    if (pc == 4 && m.dual) return;
    const int W = m.xw * m.yw, nw = W * (m.dual ? 2 : 1), wbits = ise_bits(nw, m.q);
    int cem[4] = {0, 0, 0, 0}, seed = 0, below = 128 - wbits, cstart;
    if (pc == 1) { cem[0] = (int)b.get(13, 4); cstart = 17; }
    else {
        seed = (int)b.get(13, 10);
        cstart = 29;
        const int low = (int)b.get(23, 6);
        if ((low & 3) == 0) { for (int i = 0; i < pc; i++) cem[i] = low >> 2; }
        else {
            const int hs = 3 * pc - 4;
            below -= hs;
            const int et = low | ((int)b.get(below, hs) << 6);
            const int base = (et & 3) - 1;
            for (int i = 0; i < pc; i++) cem[i] = ((base + ((et >> (2 + i)) & 1)) << 2) | ((et >> (2 + pc + 2 * i)) & 3);
        }
    }
    int ccs = -1;
    if (m.dual) { below -= 2; ccs = (int)b.get(below, 2); }
    int nv = 0;
    for (int i = 0; i < pc; i++) nv += 2 * (cem[i] >> 2) + 2;
    if (nv > 18) return;
    const int avail = below - cstart;
    int cq = -1;
    for (int q = 20; q >= 0; q--) if (ise_bits(nv, q) <= avail) { cq = q; break; }
    if (cq < 4) return;
    int cv[20], wv[64];
    decode_ise(b, cstart, nv, cq, cv);
    for (int i = 0; i < nv; i++) cv[i] = unq_color(cq, cv[i]);
    uint8_t rev[16];
    for (int i = 0; i < 16; i++) {
        int p = blk[15 - i];
        p = ((p & 0x0F) << 4) | ((p >> 4) & 0x0F); p = ((p & 0x33) << 2) | ((p >> 2) & 0x33); p = ((p & 0x55) << 1) | ((p >> 1) & 0x55);
        rev[i] = (uint8_t)p;
    }
    decode_ise(Bits{rev}, 0, nw, m.q, wv);
    for (int i = 0; i < nw; i++) o.w[i] = (uint8_t)unq_weight(m.q, wv[i]);
    int vo = 0;
    for (int i = 0; i < pc; i++) {
        int e0[4], e1[4];
        if (!decode_endpoints(cem[i], cv + vo, e0, e1)) return;
        for (int c = 0; c < 4; c++) { o.e0[i][c] = (uint8_t)e0[c]; o.e1[i][c] = (uint8_t)e1[c]; }
        vo += 2 * (cem[i] >> 2) + 2;
    }
    o.xw = m.xw; o.yw = m.yw; o.dual = m.dual ? 1 : 0; o.ccs = ccs; o.pc = pc; o.seed = seed;
    o.kind = 2;
    (void)T;
}

// The 16-bit texel (x, y) of a parsed block of footprint bx x by.
ASTC_HD void texel16(const Block& k, int bx, int by, int x, int y, uint16_t* out) {
    if (k.kind == 0) { out[0] = 0xFFFF; out[1] = 0; out[2] = 0xFFFF; out[3] = 0xFFFF; return; }
    if (k.kind == 1) { for (int c = 0; c < 4; c++) out[c] = k.vc[c]; return; }
    const int ds = (1024 + bx / 2) / (bx - 1), dt = (1024 + by / 2) / (by - 1);
    const int cs = ds * x, ct = dt * y;
    const int gs = (cs * (k.xw - 1) + 32) >> 6, gt = (ct * (k.yw - 1) + 32) >> 6;
    const int js = gs >> 4, fs = gs & 15, jt = gt >> 4, ft = gt & 15;
    const int w11 = (fs * ft + 8) >> 4, w10 = ft - w11, w01 = fs - w11, w00 = 16 - fs - ft + w11;
    const int v0 = js + jt * k.xw, W = k.xw * k.yw, np = k.dual ? 2 : 1;
    int wpl[2] = {0, 0};
    for (int pl = 0; pl < np; pl++) {
        const int g0 = v0 < W ? k.w[v0 * np + pl] : 0, g1 = v0 + 1 < W ? k.w[(v0 + 1) * np + pl] : 0;
        const int g2 = v0 + k.xw < W ? k.w[(v0 + k.xw) * np + pl] : 0, g3 = v0 + k.xw + 1 < W ? k.w[(v0 + k.xw + 1) * np + pl] : 0;
        wpl[pl] = (g0 * w00 + g1 * w01 + g2 * w10 + g3 * w11 + 8) >> 4;
    }
    const int part = k.pc > 1 ? select_partition(k.seed, x, y, k.pc, bx * by < 31) : 0;
    for (int c = 0; c < 4; c++) {
        const int w = (k.dual && c == k.ccs) ? wpl[1] : wpl[0];
        const int c0 = k.e0[part][c] * 257, c1 = k.e1[part][c] * 257;
        out[c] = (uint16_t)((c0 * (64 - w) + c1 * w + 32) >> 6);
    }
}

// 16-bit channel to 8-bit UNORM, rounded to nearest.
ASTC_HD uint8_t to_unorm8(uint32_t v) { return (uint8_t)((v * 255u + 32767u) / 65535u); }

}  // namespace dec
}  // namespace astcb200
