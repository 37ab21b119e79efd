// ASTC LDR block decoder (host), written from the ASTC specification.
// The reference has no decoder; this one measures quality (PSNR) and checks
// that every block the encoder emits decodes as the encoder intended.
#include <algorithm>
#include <cstdint>
#include <cstring>

#include "astcb200.h"
#include "tables.h"

namespace {

const int kLevels[21] = {2, 3, 4, 5, 6, 8, 10, 12, 16, 20, 24, 32, 40, 48, 64, 80, 96, 128, 160, 192, 256};

struct Bits {
    const uint8_t* p;
    uint32_t get(int off, int n) const {
        uint32_t v = 0;
        for (int i = 0; i < n; i++) v |= (uint32_t)((p[(off + i) >> 3] >> ((off + i) & 7)) & 1) << i;
        return v;
    }
};

void btq(int q, int& bits, int& trits, int& quints) {
    int L = kLevels[q];
    trits = quints = 0;
    if (L % 3 == 0) { trits = 1; L /= 3; } else if (L % 5 == 0) { quints = 1; L /= 5; }
    bits = 0;
    while ((1 << bits) < L) bits++;
}
int ise_bits(int n, int q) {
    int b, t, qu; btq(q, b, t, qu);
    if (t) return (n * (8 + 5 * b) + 4) / 5;
    if (qu) return (n * (7 + 3 * b) + 2) / 3;
    return n * b;
}
void trit_digits(int T, int t[5]) {
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
void quint_digits(int Q, int q[3]) {
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
// Integer-sequence decode of n values of method q starting at bit `off`.
void decode_ise(const Bits& b, int off, int n, int q, int* out) {
    int bits, trits, quints; btq(q, bits, trits, quints);
    if (trits) {
        static const int tb[5] = {2, 2, 1, 2, 1};
        for (int i = 0; i < n; i += 5) {
            int m[5] = {0, 0, 0, 0, 0}, T = 0, sh = 0;
            for (int e = 0; e < 5 && i + e < n; e++) {  // absent digits of a partial group read as 0
                m[e] = (int)b.get(off, bits); off += bits;
                T |= (int)b.get(off, tb[e]) << sh; off += tb[e]; sh += tb[e];
            }
            int d[5]; trit_digits(T, d);
            for (int e = 0; e < 5 && i + e < n; e++) out[i + e] = (d[e] << bits) | m[e];
        }
    } else if (quints) {
        static const int qb[3] = {3, 2, 2};
        for (int i = 0; i < n; i += 3) {
            int m[3] = {0, 0, 0}, Q = 0, sh = 0;
            for (int e = 0; e < 3 && i + e < n; e++) {
                m[e] = (int)b.get(off, bits); off += bits;
                Q |= (int)b.get(off, qb[e]) << sh; off += qb[e]; sh += qb[e];
            }
            int d[3]; quint_digits(Q, d);
            for (int e = 0; e < 3 && i + e < n; e++) out[i + e] = (d[e] << bits) | m[e];
        }
    } else {
        for (int i = 0; i < n; i++) { out[i] = (int)b.get(off, bits); off += bits; }
    }
}
int replicate(int v, int bits, int width) {
    int out = 0, have = 0;
    while (have < width) { out = (out << bits) | v; have += bits; }
    return out >> (have - width);
}
int unq_color(int q, int v) {
    int bits, trits, quints; btq(q, bits, trits, quints);
    if (!trits && !quints) return replicate(v, bits, 8);
    const int D = v >> bits, m = v & ((1 << bits) - 1), A = (m & 1) ? 0x1FF : 0;
    auto bit = [m](int i) { return (m >> i) & 1; };
    int B = 0, C;
    if (trits) {
        static const int kC[7] = {0, 204, 93, 44, 22, 11, 5};
        C = kC[bits];
        if (bits == 2) B = bit(1) * 0x116;
        else if (bits == 3) B = bit(2) * 0x10A + bit(1) * 0x85;
        else if (bits == 4) B = bit(3) * 0x104 + bit(2) * 0x82 + bit(1) * 0x41;
        else if (bits == 5) B = bit(4) * 0x102 + bit(3) * 0x81 + bit(2) * 0x40 + bit(1) * 0x20;
        else if (bits == 6) B = bit(5) * 0x101 + bit(4) * 0x80 + bit(3) * 0x40 + bit(2) * 0x20 + bit(1) * 0x10;
    } else {
        static const int kC[6] = {0, 113, 54, 26, 13, 6};
        C = kC[bits];
        if (bits == 2) B = bit(1) * 0x10C;
        else if (bits == 3) B = bit(2) * 0x105 + bit(1) * 0x82;
        else if (bits == 4) B = bit(3) * 0x102 + bit(2) * 0x81 + bit(1) * 0x40;
        else if (bits == 5) B = bit(4) * 0x101 + bit(3) * 0x80 + bit(2) * 0x40 + bit(1) * 0x20;
    }
    return (A & 0x80) | (((D * C + B) ^ A) >> 2);
}
int unq_weight(int q, int v) {
    int bits, trits, quints; btq(q, bits, trits, quints);
    int r;
    if (!trits && !quints) r = replicate(v, bits, 6);
    else {
        const int D = v >> bits, m = v & ((1 << bits) - 1), A = (m & 1) ? 0x7F : 0, b1 = (m >> 1) & 1, b2 = (m >> 2) & 1;
        if (bits == 0) {
            static const int t0[3] = {0, 32, 63}, q0[5] = {0, 16, 32, 47, 63};
            r = trits ? t0[D] : q0[D];
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
bool decode_mode(int m, Mode& o) {
    int q = (m >> 4) & 1, H = (m >> 9) & 1, D = (m >> 10) & 1, A = (m >> 5) & 3;
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
        int B = (m >> 9) & 3;
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
uint32_t hash52(uint32_t v) {
    v ^= v >> 15; v *= 0xEEDE0891; v ^= v >> 5; v += v << 16;
    v ^= v >> 7; v ^= v >> 3; v ^= v << 6; v ^= v >> 17;
    return v;
}
int select_partition(int seed, int x, int y, int pc, bool small) {
    if (small) { x <<= 1; y <<= 1; }
    seed += (pc - 1) * 1024;
    const uint32_t r = hash52((uint32_t)seed);
    uint8_t s[12];
    const int sh[12] = {0, 4, 8, 12, 16, 20, 24, 28, 18, 22, 26, 30};
    for (int i = 0; i < 12; i++) { uint32_t v = i == 11 ? ((r >> 30) | (r << 2)) : (r >> sh[i]); s[i] = (uint8_t)((v & 0xF) * (v & 0xF)); }
    int sh1, sh2;
    if (seed & 1) { sh1 = (seed & 2) ? 4 : 5; sh2 = pc == 3 ? 6 : 5; } else { sh1 = pc == 3 ? 6 : 5; sh2 = (seed & 2) ? 4 : 5; }
    for (int i = 0; i < 8; i++) s[i] >>= (i & 1) ? sh2 : sh1;
    int a = (s[0] * x + s[1] * y + (r >> 14)) & 0x3F, b = (s[2] * x + s[3] * y + (r >> 10)) & 0x3F;
    int c = (s[4] * x + s[5] * y + (r >> 6)) & 0x3F, d = (s[6] * x + s[7] * y + (r >> 2)) & 0x3F;
    if (pc <= 3) d = 0;
    if (pc <= 2) c = 0;
    if (pc <= 1) b = 0;
    if (a >= b && a >= c && a >= d) return 0;
    if (b >= c && b >= d) return 1;
    return c >= d ? 2 : 3;
}
void bts(int& a, int& b) {  // bit_transfer_signed(a, b)
    b >>= 1; b |= a & 0x80; a >>= 1; a &= 0x3F;
    if (a & 0x20) a -= 0x40;
}
int c255(int v) { return std::min(std::max(v, 0), 255); }
// LDR endpoint decode; returns false for HDR modes.
bool decode_endpoints(int cem, const int* v, int e0[4], int e1[4]) {
    auto set = [](int* e, int r, int g, int b, int a) { e[0] = r; e[1] = g; e[2] = b; e[3] = a; };
    auto bc = [](int* e) { e[0] = (e[0] + e[2]) >> 1; e[1] = (e[1] + e[2]) >> 1; };
    switch (cem) {
        case 0: set(e0, v[0], v[0], v[0], 255); set(e1, v[1], v[1], v[1], 255); return true;
        case 1: { int l0 = (v[0] >> 2) | (v[1] & 0xC0), l1 = std::min(l0 + (v[1] & 0x3F), 255); set(e0, l0, l0, l0, 255); set(e1, l1, l1, l1, 255); return true; }
        case 4: set(e0, v[0], v[0], v[0], v[2]); set(e1, v[1], v[1], v[1], v[3]); return true;
        case 5: { int a0 = v[0], b0 = v[1], a1 = v[2], b1 = v[3]; bts(b0, a0); bts(b1, a1);
                  set(e0, a0, a0, a0, a1); set(e1, c255(a0 + b0), c255(a0 + b0), c255(a0 + b0), c255(a1 + b1)); return true; }
        case 6: set(e0, (v[0] * v[3]) >> 8, (v[1] * v[3]) >> 8, (v[2] * v[3]) >> 8, 255); set(e1, v[0], v[1], v[2], 255); return true;
        case 8: case 12: {
            const int a0 = cem == 12 ? v[6] : 255, a1 = cem == 12 ? v[7] : 255;
            if (v[1] + v[3] + v[5] >= v[0] + v[2] + v[4]) { set(e0, v[0], v[2], v[4], a0); set(e1, v[1], v[3], v[5], a1); }
            else { set(e0, v[1], v[3], v[5], a1); set(e1, v[0], v[2], v[4], a0); bc(e0); bc(e1); }
            return true;
        }
        case 9: case 13: {
            int x[8]; for (int i = 0; i < 8; i++) x[i] = v[i];
            bts(x[1], x[0]); bts(x[3], x[2]); bts(x[5], x[4]);
            if (cem == 13) bts(x[7], x[6]);
            const int a0 = cem == 13 ? x[6] : 255, a1 = cem == 13 ? x[6] + x[7] : 255;
            if (x[1] + x[3] + x[5] >= 0) { set(e0, x[0], x[2], x[4], a0); set(e1, x[0] + x[1], x[2] + x[3], x[4] + x[5], a1); }
            else { set(e0, x[0] + x[1], x[2] + x[3], x[4] + x[5], a1); set(e1, x[0], x[2], x[4], a0); bc(e0); bc(e1); }
            for (int i = 0; i < 4; i++) { e0[i] = c255(e0[i]); e1[i] = c255(e1[i]); }
            return true;
        }
        case 10: set(e0, (v[0] * v[3]) >> 8, (v[1] * v[3]) >> 8, (v[2] * v[3]) >> 8, v[4]); set(e1, v[0], v[1], v[2], v[5]); return true;
        default: return false;
    }
}
// Decodes one block into 16-bit texels; returns false for error / HDR blocks.
bool decode_block(const uint8_t* blk, int bx, int by, uint16_t* out) {
    const Bits b{blk};
    const int T = bx * by;
    const int mode = (int)b.get(0, 11);
    if ((mode & 0x1FF) == 0x1FC) {  // void extent
        if (mode & 0x200) return false;  // HDR
        uint16_t c[4];
        for (int i = 0; i < 4; i++) c[i] = (uint16_t)b.get(64 + 16 * i, 16);
        for (int t = 0; t < T; t++) for (int i = 0; i < 4; i++) out[t * 4 + i] = c[i];
        return true;
    }
    Mode m;
    if (!decode_mode(mode, m) || m.xw > bx || m.yw > by) return false;
    const int pc = (int)b.get(11, 2) + 1;
    if (pc == 4 && m.dual) return false;
    const int W = m.xw * m.yw, nw = W * (m.dual ? 2 : 1), wbits = ise_bits(nw, m.q);
    int cem[4], seed = 0, below = 128 - wbits, cstart;
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
    if (nv > 18) return false;
    const int avail = below - cstart;
    int cq = -1;
    for (int q = 20; q >= 0; q--) if (ise_bits(nv, q) <= avail) { cq = q; break; }
    if (cq < 4) return false;
    int cv[32], wv[64];
    decode_ise(b, cstart, nv, cq, cv);
    for (int i = 0; i < nv; i++) cv[i] = unq_color(cq, cv[i]);
    uint8_t rev[16];
    for (int i = 0; i < 16; i++) {
        int p = blk[15 - i];
        p = ((p & 0x0F) << 4) | ((p >> 4) & 0x0F); p = ((p & 0x33) << 2) | ((p >> 2) & 0x33); p = ((p & 0x55) << 1) | ((p >> 1) & 0x55);
        rev[i] = (uint8_t)p;
    }
    decode_ise(Bits{rev}, 0, nw, m.q, wv);
    for (int i = 0; i < nw; i++) wv[i] = unq_weight(m.q, wv[i]);
    int e0[4][4], e1[4][4], vo = 0;
    for (int i = 0; i < pc; i++) {
        if (!decode_endpoints(cem[i], cv + vo, e0[i], e1[i])) return false;
        vo += 2 * (cem[i] >> 2) + 2;
    }
    const int ds = (1024 + bx / 2) / (bx - 1), dt = (1024 + by / 2) / (by - 1);
    const bool small = T < 31;
    for (int y = 0; y < by; y++)
        for (int x = 0; x < bx; x++) {
            const int cs = ds * x, ct = dt * y;
            const int gs = (cs * (m.xw - 1) + 32) >> 6, gt = (ct * (m.yw - 1) + 32) >> 6;
            const int js = gs >> 4, fs = gs & 15, jt = gt >> 4, ft = gt & 15;
            const int w11 = (fs * ft + 8) >> 4, w10 = ft - w11, w01 = fs - w11, w00 = 16 - fs - ft + w11;
            const int v0 = js + jt * m.xw;
            int wpl[2];
            for (int pl = 0; pl < (m.dual ? 2 : 1); pl++) {
                auto g = [&](int idx) { return idx < W ? wv[idx * (m.dual ? 2 : 1) + pl] : 0; };
                wpl[pl] = (g(v0) * w00 + g(v0 + 1) * w01 + g(v0 + m.xw) * w10 + g(v0 + m.xw + 1) * w11 + 8) >> 4;
            }
            const int part = pc > 1 ? select_partition(seed, x, y, pc, small) : 0;
            const int t = y * bx + x;
            for (int c = 0; c < 4; c++) {
                const int w = (m.dual && c == ccs) ? wpl[1] : wpl[0];
                const int c0 = e0[part][c] * 257, c1 = e1[part][c] * 257;
                out[t * 4 + c] = (uint16_t)((c0 * (64 - w) + c1 * w + 32) >> 6);
            }
        }
    return true;
}

}  // namespace

extern "C" int astcb200_decode(uint32_t bx, uint32_t by, uint32_t dx, uint32_t dy, const uint8_t* blocks, size_t len, uint8_t* out) {
    if (!blocks || !out || !astcb200::valid_footprint((int)bx, (int)by) || dx == 0 || dy == 0) return ASTCB200_BAD_ARG;
    const uint32_t nbx = (dx + bx - 1) / bx, nby = (dy + by - 1) / by;
    if (len < (size_t)nbx * nby * 16) return ASTCB200_BAD_ARG;
    uint16_t tex[144 * 4];
    for (uint32_t j = 0; j < nby; j++)
        for (uint32_t i = 0; i < nbx; i++) {
            if (!decode_block(blocks + ((size_t)j * nbx + i) * 16, (int)bx, (int)by, tex)) {
                for (uint32_t t = 0; t < bx * by; t++) { tex[t * 4] = 0xFFFF; tex[t * 4 + 1] = 0; tex[t * 4 + 2] = 0xFFFF; tex[t * 4 + 3] = 0xFFFF; }
            }
            for (uint32_t y = 0; y < by; y++)
                for (uint32_t x = 0; x < bx; x++) {
                    const uint32_t px = i * bx + x, py = j * by + y;
                    if (px >= dx || py >= dy) continue;
                    for (int c = 0; c < 4; c++) out[((size_t)py * dx + px) * 4 + c] = (uint8_t)(((uint32_t)tex[(y * bx + x) * 4 + c] * 255u + 32767u) / 65535u);
                }
        }
    return ASTCB200_OK;
}
