// Refinement and final-selection kernels of the ASTC encoder (sm_100a).
//
//   k_refine       passes 13-17 (shaders/pass13..pass17), six iterations as
//                  driven by compression_pipeline.cpp:473-484: least-squares
//                  endpoints, colour endpoint packing (every LDR encoding the
//                  reference tries), unpacking, weight realignment, final
//                  error with a best-so-far snapshot.  One thread owns one
//                  candidate for all six iterations; the 8 candidates of a
//                  partitioned block share a CTA and its staged texels.
//   k_select_pack  pass18 plus the host argmin over candidates and partition
//                  counts (compression_pipeline.cpp:500-519), then the ASTC
//                  physical block layout (code/physical_compression.cpp:843)
//                  written straight to the 16-byte output block.
#include <algorithm>
#include <mutex>
#include <type_traits>

#include "decode_block.cuh"
#include "device_math.cuh"
#include "kernels.h"

namespace astcb200 {

using namespace dev;

namespace {

constexpr float ERR_DEFAULT = 1e37f;
__constant__ int c_levels_r[21] = {2, 3, 4, 5, 6, 8, 10, 12, 16, 20, 24, 32, 40, 48, 64, 80, 96, 128, 160, 192, 256};

enum {
    FMT_LUMINANCE = 0, FMT_LUMINANCE_DELTA = 1, FMT_LUMINANCE_ALPHA = 4, FMT_LUMINANCE_ALPHA_DELTA = 5,
    FMT_RGB_SCALE = 6, FMT_RGB = 8, FMT_RGB_DELTA = 9, FMT_RGB_SCALE_ALPHA = 10, FMT_RGBA = 12, FMT_RGBA_DELTA = 13
};

struct I4 { int32_t x, y, z, w; };
__device__ __forceinline__ int32_t ic(const I4& v, int c) { return c == 0 ? v.x : c == 1 ? v.y : c == 2 ? v.z : v.w; }
__device__ __forceinline__ I4 ivec(float4 v) { return {f2i(v.x), f2i(v.y), f2i(v.z), f2i(v.w)}; }
__device__ __forceinline__ float4 rnev(float4 v) { return make_float4(rintf(v.x), rintf(v.y), rintf(v.z), rintf(v.w)); }
__device__ __forceinline__ int32_t shl1(int32_t v) { return (int32_t)((uint32_t)v << 1); }

// ------------------------------------------------------------ pass14 colour endpoint packing
struct Packer {
    const uint8_t* cu2u;  // [17][512]
    __device__ int32_t tab(uint32_t q, int32_t idx) const { return cu2u[(q - 4) * 512 + idx]; }
    __device__ float enc_err(float4 u0, float4 u1, I4 q0, I4 q1) const {
        const float4 e0 = u0 - make_float4((float)q0.x, (float)q0.y, (float)q0.z, (float)q0.w);
        const float4 e1 = u1 - make_float4((float)q1.x, (float)q1.y, (float)q1.z, (float)q1.w);
        const float4 e = e0 * e0 + e1 * e1;
        return ((e.x + e.y) + e.z) + e.w;
    }
    __device__ I4 q3int(uint32_t q, I4 v) const { return {tab(q, v.x * 2 + 1), tab(q, v.y * 2 + 1), tab(q, v.z * 2 + 1), 0}; }
    __device__ int32_t qf1(uint32_t q, int32_t v, float vf) const { return tab(q, v * 2 + ((vf - (float)v) >= -0.1f ? 1 : 0)); }
    __device__ I4 q3flt(uint32_t q, I4 v, float4 vf) const { return {qf1(q, v.x, vf.x), qf1(q, v.y, vf.y), qf1(q, v.z, vf.z), 0}; }
    __device__ uint32_t qint(uint32_t q, int32_t v) const { return (uint32_t)tab(q, v * 2 + 1); }
    __device__ uint32_t qflt(uint32_t q, int32_t v, float vf) const { return (uint32_t)qf1(q, v, vf); }

    // bit_transfer_signed(&a, &b) (pass14:355-369)
    __device__ static void bts(I4& a, I4& b) {
        int32_t* pa = &a.x; int32_t* pb = &b.x;
#pragma unroll
        for (int c = 0; c < 4; c++) {
            const uint32_t a0 = (uint32_t)pa[c], b0 = (uint32_t)pb[c];
            int32_t na = (int32_t)((a0 >> 1) & 0x3F);
            if (na & 0x20) na -= 0x40;
            pb[c] = (int32_t)((b0 >> 1) | (a0 & 0x80));
            pa[c] = na;
        }
    }
    __device__ static I4 uncontract(I4 v) { return {(v.x + v.z) >> 1, (v.y + v.z) >> 1, v.z, v.w}; }
    __device__ static int32_t clamp255(int32_t v) { return min(max(v, 0), 255); }
    __device__ static void delta_unpack(I4 i0, I4 i1, I4& o0, I4& o1) {
        bts(i1, i0);
        const int32_t s = i1.x + i1.y + i1.z;
        i1 = {i1.x + i0.x, i1.y + i0.y, i1.z + i0.z, i1.w + i0.w};
        if (s < 0) { I4 t = uncontract(i0); i0 = uncontract(i1); i1 = t; }
        o0 = {clamp255(i0.x), clamp255(i0.y), clamp255(i0.z), clamp255(i0.w)};
        o1 = {clamp255(i1.x), clamp255(i1.y), clamp255(i1.z), clamp255(i1.w)};
    }
    __device__ static void rgba_unpack(I4 i0, I4 i1, I4& o0, I4& o1) {
        if ((i0.x + i0.y + i0.z) > (i1.x + i1.y + i1.z)) { I4 t = uncontract(i0); i0 = uncontract(i1); i1 = t; }
        o0 = i0; o1 = i1;
    }
    __device__ static bool out_of_range(float4 c) {
        return c.x < 0.0f || c.x > 255.0f || c.y < 0.0f || c.y > 255.0f || c.z < 0.0f || c.z > 255.0f || c.w < 0.0f || c.w > 255.0f;
    }
    __device__ static float4 inv_bc(float4 c) { return make_float4((c.x + c.x) - c.z, (c.y + c.y) - c.z, (c.z + c.z) - c.z, (c.w + c.w) - c.w); }

    // try_quantize_rgb_delta(_blue_contract) body after the optional inverse contraction
    __device__ bool rgb_delta(float4 c0, float4 c1, I4& o0, I4& o1, uint32_t q, bool want_bc) const {
        I4 c0a = ivec(rnev(c0));
        c0a = {shl1(c0a.x), shl1(c0a.y), shl1(c0a.z), shl1(c0a.w)};
        I4 c0b = {c0a.x & 0xFF, c0a.y & 0xFF, c0a.z & 0xFF, c0a.w & 0xFF};
        const I4 c0be = q3int(q, c0b);
        c0b = {c0be.x | (c0a.x & 0x100), c0be.y | (c0a.y & 0x100), c0be.z | (c0a.z & 0x100), c0be.w | (c0a.w & 0x100)};
        I4 c1d = ivec(rnev(c1));
        c1d = {shl1(c1d.x) - c0b.x, shl1(c1d.y) - c0b.y, shl1(c1d.z) - c0b.z, 0};
        if (c1d.x > 63 || c1d.x < -64 || c1d.y > 63 || c1d.y < -64 || c1d.z > 63 || c1d.z < -64) return false;
        c1d = {(c1d.x & 0x7F) | ((c0b.x & 0x100) >> 1), (c1d.y & 0x7F) | ((c0b.y & 0x100) >> 1),
               (c1d.z & 0x7F) | ((c0b.z & 0x100) >> 1), (c1d.w & 0x7F) | ((c0b.w & 0x100) >> 1)};
        const I4 c1de = q3int(q, c1d);
        if (((c1d.x ^ c1de.x) & 0xC0) || ((c1d.y ^ c1de.y) & 0xC0) || ((c1d.z ^ c1de.z) & 0xC0)) return false;
        I4 e0 = c0be, e1 = c1de;
        bts(e1, e0);
        const int32_t s = e1.x + e1.y + e1.z;
        if (want_bc ? (s >= 0) : (s < 0)) return false;
        e0 = {e0.x + e1.x, e0.y + e1.y, e0.z + e1.z, e0.w + e1.w};
        if (e0.x < 0 || e0.x > 0xFF || e0.y < 0 || e0.y > 0xFF || e0.z < 0 || e0.z > 0xFF || e0.w < 0 || e0.w > 0xFF) return false;
        o0 = c0be; o1 = c1de;
        return true;
    }
    __device__ bool try_rgb_delta_bc(float4 a0, float4 a1, I4& o0, I4& o1, uint32_t q) const {
        const float4 c0 = inv_bc(a1), c1 = inv_bc(a0);
        if (out_of_range(c0) || out_of_range(c1)) return false;
        return rgb_delta(c0, c1, o0, o1, q, true);
    }
    __device__ bool try_rgb_bc(float4 a0, float4 a1, I4& o0, I4& o1, uint32_t q) const {
        const float4 c0 = inv_bc(a0), c1 = inv_bc(a1);
        if (out_of_range(c0) || out_of_range(c1)) return false;
        const I4 c0i = q3flt(q, ivec(rnev(c0)), c0), c1i = q3flt(q, ivec(rnev(c1)), c1);
        if ((c1i.x + c1i.y + c1i.z) <= (c0i.x + c0i.y + c0i.z)) return false;
        o0 = c1i; o1 = c0i;
        return true;
    }
    // Quantised channel sums of the endpoints at one step of the loop below: true when the
    // step ends it (the low endpoint's sum no longer above the high one's).
    __device__ bool qrgb_probe(uint32_t q, float x0, float y0, float z0, float x1, float y1, float z1, I4& c0i, I4& c1i) const {
        c0i = q3flt(q, I4{max(f2i(rintf(x0)), 0), max(f2i(rintf(y0)), 0), max(f2i(rintf(z0)), 0), 0}, make_float4(x0, y0, z0, 0.0f));
        c1i = q3flt(q, I4{min(f2i(rintf(x1)), 255), min(f2i(rintf(y1)), 255), min(f2i(rintf(z1)), 255), 0}, make_float4(x1, y1, z1, 0.0f));
        return (c0i.x + c0i.y + c0i.z) <= (c1i.x + c1i.y + c1i.z);
    }
    // The reference's loop nudges the endpoints 0.2 apart per step (at most 4096 steps) and
    // stops at the first step whose quantised channel sums no longer cross.  A rounded
    // channel and its half-step bit move monotonically with its endpoint and the table is
    // monotonic, so the low sum never rises and the high one never falls from step to step:
    // the stopping test is monotonic in the step.  The stop is found by probing steps 0, 1,
    // 3, 7, ... and bisecting the last bracket; the endpoints are always brought to a probed
    // step by the loop's own float subtractions and additions from an earlier probed step,
    // so each probe sees the values the loop would.
    __device__ void quant_rgb(float4 c0, float4 c1, I4& o0, I4& o1, uint32_t q) const {
        float x0 = c0.x, y0 = c0.y, z0 = c0.z, x1 = c1.x, y1 = c1.y, z1 = c1.z;  // step lo
        I4 c0i, c1i;
        if (!qrgb_probe(q, x0, y0, z0, x1, y1, z1, c0i, c1i)) {
            auto advance = [](float& a, float& b, float& c, float& d, float& e, float& f, int n) {
#pragma unroll 4
                for (int i = 0; i < n; i++) { a = a - 0.2f; b = b - 0.2f; c = c - 0.2f; d = d + 0.2f; e = e + 0.2f; f = f + 0.2f; }
            };
            int lo = 0, hi = 0, step = 1;
            for (;;) {  // the test fails at lo; at most 13 trips
                hi = min(lo + step, 4095);
                float a = x0, b = y0, c = z0, d = x1, e = y1, f = z1;
                advance(a, b, c, d, e, f, hi - lo);
                if (qrgb_probe(q, a, b, c, d, e, f, c0i, c1i) || hi == 4095) break;
                x0 = a; y0 = b; z0 = c; x1 = d; y1 = e; z1 = f;
                lo = hi;
                step *= 2;
            }
            while (hi - lo > 1) {  // the stop is in (lo, hi] (hi = 4095: the last step)
                const int mid = lo + (hi - lo) / 2;
                float a = x0, b = y0, c = z0, d = x1, e = y1, f = z1;
                advance(a, b, c, d, e, f, mid - lo);
                if (qrgb_probe(q, a, b, c, d, e, f, c0i, c1i)) {
                    hi = mid;
                } else {
                    lo = mid;
                    x0 = a; y0 = b; z0 = c; x1 = d; y1 = e; z1 = f;
                }
            }
            advance(x0, y0, z0, x1, y1, z1, 1);
            qrgb_probe(q, x0, y0, z0, x1, y1, z1, c0i, c1i);
        }
        o0 = c0i; o1 = c1i;
    }
    __device__ bool try_alpha_delta(float4 color0, float4 color1, I4& o0, I4& o1, uint32_t q) const {
        const int32_t a0a = shl1(f2i(rintf(color0.w)));
        int32_t a0b = a0a & 0xFF;
        const int32_t a0be = (int32_t)qint(q, a0b);
        a0b = a0be | (a0a & 0x100);
        int32_t a1d = shl1(f2i(rintf(color1.w))) - a0b;
        if (a1d > 63 || a1d < -64) return false;
        a1d = (a1d & 0x7F) | ((a0b & 0x100) >> 1);
        const int32_t a1de = (int32_t)qint(q, a1d);
        if (((a1d ^ a1de) & 0xC0) != 0) return false;
        int32_t a1du = a1de & 0x7F;
        if (a1du & 0x40) a1du -= 0x80;
        a1du += a0b;
        if (a1du < 0 || a1du > 0x1FF) return false;
        o0.w = a0be; o1.w = a1de;
        return true;
    }
    __device__ void quant_rgbs(float4 color, uint32_t* out, uint32_t q) const {
        const float scale = 1.0f / 257.0f;
        const float r = clampf(color.x * scale, 0.0f, 255.0f), g = clampf(color.y * scale, 0.0f, 255.0f), b = clampf(color.z * scale, 0.0f, 255.0f);
        const uint32_t ri = qflt(q, f2i(rintf(r)), r), gi = qflt(q, f2i(rintf(g)), g), bi = qflt(q, f2i(rintf(b)), b);
        const float oldsum = ((color.x + color.y) + color.z) * scale;
        const float newsum = (float)(ri + gi + bi);
        const float sa = clampf((color.w * (oldsum + 1e-10f)) / (newsum + 1e-10f), 0.0f, 1.0f);
        const int32_t si = min(max(f2i(rintf(sa * 256.0f)), 0), 255);
        out[0] = ri; out[1] = gi; out[2] = bi; out[3] = qint(q, si);
    }
    __device__ bool try_la_delta(float4 c0, float4 c1, uint32_t* out, uint32_t q) const {
        const float l0 = ((c0.x + c0.y) + c0.z) / 3.0f, l1 = ((c1.x + c1.y) + c1.z) / 3.0f;
        const int32_t l0a = shl1(f2i(rintf(l0))), a0a = shl1(f2i(rintf(c0.w)));
        const uint32_t l0be = qint(q, l0a & 0xFF), a0be = qint(q, a0a & 0xFF);
        const int32_t l0b = (int32_t)l0be | (l0a & 0x100), a0b = (int32_t)a0be | (a0a & 0x100);
        int32_t l1d = shl1(f2i(rintf(l1))) - l0b, a1d = shl1(f2i(rintf(c1.w))) - a0b;
        if (l1d > 63 || l1d < -64 || a1d > 63 || a1d < -64) return false;
        l1d = (l1d & 0x7F) | ((l0b & 0x100) >> 1);
        a1d = (a1d & 0x7F) | ((a0b & 0x100) >> 1);
        const uint32_t l1de = qint(q, l1d), a1de = qint(q, a1d);
        int32_t l1du = (int32_t)l1de, a1du = (int32_t)a1de;
        if (((l1d ^ l1du) & 0xC0) != 0) return false;
        if (((a1d ^ a1du) & 0xC0) != 0) return false;
        l1du &= 0x7F; a1du &= 0x7F;
        if (l1du & 0x40) l1du -= 0x80;
        if (a1du & 0x40) a1du -= 0x80;
        l1du += l0b; a1du += a0b;
        if (l1du < 0 || l1du > 0x1FF || a1du < 0 || a1du > 0x1FF) return false;
        out[0] = l0be; out[1] = l1de; out[2] = a0be; out[3] = a1de;
        return true;
    }
    // pack_color_endpoints_helper (pass14:917-1224)
    __device__ __noinline__ uint32_t pack(float4 color0, float4 color1, float4 rgbs, uint32_t fmt, uint32_t q, uint32_t* out) const {
        const float4 c0 = vmin(vmax(color0, mk(0.0f)), mk(65535.0f)) / mk(257.0f);
        const float4 c1 = vmin(vmax(color1, mk(0.0f)), mk(65535.0f)) / mk(257.0f);
        float best = ERR_DEFAULT;
#pragma unroll
        for (int i = 0; i < 8; i++) out[i] = 0;
        uint32_t bf = FMT_LUMINANCE;
        if (fmt == FMT_RGB || fmt == FMT_RGBA) {
            const bool rgba = fmt == FMT_RGBA;
            const uint32_t dfmt = rgba ? FMT_RGBA_DELTA : FMT_RGB_DELTA;
            I4 o0 = {0, 0, 0, 0}, o1 = {0, 0, 0, 0}, p0 = {0, 0, 0, 0}, p1 = {0, 0, 0, 0}, u0, u1;
            if (q <= 18) {
                bool ok = try_rgb_delta_bc(c0, c1, o0, o1, q);
                if (rgba && ok) ok = try_alpha_delta(c1, c0, o0, o1, q);
                if (ok) { delta_unpack(o0, o1, u0, u1); bf = dfmt; best = enc_err(c0, c1, u0, u1); }
                ok = rgb_delta(c0, c1, p0, p1, q, false);
                if (rgba && ok) ok = try_alpha_delta(c0, c1, p0, p1, q);
                if (ok) {
                    delta_unpack(p0, p1, u0, u1);
                    const float e = enc_err(c0, c1, u0, u1);
                    if (e < best) { best = e; bf = dfmt; o0 = p0; o1 = p1; }
                }
            }
            if (q < 20 && try_rgb_bc(c0, c1, p0, p1, q)) {
                if (rgba) { p0.w = (int32_t)qflt(q, f2i(rintf(c1.w)), c1.w); p1.w = (int32_t)qflt(q, f2i(rintf(c0.w)), c0.w); }
                rgba_unpack(p0, p1, u0, u1);
                const float e = enc_err(c0, c1, u0, u1);
                if (e < best) { best = e; bf = fmt; o0 = p0; o1 = p1; }
            }
            {
                quant_rgb(c0, c1, p0, p1, q);
                if (rgba) { p0.w = (int32_t)qflt(q, f2i(rintf(c0.w)), c0.w); p1.w = (int32_t)qflt(q, f2i(rintf(c1.w)), c1.w); }
                rgba_unpack(p0, p1, u0, u1);
                const float e = enc_err(c0, c1, u0, u1);
                if (e < best) { best = e; bf = fmt; o0 = p0; o1 = p1; }
            }
            out[0] = (uint32_t)o0.x; out[1] = (uint32_t)o1.x; out[2] = (uint32_t)o0.y;
            out[3] = (uint32_t)o1.y; out[4] = (uint32_t)o0.z; out[5] = (uint32_t)o1.z;
            if (rgba) { out[6] = (uint32_t)o0.w; out[7] = (uint32_t)o1.w; }
        } else if (fmt == FMT_RGB_SCALE) {
            quant_rgbs(rgbs, out, q); bf = FMT_RGB_SCALE;
        } else if (fmt == FMT_RGB_SCALE_ALPHA) {
            out[4] = qflt(q, f2i(rintf(c0.w)), c0.w); out[5] = qflt(q, f2i(rintf(c1.w)), c1.w);
            quant_rgbs(rgbs, out, q); bf = FMT_RGB_SCALE_ALPHA;
        } else if (fmt == FMT_LUMINANCE_ALPHA) {
            if (q <= 18 && try_la_delta(c0, c1, out, q)) {
                bf = FMT_LUMINANCE_ALPHA_DELTA;
            } else {
                const float l0 = ((c0.x + c0.y) + c0.z) / 3.0f, l1 = ((c1.x + c1.y) + c1.z) / 3.0f;
                out[0] = qflt(q, f2i(rintf(l0)), l0); out[1] = qflt(q, f2i(rintf(l1)), l1);
                out[2] = qflt(q, f2i(rintf(c0.w)), c0.w); out[3] = qflt(q, f2i(rintf(c1.w)), c1.w);
                bf = FMT_LUMINANCE_ALPHA;
            }
        } else {  // FMT_LUMINANCE and any other format
            float l0 = ((c0.x + c0.y) + c0.z) / 3.0f, l1 = ((c1.x + c1.y) + c1.z) / 3.0f;
            if (l0 > l1) { const float av = (l0 + l1) * 0.5f; l0 = av; l1 = av; }
            out[0] = qflt(q, f2i(rintf(l0)), l0); out[1] = qflt(q, f2i(rintf(l1)), l1);
            bf = FMT_LUMINANCE;
        }
        return bf;
    }
};

// pass15: decode packed endpoints of one partition, scaled by 257.
__device__ __noinline__ void unpack_endpoints(uint32_t fmt, const uint8_t* v, uint16_t* e0, uint16_t* e1) {
    I4 o0, o1;
    auto I = [&](int k) { return (int32_t)v[k]; };
    switch (fmt) {
        case FMT_LUMINANCE_DELTA: {
            const int32_t l0 = (I(0) >> 2) | (I(1) & 0xC0), l1 = min(l0 + (I(1) & 0x3F), 255);
            o0 = {l0, l0, l0, 255}; o1 = {l1, l1, l1, 255}; break;
        }
        case FMT_LUMINANCE_ALPHA: o0 = {I(0), I(0), I(0), I(2)}; o1 = {I(1), I(1), I(1), I(3)}; break;
        case FMT_LUMINANCE_ALPHA_DELTA: {
            int32_t l0 = I(0), l1 = I(1), a0 = I(2), a1 = I(3);
            l0 |= (l1 & 0x80) << 1; a0 |= (a1 & 0x80) << 1;
            l1 &= 0x7F; a1 &= 0x7F;
            if (l1 & 0x40) l1 -= 0x80;
            if (a1 & 0x40) a1 -= 0x80;
            l0 >>= 1; l1 >>= 1; a0 >>= 1; a1 >>= 1;
            l1 = min(max(l0 + l1, 0), 255); a1 = min(max(a0 + a1, 0), 255);
            o0 = {l0, l0, l0, a0}; o1 = {l1, l1, l1, a1}; break;
        }
        case FMT_RGB_SCALE: {
            const int32_t s = I(3);
            o1 = {I(0), I(1), I(2), 255};
            o0 = {(I(0) * s) >> 8, (I(1) * s) >> 8, (I(2) * s) >> 8, 255}; break;
        }
        case FMT_RGB_SCALE_ALPHA: {
            const int32_t s = I(3);
            o1 = {I(0), I(1), I(2), I(5)};
            o0 = {(I(0) * s) >> 8, (I(1) * s) >> 8, (I(2) * s) >> 8, I(4)}; break;
        }
        case FMT_RGB: Packer::rgba_unpack({I(0), I(2), I(4), 0}, {I(1), I(3), I(5), 0}, o0, o1); o0.w = 255; o1.w = 255; break;
        case FMT_RGB_DELTA: Packer::delta_unpack({I(0), I(2), I(4), 0}, {I(1), I(3), I(5), 0}, o0, o1); o0.w = 255; o1.w = 255; break;
        case FMT_RGBA: Packer::rgba_unpack({I(0), I(2), I(4), I(6)}, {I(1), I(3), I(5), I(7)}, o0, o1); break;
        case FMT_RGBA_DELTA: Packer::delta_unpack({I(0), I(2), I(4), I(6)}, {I(1), I(3), I(5), I(7)}, o0, o1); break;
        default: o0 = {I(0), I(0), I(0), 255}; o1 = {I(1), I(1), I(1), 255}; break;
    }
    e0[0] = (uint16_t)(o0.x * 257); e0[1] = (uint16_t)(o0.y * 257); e0[2] = (uint16_t)(o0.z * 257); e0[3] = (uint16_t)(o0.w * 257);
    e1[0] = (uint16_t)(o1.x * 257); e1[1] = (uint16_t)(o1.y * 257); e1[2] = (uint16_t)(o1.z * 257); e1[3] = (uint16_t)(o1.w * 257);
}

// ------------------------------------------------------------ k_refine
constexpr int kRefineThreads = 128;

// Candidate threads per partitioned block (the refinement top-N rounded up to a power of
// two) and partitioned blocks per CTA: 16 x 8 for the full search; more, narrower ones when
// the proposal search keeps fewer candidates, capped so the staged texels stay <= 40 KB.
__host__ __device__ inline int refine_cpb(int topn) { return topn <= 1 ? 1 : topn <= 2 ? 2 : topn <= 4 ? 4 : 8; }
__host__ __device__ inline int refine_pbs(int T, int topn) {
    const int by_threads = kRefineThreads / refine_cpb(topn);
    const int by_smem = 40960 / (T * (T > 16 ? 4 : 16));
    return by_threads < by_smem ? by_threads : (by_smem > 16 ? by_smem : 16);
}

// A candidate's state in shared memory, kept at the candidate's staging position for all
// iterations whichever thread runs it (73 words: an odd stride, so distinct candidates of a
// warp mostly hit distinct banks).
struct CandSmem {
    uint16_t u0[4][4], u1[4][4];  // unpacked endpoints x257 (0..65535)
    uint8_t qw[64];
    uint8_t packed[32];
    float ep[4][8];               // per partition: the least-squares endpoints ep0 (xyzw), ep1 (xyzw)
    uint32_t item;                // partitioned block of this staging position (lb + 1 | slot << 27), 0 if none
};
static_assert(sizeof(CandSmem) == 292, "odd word stride");
__device__ __forceinline__ float4 ld_ep(const float* e) { return make_float4(e[0], e[1], e[2], e[3]); }
__device__ __forceinline__ void st_ep(float* e, float4 v) { e[0] = v.x; e[1] = v.y; e[2] = v.z; e[3] = v.w; }
__device__ __forceinline__ uint4 ld_u4(const uint8_t* p) {  // 4-byte aligned shared memory
    const uint32_t* w = reinterpret_cast<const uint32_t*>(p);
    return make_uint4(w[0], w[1], w[2], w[3]);
}


struct RTabs {
    const uint8_t* b;
    const TableLayout* L;
    __device__ const DevDm& dm(int m) const { return reinterpret_cast<const DevDm*>(b + L->off_dm)[m]; }
    __device__ const DevBm& bm(int i) const { return reinterpret_cast<const DevBm*>(b + L->off_bm)[i]; }
    __device__ int tw_count(int m, int t) const { return b[L->off_tw_count + m * L->T + t]; }
    __device__ int tw_start(int m, int t) const { return reinterpret_cast<const uint16_t*>(b + L->off_tw_start)[m * L->T + t]; }
    __device__ int wt_count(int m, int w) const { return b[L->off_wt_count + m * 64 + w]; }
    __device__ int wt_start(int m, int w) const { return reinterpret_cast<const uint16_t*>(b + L->off_wt_start)[m * 64 + w]; }
    __device__ uint32_t t2w(int i) const { return reinterpret_cast<const uint16_t*>(b + L->off_t2w)[i]; }
    __device__ uint32_t w2t(int i) const { return reinterpret_cast<const uint16_t*>(b + L->off_w2t)[i]; }
    __device__ uint64_t tw4(int m, int t) const { return reinterpret_cast<const uint64_t*>(b + L->off_tw4)[m * L->T + t]; }
    __device__ int part_count(int P, int e, int q) const { return b[L->off_part_counts + ((P - 2) * 1024 + e) * 4 + q]; }
    __device__ uint32_t prev_next(int q, int v) const { return reinterpret_cast<const uint16_t*>(b + L->off_prev_next)[q * 65 + v]; }
};

// Infilled weight of texel t from the 0..64 weights (pass13:165-184, pass17:127-146).
// Padding entries of the dense list add qw[0]/64 * 0 = +0, which never changes v.
__device__ __forceinline__ float undec_weight(const RTabs& tb, int dm, const uint8_t* qw, int t, bool direct) {
    if (direct) return (float)qw[t] / 64.0f;
    const uint64_t e4 = tb.tw4(dm, t);
    float v = 0.0f;
#pragma unroll
    for (int j = 0; j < 4; j++) {
        const uint32_t e = (uint32_t)(e4 >> (16 * j)) & 0xFFFF;
        v = v + ((float)qw[e & 0xFF] / 64.0f) * ((float)(e >> 8) * (1.0f / 16.0f));
    }
    return v;
}


// A partitioned block's staged texels.  Up to 16 texels they are floats; larger blocks
// stage RGBA8 (4 bytes a texel, so more CTAs fit on an SM) read back through the CTA's
// table of (v / 255) * 65536, the value src_texel computes.
__host__ __device__ inline bool refine_u8(int T) { return T > 16; }
template <bool U8> struct TexelRow;
template <> struct TexelRow<true> {
    const uchar4* c;
    const float* lut;
    __device__ __forceinline__ float4 operator[](int t) const {
        const uchar4 v = c[t];
        return make_float4(lut[v.x], lut[v.y], lut[v.z], lut[v.w]);
    }
};
template <> struct TexelRow<false> {
    const float4* c;
    __device__ __forceinline__ float4 operator[](int t) const { return c[t]; }
};

// One refinement iteration (passes 13-17) of candidate k of a partitioned block, its
// state in cs; iteration 0 first loads the front's initial state.  Returns whether pass16
// moved a weight: a pass16 that moved none leaves a fixed point, where the next iteration's
// pass13 recomputes the same endpoints from the same weights (channels whose system is
// degenerate keep the previous values, which are these), so packing, unpacking, realignment
// and the final error repeat exactly and can never lower the error: stopping there gives
// the result of running the remaining iterations.
template <class Row>
__device__ bool refine_step(const KernelArgs& a, const PBRec& rec, const int P, int k, const Row px, const uint8_t* tp,
                            CandSmem& cs, Snap* snap, const int it) {
    const RTabs tb{a.tables, &a.L};
    const int T = a.L.T;
    const CandInit& ci = rec.c[k];
    const DevBm bm = tb.bm(ci.bm);
    const DevDm dmi = tb.dm(bm.dm);
    const bool direct = dmi.W == T;
    const float4 cw = chan_w();
    const float lsw = (cw.x + cw.y) + cw.z;
    const Packer pk{a.tables + a.L.off_cu2u};
    float4 rgbs[4];
    uint8_t packed_mod[32];
    if (it == 0) {
#pragma unroll
        for (int q = 0; q < 4; q++) { st_ep(cs.ep[q], rec.ep0[q]); st_ep(cs.ep[q] + 4, rec.ep1[q]); }
        const uint32_t* src = reinterpret_cast<const uint32_t*>(ci.qw);  // 8-byte aligned in PBRec
        uint32_t* dst = reinterpret_cast<uint32_t*>(cs.qw);
#pragma unroll
        for (int w = 0; w < 16; w++) dst[w] = src[w];
    }
    uint32_t ffmt[4] = {0, 0, 0, 0}, matched = 0, final_q = ci.ql;
    // infilled weights are recomputed where read: caching them per thread in shared memory
    // costs more resident CTAs than the recomputation
    auto UW = [&](int t) { return undec_weight(tb, bm.dm, cs.qw, t, direct); };

    auto final_error = [&]() {
        float total = 0.0f;
        for (int t = 0; t < T; t++) {
            const int p = tp[t];
            const float w = UW(t);
            const int32_t w1 = f2i(rintf(w * 64.0f)), w0 = 64 - w1;
            const float4 x = px[t];
            float4 d;
            d.x = x.x - (float)((((int32_t)cs.u0[p][0] * w0) + ((int32_t)cs.u1[p][0] * w1) + 32) >> 6);
            d.y = x.y - (float)((((int32_t)cs.u0[p][1] * w0) + ((int32_t)cs.u1[p][1] * w1) + 32) >> 6);
            d.z = x.z - (float)((((int32_t)cs.u0[p][2] * w0) + ((int32_t)cs.u1[p][2] * w1) + 32) >> 6);
            d.w = x.w - (float)((((int32_t)cs.u0[p][3] * w0) + ((int32_t)cs.u1[p][3] * w1) + 32) >> 6);
            d = vmin(make_float4(fabsf(d.x), fabsf(d.y), fabsf(d.z), fabsf(d.w)), mk(1e15f));
            total = total + fminf(dot4(d * d, cw), ERR_DEFAULT);
        }
        if (total < snap->err) {  // the snapshot's error is the best so far (ERR_DEFAULT at first)
            uint4* d = reinterpret_cast<uint4*>(snap);  // 16-byte aligned: 112-byte records
            d[0] = make_uint4(__float_as_uint(total), (uint32_t)ci.bm | final_q << 16 | matched << 24,
                              ffmt[0] | ffmt[1] << 8 | ffmt[2] << 16 | ffmt[3] << 24, 0u);
            d[1] = ld_u4(cs.packed); d[2] = ld_u4(cs.packed + 16);
#pragma unroll
            for (int i = 0; i < 4; i++) d[3 + i] = ld_u4(cs.qw + 16 * i);
        }
    };

    // ---------------- pass13: least-squares endpoints from the current weights
#pragma unroll 1
    for (int q = 0; q < P; q++) {
        const float ps = P == 1 ? (float)T : (float)tb.part_count(P, rec.entry, q);
        const float4 rsum = (rec.avg[q] * ps) * cw;
        const float4 rws = vmax(cw * ps, mk(1e-17f));
        float4 sv = rsum / rws; sv.w = 0.0f;
        const float4 sdir = normalize4(sv);
        float wmin = 1.0f, wmax = 0.0f, ls = 0.0f, ms = 0.0f, rs = 0.0f, smin = 1e10f, smax = 0.0f, sv0 = 0.0f, sv1 = 0.0f;
        float4 cx = mk(0.0f), cy = mk(0.0f);
        for (int t = 0; t < T; t++) {
            if (tp[t] != q) continue;
            const float4 rgba = px[t];
            const float w = UW(t);
            if (w < wmin) wmin = w;
            if (w > wmax) wmax = w;
            const float sc = dot3(rgba, sdir);
            if (sc < smin) smin = sc;
            if (sc > smax) smax = sc;
            const float om = 1.0f - w;
            ls = ls + om * om; ms = ms + om * w; rs = rs + w * w;
            const float4 cyc = rgba * w;
            cy = cy + cyc;
            cx = cx + (rgba - cyc);
            sv0 = sv0 + (om * sc) * lsw;
            sv1 = sv1 + (w * sc) * lsw;
        }
        const float4 colx = cx * cw, coly = cy * cw;
        const float4 lv = mk(ls) * cw, mv = mk(ms) * cw, rv = mk(rs) * cw;
        const float lx = ls * lsw, my = ms * lsw, rz = rs * lsw;
        const float scalediv = clampf(smin / fmaxf(smax, 1e-10f), 0.0f, 1.0f);
        const float4 sds = sdir * smax;
        rgbs[q] = make_float4(sds.x, sds.y, sds.z, scalediv);
        float4 e0 = ld_ep(cs.ep[q]), e1 = ld_ep(cs.ep[q] + 4);
        if (wmin >= wmax * 0.999f) {
            const float4 ac = (colx + coly) / vmax(cw * ps, mk(1e-17f));
            if (ac.x == ac.x) { e0.x = ac.x; e1.x = ac.x; }
            if (ac.y == ac.y) { e0.y = ac.y; e1.y = ac.y; }
            if (ac.z == ac.z) { e0.z = ac.z; e1.z = ac.z; }
            if (ac.w == ac.w) { e0.w = ac.w; e1.w = ac.w; }
            rgbs[q] = make_float4(sds.x, sds.y, sds.z, 1.0f);
        } else {
            const float4 det = (lv * rv) - (mv * mv);
            const float4 rdet = mk(1.0f) / det;
            const float lsdet = (lx * rz) - (my * my), lsrdet = 1.0f / lsdet;
            const float4 mss = ((lv * lv) + mk(2.0f) * (mv * mv)) + (rv * rv);
            const float lsmss = ((lx * lx) + 2.0f * (my * my)) + (rz * rz);
            const float4 ne0 = ((rv * colx) - (mv * coly)) * rdet;
            const float4 ne1 = ((lv * coly) - (mv * colx)) * rdet;
            if (fabsf(det.x) > (mss.x * 1e-4f) && ne0.x == ne0.x && ne1.x == ne1.x) { e0.x = ne0.x; e1.x = ne1.x; }
            if (fabsf(det.y) > (mss.y * 1e-4f) && ne0.y == ne0.y && ne1.y == ne1.y) { e0.y = ne0.y; e1.y = ne1.y; }
            if (fabsf(det.z) > (mss.z * 1e-4f) && ne0.z == ne0.z && ne1.z == ne1.z) { e0.z = ne0.z; e1.z = ne1.z; }
            if (fabsf(det.w) > (mss.w * 1e-4f) && ne0.w == ne0.w && ne1.w == ne1.w) { e0.w = ne0.w; e1.w = ne1.w; }
            const float se0 = ((rz * sv0) - (my * sv1)) * lsrdet;
            const float se1 = ((lx * sv1) - (my * sv0)) * lsrdet;
            if ((fabsf(lsdet) > (lsmss * 1e-4f)) && se0 == se0 && se1 == se1 && se0 < se1) {
                const float4 sdsm = sdir * se1;
                rgbs[q] = make_float4(sdsm.x, sdsm.y, sdsm.z, se0 / se1);
            }
        }
        st_ep(cs.ep[q], e0); st_ep(cs.ep[q] + 4, e1);
    }
    // ---------------- pass14: pack at the trial quant level, then the "mod" level
    {
        bool all_same = ci.ql != ci.qlm;
        uint32_t fn[4] = {0, 0, 0, 0}, vals[8];
        for (int i = 0; i < 32; i++) cs.packed[i] = 0;
#pragma unroll 1
        for (int q = 0; q < P; q++) {
            const uint32_t f = pk.pack(ld_ep(cs.ep[q]), ld_ep(cs.ep[q] + 4), rgbs[q], ci.fmt[q], ci.ql, vals);
            fn[0] = q == 0 ? f : fn[0]; fn[1] = q == 1 ? f : fn[1]; fn[2] = q == 2 ? f : fn[2]; fn[3] = q == 3 ? f : fn[3];
#pragma unroll
            for (int i = 0; i < 8; i++) cs.packed[q * 8 + i] = (uint8_t)vals[i];
            if (q > 0) all_same = all_same && f == fn[0];
        }
        bool m = false;
        if (P >= 2 && all_same) {
            uint32_t fm[4] = {0, 0, 0, 0};
            uint8_t* vm = packed_mod;
            bool same_mod = true;
#pragma unroll 1
            for (int q = 0; q < P; q++) {
                const uint32_t f = pk.pack(ld_ep(cs.ep[q]), ld_ep(cs.ep[q] + 4), rgbs[q], ci.fmt[q], ci.qlm, vals);
                fm[0] = q == 0 ? f : fm[0]; fm[1] = q == 1 ? f : fm[1]; fm[2] = q == 2 ? f : fm[2]; fm[3] = q == 3 ? f : fm[3];
#pragma unroll
                for (int i = 0; i < 8; i++) vm[q * 8 + i] = (uint8_t)vals[i];
                if (q > 0 && f != fm[0]) { same_mod = false; break; }
            }
            if (same_mod) {
                m = true;
#pragma unroll
                for (int q = 0; q < 4; q++) fn[q] = fm[q];
                for (int i = 0; i < 32; i++) cs.packed[i] = i < P * 8 ? vm[i] : 0;
            }
        }
        matched = m ? 1 : 0;
        final_q = m ? ci.qlm : ci.ql;
#pragma unroll
        for (int q = 0; q < 4; q++) ffmt[q] = fn[q];
    }
    // ---------------- pass15
#pragma unroll 1
    for (int q = 0; q < P; q++) unpack_endpoints(ffmt[q], cs.packed + q * 8, cs.u0[q], cs.u1[q]);
    if (it == 0) final_error();
    // ---------------- pass16: move each weight one quant step if that lowers the error
    bool moved = false;
    if (direct) {
        for (int t = 0; t < T; t++) {
            const int p = tp[t];
            const int32_t uqw = cs.qw[t];
            const uint32_t pn = tb.prev_next(bm.quant, uqw);
            const int32_t dn = pn & 0xFF, up = (pn >> 8) & 0xFF;
            const float4 base = make_float4((float)cs.u0[p][0], (float)cs.u0[p][1], (float)cs.u0[p][2], (float)cs.u0[p][3]);
            const float4 offs = make_float4((float)((int32_t)cs.u1[p][0] - (int32_t)cs.u0[p][0]), (float)((int32_t)cs.u1[p][1] - (int32_t)cs.u0[p][1]),
                                            (float)((int32_t)cs.u1[p][2] - (int32_t)cs.u0[p][2]), (float)((int32_t)cs.u1[p][3] - (int32_t)cs.u0[p][3])) * (1.0f / 64.0f);
            const float4 cd = (base + offs * (float)uqw) - px[t];
            const float4 cdd = cd + offs * (float)(dn - uqw), cdu = cd + offs * (float)(up - uqw);
            const float eb = dot4(cd * cd, cw), ed = dot4(cdd * cdd, cw), eu = dot4(cdu * cdu, cw);
            if ((eu < eb) && (eu < ed) && (uqw < 64)) { cs.qw[t] = (uint8_t)up; moved |= up != uqw; }
            else if ((ed < eb) && (uqw > 0)) { cs.qw[t] = (uint8_t)dn; moved |= dn != uqw; }
        }
    } else {
        for (int we = 0; we < dmi.W; we++) {
            const int32_t uqw = cs.qw[we];
            const uint32_t pn = tb.prev_next(bm.quant, uqw);
            const float dn = (float)(pn & 0xFF), up = (float)((pn >> 8) & 0xFF), ub = (float)uqw;
            const float ddn = dn - ub, dup = up - ub;
            float4 ebv = mk(0.0f), edv = mk(0.0f), euv = mk(0.0f);
            const int nt = tb.wt_count(bm.dm, we), wbase = dmi.wt_base + tb.wt_start(bm.dm, we);
            for (int te = 0; te < nt; te++) {
                // the weight's own contribution to texel t is the w2t entry's
                // (each (texel, weight) pair appears once in both maps)
                const uint32_t we2 = tb.w2t(wbase + te);
                const int t = we2 & 0xFF;
                const float twb = (float)(we2 >> 8) * (1.0f / 16.0f);
                const uint64_t e4 = tb.tw4(bm.dm, t);
                float wb = 0.0f;
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    const uint32_t e = (uint32_t)(e4 >> (16 * j)) & 0xFFFF;
                    wb = wb + (float)cs.qw[e & 0xFF] * ((float)(e >> 8) * (1.0f / 16.0f));
                }
                const int p = tp[t];
                const float4 base = make_float4((float)cs.u0[p][0], (float)cs.u0[p][1], (float)cs.u0[p][2], (float)cs.u0[p][3]);
                const float4 offs = make_float4((float)((int32_t)cs.u1[p][0] - (int32_t)cs.u0[p][0]), (float)((int32_t)cs.u1[p][1] - (int32_t)cs.u0[p][1]),
                                                (float)((int32_t)cs.u1[p][2] - (int32_t)cs.u0[p][2]), (float)((int32_t)cs.u1[p][3] - (int32_t)cs.u0[p][3])) * (1.0f / 64.0f);
                const float4 cd = (base + offs * wb) - px[t];
                const float4 cdd = cd + offs * (ddn * twb), cdu = cd + offs * (dup * twb);
                ebv = ebv + cd * cd; edv = edv + cdd * cdd; euv = euv + cdu * cdu;
            }
            const float eb = dot4(ebv, cw), ed = dot4(edv, cw), eu = dot4(euv, cw);
            if ((eu < eb) && (eu < ed) && (uqw < 64)) { cs.qw[we] = (uint8_t)up; moved |= (int32_t)up != uqw; }
            else if ((ed < eb) && (uqw > 0)) { cs.qw[we] = (uint8_t)dn; moved |= (int32_t)dn != uqw; }
        }
    }
    // In iteration 0 a pass16 that moved no weight leaves the weights and endpoints of the
    // error taken before it: the same total, which cannot improve the snapshot.
    if (it > 0 || moved) final_error();
    return moved;
}

// A refinement-tail entry: the partitioned block (lb * slots + slot), the candidate, the
// next iteration, then the state an iteration carries over (endpoints, weights; the best
// result so far is in the candidate's snapshot already).
__device__ __forceinline__ void write_tail(const KernelArgs& a, const CandSmem& c, uint32_t pbi, int k, int it, int pos) {
    uint4* e = a.tail + (size_t)pos * kTailWords;
    e[0] = make_uint4(pbi, (uint32_t)k | (uint32_t)it << 8, 0u, 0u);
    const uint8_t* ep = reinterpret_cast<const uint8_t*>(c.ep);
#pragma unroll
    for (int i = 0; i < 8; i++) e[1 + i] = ld_u4(ep + 16 * i);
#pragma unroll
    for (int i = 0; i < 4; i++) e[9 + i] = ld_u4(c.qw + 16 * i);
}
__device__ __forceinline__ void st_u4(uint8_t* p, uint4 v) {  // 4-byte aligned shared memory
    uint32_t* w = reinterpret_cast<uint32_t*>(p);
    w[0] = v.x; w[1] = v.y; w[2] = v.z; w[3] = v.w;
}

// CPB: candidate threads per partitioned block (refine_cpb of the launch's top-N), a
// template parameter so that the full search's instance (8) keeps constant indexing.
// U8: texels staged as RGBA8 (refine_u8).  Registers are capped for five resident CTAs
// (the packer's call would otherwise raise the whole kernel's allocation).
template <int CPB, bool U8>
__global__ void __launch_bounds__(kRefineThreads, 5) k_refine(const __grid_constant__ KernelArgs a) {
    extern __shared__ __align__(16) uint8_t smem[];
    const int T = a.L.T;
    constexpr int cpb = CPB;
    const int pbs = CPB == 8 ? kRefineThreads / 8 : refine_pbs(T, CPB);
    CandSmem* cs = reinterpret_cast<CandSmem*>(smem);
    float* lut = reinterpret_cast<float*>(smem + sizeof(CandSmem) * kRefineThreads);
    using Px = typename std::conditional<U8, uchar4, float4>::type;
    Px* pxs = reinterpret_cast<Px*>(U8 ? smem + sizeof(CandSmem) * kRefineThreads + 256 * 4 : smem + sizeof(CandSmem) * kRefineThreads);
    uint8_t* tps = reinterpret_cast<uint8_t*>(pxs + pbs * T);
    int* keys = reinterpret_cast<int*>(tps + ((pbs * T + 15) & ~15));
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    // Items: every slot of every block in slot-major order (consecutive CTAs hold
    // partitioned blocks of the same slot, hence the same partition count, so
    // co-resident warps run the same code), or the proposal pass's work list.
    const int nb = list_blocks(a);
    const int npb = a.pb_list ? pb_total(a) : nb * a.slots;
    const int ngroups = (npb + pbs - 1) / pbs;
    const int iters = a.refine_iters > 0 ? a.refine_iters : 6;
    __shared__ unsigned int refined[4];  // candidates refined by this CTA, by P (work counters)
    __shared__ int live_in_warp[kRefineThreads / 32];
    __shared__ int spill_base;
    if (tid < 4) refined[tid] = 0;
    bool spill = a.tail != nullptr && T <= kTailMaxTexels;  // until the tail is found full
    if (U8)
        for (int v = tid; v < 256; v += kRefineThreads) lut[v] = ((float)v / 255.0f) * 65536.0f;  // as src_texel
    // (the first group's barrier below orders these writes before any read)
    for (int grp = blockIdx.x; grp < ngroups; grp += gridDim.x) {
        {
            const int pbl = tid / cpb, k = tid % cpb;
            const int li = grp * pbs + pbl;
            int key = 0x3FFFFF;  // empty slots sort last
            uint32_t item = 0;
            if (pbl < pbs && li < npb) {
                int slot, lb;
                if (a.pb_list) pb_item(a, li, lb, slot);
                else { slot = li / nb; lb = li % nb; }
                item = (uint32_t)(lb + 1) | ((uint32_t)slot << 27);
                const PBRec& r = a.pbrec[lb * a.slots + slot];
                if (k < (int)r.ncand) {
                    const int dm = reinterpret_cast<const DevBm*>(a.tables + a.L.off_bm)[r.c[k].bm].dm;
                    int fk = 0;
                    for (int q = 0; q < 4; q++) { const int f = r.c[k].fmt[q]; fk = fk * 8 + (f == 0 ? 0 : f == 4 ? 1 : f == 6 ? 2 : f == 8 ? 3 : f == 10 ? 4 : f == 12 ? 5 : 6); }
                    key = ((((int)r.P - 1) << 12 | fk) << 7) | dm;  // partition count, formats, decimation mode
                }
                if (r.ncand > 0) {
                    const int P = r.P;
                    const uint8_t* prow = P > 1 ? a.tables + a.L.off_part_texel + ((size_t)(P - 2) * 1024 + r.entry) * T : nullptr;
                    const BlockSrc src = block_src(a, chunk_block(a, lb));
                    for (int t = k; t < T; t += cpb) {
                        if constexpr (U8) pxs[pbl * T + t] = src_rgba8(src, a.L.bx, t);
                        else pxs[pbl * T + t] = src_texel(src, a.L.bx, t);
                        tps[pbl * T + t] = P > 1 ? prow[t] : 0;
                    }
                }
            }
            keys[tid] = key * kRefineThreads + tid;  // unique keys: P, formats, decimation mode, then position
            cs[tid].item = item;  // of staging position tid
        }
        __syncthreads();
        // Thread tid takes the candidate of rank tid in (partition count, endpoint formats,
        // decimation mode) order, so a warp's candidates mostly take the same packing path
        // and share loop bounds and table rows.
        int cand = -1;  // staging position of the candidate this thread runs
        {
            const int kk = keys[tid];
            int rank = 0;
            for (int j = 0; j < kRefineThreads; j++) rank += keys[j] < kk;
            __syncthreads();
            keys[rank] = tid;
            __syncthreads();
            const int mine = keys[tid];
            const int pbl = mine / cpb, k = mine % cpb;
            const uint32_t item = cs[pbl * cpb].item;
            if (item != 0) {
                const int lb = (int)(item & 0x07FFFFFFu) - 1, slot = (int)(item >> 27);
                const size_t pbi = (size_t)lb * a.slots + slot;
                a.snaps[pbi * kNumCand + k].err = ERR_DEFAULT;  // inert slot unless refined below
                if (k < (int)a.pbrec[pbi].ncand) {
                    cand = mine;
                    if (a.work) atomicAdd(&refined[a.pbrec[pbi].P - 1], 1u);
                }
            }
        }
        // Iterations.  Candidates stop at different iterations (at a fixed point of pass16),
        // so after every iteration the live candidates are gathered onto the lowest threads,
        // in the same order: warps stay full while any work is left, and warps with none
        // wait at the barrier without issuing.  The staged texels and each candidate's state
        // stay where they are; only the candidate-to-thread map changes.
        for (int it = 0; ; it++) {
            const bool live = cand >= 0;
            const unsigned bal = __ballot_sync(0xFFFFFFFFu, live);
            if (lane == 0) live_in_warp[warp] = __popc(bal);
            __syncthreads();  // also: every thread has read keys[] before it is rewritten
            int nlive = 0, before = 0;
#pragma unroll
            for (int w = 0; w < kRefineThreads / 32; w++) {
                const int n = live_in_warp[w];
                nlive += n;
                before += w < warp ? n : 0;
            }
            if (nlive == 0) break;
            const int rank = before + __popc(bal & ((1u << lane) - 1u));
            if (spill && it > 0 && nlive <= a.spill_live) {
                // Few candidates left: hand them to the tail pass, which runs them densely, and
                // take the next group instead of holding the CTA for them.  The item words are
                // read before the barrier: after it, threads that are done stage the next group.
                uint32_t pbi = 0;
                if (live) {
                    const uint32_t item = cs[(cand / cpb) * cpb].item;
                    pbi = (uint32_t)((int)(item & 0x07FFFFFFu) - 1) * (uint32_t)a.slots + (item >> 27);
                }
                if (tid == 0) {
                    spill_base = atomicAdd(a.tail_count, nlive);
                    if (a.work) atomicAdd(a.work + 13, (unsigned long long)nlive);
                }
                __syncthreads();
                const int sb = spill_base, pos = sb + rank;
                if (sb + nlive <= a.tail_cap) {
                    // (the next group's staging writes no candidate state: ep and qw are first
                    // written by its iteration 0, after its barriers)
                    if (live) write_tail(a, cs[cand], pbi, cand % cpb, it, pos);
                    break;
                }
                if (live && pos < a.tail_cap) a.tail[(size_t)pos * kTailWords].x = 0xFFFFFFFFu;  // reserved, left empty
                spill = false;  // the tail is full: finish here
            }
            if (live) keys[rank] = cand;
            __syncthreads();
            cand = tid < nlive ? keys[tid] : -1;
            if (cand >= 0) {
                const int pbl = cand / cpb, k = cand % cpb;
                const uint32_t item = cs[pbl * cpb].item;
                const int lb = (int)(item & 0x07FFFFFFu) - 1, slot = (int)(item >> 27);
                const size_t pbi = (size_t)lb * a.slots + slot;
                const PBRec& rec = a.pbrec[pbi];
                Snap* snap = &a.snaps[pbi * kNumCand + k];
                bool moved;
                if constexpr (U8) moved = refine_step(a, rec, (int)rec.P, k, TexelRow<true>{pxs + pbl * T, lut}, tps + pbl * T, cs[cand], snap, it);
                else moved = refine_step(a, rec, (int)rec.P, k, TexelRow<false>{pxs + pbl * T}, tps + pbl * T, cs[cand], snap, it);
                if (!moved || it + 1 >= iters) cand = -1;
            }
            // (the next pass's first barrier orders this iteration's state writes before
            // other threads read them; the counts and the map were read before its second)
        }
    }
    if (a.work && tid < 4 && refined[tid]) atomicAdd(a.work + 6 + tid, (unsigned long long)refined[tid]);
}

// The candidates k_refine handed over, one per thread with its own staged texels (RGBA8
// through the table of src_texel's values, so every texel value is the same), iterated
// with the same gathering of live candidates onto the lowest threads.  The CTAs stay
// resident: a CTA's 128 slots are refilled whenever at most kTailRefillAt of them hold a
// live candidate, each warp claiming list entries for its own free slots from
// tail_count[1], and the new candidates join the live list behind the running ones.  (Fixed
// batches of 128 entries would hold each CTA until the slowest candidate of its batch ended.)
constexpr int kTailCtas = 4;
constexpr int kTailRefillAt = 64;
__global__ void __launch_bounds__(kRefineThreads, kTailCtas) k_refine_tail(const __grid_constant__ KernelArgs a) {
    extern __shared__ __align__(16) uint8_t smem[];
    const int T = a.L.T;
    CandSmem* cs = reinterpret_cast<CandSmem*>(smem);
    float* lut = reinterpret_cast<float*>(smem + sizeof(CandSmem) * kRefineThreads);
    uchar4* pxs = reinterpret_cast<uchar4*>(smem + sizeof(CandSmem) * kRefineThreads + 256 * 4);
    uint8_t* tps = reinterpret_cast<uint8_t*>(pxs + kRefineThreads * T);
    int* keys = reinterpret_cast<int*>(tps + ((kRefineThreads * T + 15) & ~15));
    int* next_it = keys + kRefineThreads;                                  // by slot
    uint32_t* pbi_of = reinterpret_cast<uint32_t*>(next_it + kRefineThreads);  // by slot
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const unsigned below = (1u << lane) - 1u;
    __shared__ int live_in_warp[kRefineThreads / 32], new_in_warp[kRefineThreads / 32];
    __shared__ uint8_t busy[kRefineThreads];  // slot holds a candidate that has not ended
    __shared__ int dry_flag;                  // the list has no unclaimed entry left
    for (int v = tid; v < 256; v += kRefineThreads) lut[v] = ((float)v / 255.0f) * 65536.0f;  // as src_texel
    busy[tid] = 0;
    if (tid == 0) dry_flag = 0;
    const int total = min(*a.tail_count, a.tail_cap);
    int* claim = a.tail_count + 1;
    const int iters = a.refine_iters > 0 ? a.refine_iters : 6;
    int cand = -1;     // the slot whose candidate this thread runs
    bool dry = false;  // CTA-uniform
    for (;;) {
        const bool live = cand >= 0;
        const unsigned bal = __ballot_sync(0xFFFFFFFFu, live);
        if (lane == 0) live_in_warp[warp] = __popc(bal);
        __syncthreads();  // also orders the last step's state writes and slot releases
        int nlive = 0, before = 0;
#pragma unroll
        for (int w = 0; w < kRefineThreads / 32; w++) {
            const int n = live_in_warp[w];
            nlive += n;
            before += w < warp ? n : 0;
        }
        int nnew = 0, new_before = 0, staged = -1;
        unsigned bnew = 0;
        if (!dry && nlive <= kTailRefillAt) {
            // Thread tid stages into slot tid when that slot is free and its warp's claim
            // reached an entry for it.
            const bool fr = busy[tid] == 0;
            const unsigned fb = __ballot_sync(0xFFFFFFFFu, fr);
            const int nfree = __popc(fb);
            int base = 0;
            if (lane == 0 && nfree > 0) base = atomicAdd(claim, nfree);
            base = __shfl_sync(0xFFFFFFFFu, base, 0);
            if (lane == 0 && nfree > 0 && base + nfree >= total) dry_flag = 1;
            const int idx = base + __popc(fb & below);
            if (fr && idx < total) {
                const uint4* e = a.tail + (size_t)idx * kTailWords;
                const uint4 h = e[0];
                if (h.x != 0xFFFFFFFFu) {
                    const int lb = (int)(h.x / (uint32_t)a.slots);
                    const PBRec& r = a.pbrec[h.x];
                    const int P = (int)r.P;
                    const uint8_t* prow = P > 1 ? a.tables + a.L.off_part_texel + ((size_t)(P - 2) * 1024 + r.entry) * T : nullptr;
                    const BlockSrc src = block_src(a, chunk_block(a, lb));
                    for (int t = 0; t < T; t++) {
                        pxs[tid * T + t] = src_rgba8(src, a.L.bx, t);
                        tps[tid * T + t] = P > 1 ? prow[t] : 0;
                    }
                    uint8_t* ep = reinterpret_cast<uint8_t*>(cs[tid].ep);
                    for (int i = 0; i < 8; i++) st_u4(ep + 16 * i, e[1 + i]);
                    for (int i = 0; i < 4; i++) st_u4(cs[tid].qw + 16 * i, e[9 + i]);
                    cs[tid].item = h.y & 0xFF;  // the candidate
                    next_it[tid] = (int)((h.y >> 8) & 0xFF);
                    pbi_of[tid] = h.x;
                    busy[tid] = 1;
                    staged = tid;
                }
            }
            bnew = __ballot_sync(0xFFFFFFFFu, staged >= 0);
            if (lane == 0) new_in_warp[warp] = __popc(bnew);
            __syncthreads();  // the staged slots, the new counts and the flag
#pragma unroll
            for (int w = 0; w < kRefineThreads / 32; w++) {
                const int n = new_in_warp[w];
                nnew += n;
                new_before += w < warp ? n : 0;
            }
            dry = dry_flag != 0;
        }
        const int n = nlive + nnew;
        if (n == 0) {
            if (dry) break;
            continue;  // every claimed entry was a reservation left empty: claim again
        }
        if (live) keys[before + __popc(bal & below)] = cand;
        if (staged >= 0) keys[nlive + new_before + __popc(bnew & below)] = staged;
        __syncthreads();
        cand = tid < n ? keys[tid] : -1;
        if (cand >= 0) {
            const uint32_t pbi = pbi_of[cand];
            const int k = (int)cs[cand].item, it = next_it[cand];
            const PBRec& rec = a.pbrec[pbi];
            Snap* snap = &a.snaps[(size_t)pbi * kNumCand + k];
            const bool moved = refine_step(a, rec, (int)rec.P, k, TexelRow<true>{pxs + cand * T, lut}, tps + cand * T, cs[cand], snap, it);
            next_it[cand] = it + 1;
            if (!moved || it + 1 >= iters) {
                busy[cand] = 0;  // released: read by the next refill, after the next barrier
                cand = -1;
            }
        }
    }
}

size_t refine_tail_smem_bytes(int T) {
    return sizeof(CandSmem) * kRefineThreads + 256 * 4 + (size_t)kRefineThreads * T * 4 +
           (((size_t)kRefineThreads * T + 15) & ~(size_t)15) + kRefineThreads * 4 * 3;
}

// ------------------------------------------------------------ k_select_pack
__device__ __forceinline__ void write_bits(uint32_t value, uint32_t count, uint32_t off, uint8_t* p) {
    uint32_t mask = (1u << count) - 1;
    value &= mask;
    p += off >> 3;
    off &= 7;
    value <<= off; mask <<= off; mask = ~mask;
    p[0] &= mask; p[0] |= value;
    p[1] &= mask >> 8; p[1] |= value >> 8;
}

__device__ void btq(int q, int& bits, int& trits, int& quints) {
    int L = c_levels_r[q];
    trits = quints = 0;
    if (L % 3 == 0) { trits = 1; L /= 3; } else if (L % 5 == 0) { quints = 1; L /= 5; }
    bits = 0;
    while ((1 << bits) < L) bits++;
}
__device__ uint32_t ise_bits(uint32_t n, int q) {
    int b, t, qu; btq(q, b, t, qu);
    if (t) return (n * (8 + 5 * b) + 4) / 5;
    if (qu) return (n * (7 + 3 * b) + 2) / 3;
    return n * b;
}

// encode_ise (code/physical_compression.cpp:672-826); out has 2 spare bytes.
__device__ void encode_ise(const TableLayout& L, const uint8_t* tabs, int q, uint32_t n, const uint8_t* in, uint8_t* out, uint32_t off) {
    int bits, trits, quints; btq(q, bits, trits, quints);
    const uint32_t mask = (1u << bits) - 1;
    const uint8_t* tt = tabs + L.off_trits;
    const uint8_t* qt = tabs + L.off_quints;
    if (trits) {
        const uint8_t tb[5] = {2, 2, 1, 2, 1}, ts[5] = {0, 2, 4, 5, 7};
        for (uint32_t i = 0; i < n; i += 5) {
            uint32_t d[5];
            for (int e = 0; e < 5; e++) d[e] = i + e < n ? (uint32_t)(in[i + e] >> bits) : 0;
            const uint32_t T = tt[(((d[4] * 3 + d[3]) * 3 + d[2]) * 3 + d[1]) * 3 + d[0]];
            for (int e = 0; e < 5 && i + e < n; e++) {
                const uint32_t pack = (in[i + e] & mask) | (((T >> ts[e]) & ((1u << tb[e]) - 1)) << bits);
                write_bits(pack, bits + tb[e], off, out);
                off += bits + tb[e];
            }
        }
    } else if (quints) {
        const uint8_t qb[3] = {3, 2, 2}, qs[3] = {0, 3, 5};
        for (uint32_t i = 0; i < n; i += 3) {
            uint32_t d[3];
            for (int e = 0; e < 3; e++) d[e] = i + e < n ? (uint32_t)(in[i + e] >> bits) : 0;
            const uint32_t Q = qt[(d[2] * 5 + d[1]) * 5 + d[0]];
            for (int e = 0; e < 3 && i + e < n; e++) {
                const uint32_t pack = (in[i + e] & mask) | (((Q >> qs[e]) & ((1u << qb[e]) - 1)) << bits);
                write_bits(pack, bits + qb[e], off, out);
                off += bits + qb[e];
            }
        }
    } else {
        for (uint32_t i = 0; i < n; i++) { write_bits(in[i], bits, off, out); off += bits; }
    }
}

__device__ __forceinline__ int bitrev8(int p) {
    p = ((p & 0x0F) << 4) | ((p >> 4) & 0x0F);
    p = ((p & 0x33) << 2) | ((p >> 2) & 0x33);
    p = ((p & 0x55) << 1) | ((p >> 1) & 0x55);
    return p;
}

__device__ __noinline__ void select_pack_one(const KernelArgs& a, int lb, int blk) {
    float best = 1e30f;
    int win_slot = -1, win_k = 0;
    // slots the front filled: all of them, or P=1 (unless skipped) plus the proposed partitionings
    const int nslots = a.prop ? 1 + (int)a.prop[lb].n : a.slots;
    const int s0 = a.prop && (a.prop[lb].flags & 1) ? 1 : 0;
    for (int s = s0; s < nslots; s++) {
        const PBRec& r = a.pbrec[(size_t)lb * a.slots + s];
        const int n = r.ncand;
        for (int k = 0; k < n; k++) {
            const float e = a.snaps[((size_t)lb * a.slots + s) * kNumCand + k].err;
            if (e < best) { best = e; win_slot = s; win_k = k; }
        }
    }
    if (win_slot < 0 && a.reroute_list) {  // proposal search found nothing: hand the block to the full search
        const int pos = atomicAdd(a.reroute_count, 1);
        a.reroute_list[pos] = blk;
        a.reroute_err[pos] = 3e38f;
        return;
    }
    if (a.prev_err && !(best < a.prev_err[lb])) return;  // the proposal search's result stands
    if (a.reroute_list && a.reroute_above > 0.0f && best > a.reroute_above) {
        // a poor proposal-search result: write it, and let the full search try to beat it
        const int pos = atomicAdd(a.reroute_count, 1);
        a.reroute_list[pos] = blk;
        a.reroute_err[pos] = best;
    }
    uint8_t blockbytes[18];
    uint32_t sym[8 + 4 + 32];  // header words of the SymbolicBlock record
    for (int i = 0; i < 18; i++) blockbytes[i] = 0;
    for (int i = 0; i < 44; i++) sym[i] = 0;
    const Snap* sn = nullptr;
    const PBRec* rec = nullptr;
    if (win_slot >= 0) {
        rec = &a.pbrec[(size_t)lb * a.slots + win_slot];
        sn = &a.snaps[((size_t)lb * a.slots + win_slot) * kNumCand + win_k];
        const DevBm bm = reinterpret_cast<const DevBm*>(a.tables + a.L.off_bm)[sn->bm];
        const DevDm dm = reinterpret_cast<const DevDm*>(a.tables + a.L.off_dm)[bm.dm];
        const uint32_t pc = rec->P, q = bm.quant;
        sym[0] = __float_as_uint(best); sym[1] = bm.mode_index; sym[2] = pc; sym[3] = rec->seed;
        sym[4] = sn->matched; sym[5] = sn->final_q;
        for (int i = 0; i < 4; i++) sym[8 + i] = sn->ffmt[i];
        for (int i = 0; i < 32; i++) sym[12 + i] = sn->packed[i];
        // weights: requantise 0..64 to the ISE alphabet, scramble, encode, bit-reverse
        const uint8_t* wscr = a.tables + a.L.off_wscr + q * 32;
        const float levels = (float)c_levels_r[q];
        uint8_t wv[64], wbuf[18];
        for (int i = 0; i < 18; i++) wbuf[i] = 0;
        for (int i = 0; i < dm.W; i++) {
            const float uqw = (float)sn->qw[i];
            const float qw = (uqw / 64.0f) * (levels - 1.0f);
            wv[i] = wscr[(int)(qw + 0.5f)];
        }
        const uint32_t wbits = ise_bits(dm.W, (int)q);
        encode_ise(a.L, a.tables, (int)q, dm.W, wv, wbuf, 0);
        for (int i = 0; i < 16; i++) blockbytes[i] = (uint8_t)bitrev8(wbuf[15 - i]);
        write_bits(bm.mode_index, 11, 0, blockbytes);
        write_bits(pc - 1, 2, 11, blockbytes);
        if (pc > 1) {
            write_bits(rec->seed, 6, 13, blockbytes);
            write_bits(rec->seed >> 6, 4, 19, blockbytes);
            if (sn->matched) {
                write_bits((uint32_t)sn->ffmt[0] << 2, 6, 23, blockbytes);
            } else {
                int low = 4;
                for (uint32_t i = 0; i < pc; i++) low = min((int)(sn->ffmt[i] >> 2), low);
                if (low == 3) low = 2;
                int et = low + 1, bp = 2;
                for (uint32_t i = 0; i < pc; i++) { et |= ((int)(sn->ffmt[i] >> 2) - low) << bp; bp++; }
                for (uint32_t i = 0; i < pc; i++) { et |= (int)(sn->ffmt[i] & 3) << bp; bp += 2; }
                const int hs = 3 * (int)pc - 4;
                write_bits(et & 0x3F, 6, 23, blockbytes);
                write_bits((uint32_t)et >> 6, hs, 128 - wbits - hs, blockbytes);
            }
        } else {
            write_bits(sn->ffmt[0], 4, 13, blockbytes);
        }
        const uint8_t* cscr = a.tables + a.L.off_cscr + (sn->final_q - 4) * 256;
        uint8_t vals[32];
        int nv = 0;
        for (uint32_t i = 0; i < pc; i++) {
            const int n = 2 * (sn->ffmt[i] >> 2) + 2;
            for (int j = 0; j < n; j++) vals[nv + j] = cscr[sn->packed[i * 8 + j]];
            nv += n;
        }
        encode_ise(a.L, a.tables, sn->final_q, nv, vals, blockbytes, pc == 1 ? 17 : 29);
    }
    uint4 o;
    o.x = blockbytes[0] | (blockbytes[1] << 8) | (blockbytes[2] << 16) | ((uint32_t)blockbytes[3] << 24);
    o.y = blockbytes[4] | (blockbytes[5] << 8) | (blockbytes[6] << 16) | ((uint32_t)blockbytes[7] << 24);
    o.z = blockbytes[8] | (blockbytes[9] << 8) | (blockbytes[10] << 16) | ((uint32_t)blockbytes[11] << 24);
    o.w = blockbytes[12] | (blockbytes[13] << 8) | (blockbytes[14] << 16) | ((uint32_t)blockbytes[15] << 24);
    *block_dst(a, blk) = o;
    if (a.symbolic) {
        uint32_t* s = a.symbolic + (size_t)blk * 108;
        if (win_slot < 0) sym[0] = __float_as_uint(1e30f);
        for (int i = 0; i < 44; i++) s[i] = sym[i];
        for (int i = 0; i < 64; i++) s[44 + i] = sn ? sn->qw[i] : 0;
    }
}

__global__ void __launch_bounds__(128) k_select_pack(const __grid_constant__ KernelArgs a) {
    const int nb = list_blocks(a);
    for (int lb = blockIdx.x * blockDim.x + threadIdx.x; lb < nb; lb += gridDim.x * blockDim.x)
        select_pack_one(a, lb, chunk_block(a, lb));
}

}  // namespace

namespace {

// ------------------------------------------------------------ optional encodings
// Encodings the reference never emits, enabled by ASTCB200_FLAG_VOID_EXTENT and
// ASTCB200_FLAG_DUAL_PLANE, applied to a chunk's blocks after the search has written them:
// a block whose texels are all equal becomes an LDR void-extent block; otherwise single-
// partition dual-plane encodings are tried (plane-2 component 0..3, every dual-plane block
// mode on a trial decimation mode) and the best replaces the search's block when its exact
// decoded error is lower.  The search's block is decoded with the library's decoder; the
// candidates' texels are computed the way a decoder produces them (integer weight infill,
// endpoints x257, integer interpolation, 16-bit to 8-bit rounding); errors are integer
// weighted squared differences (channel weights x 10^4).  One warp per block; the CPU
// oracle (orc_set_extensions) computes the same choices bit for bit.
constexpr int kExtWarps = 4;
__constant__ int c_cwi[4] = {6750, 13275, 2475, 10000};

struct ExtWarp {
    uchar4 c8[kMaxTexels];
    float w1[kMaxTexels], w2[kMaxTexels];
    float S[4][4];
    dec::Block kb;
    uint8_t qw[32][2][32];  // per lane: two planes of up to 32 grid weights
};

__device__ __forceinline__ int ext_dec8(int v16) { return (int)(((uint32_t)v16 * 255u + 32767u) / 65535u); }
__device__ __forceinline__ int ext_lerp(int e0, int e1, int w) { return (e0 * (64 - w) + e1 * w + 32) >> 6; }

// Integer infill of texel t from 0..64 grid weights (the specification's weights / 16).
__device__ __forceinline__ int ext_infill(const uint8_t* tabs, const TableLayout& L, int W, int dmi, const uint8_t* qw, int t) {
    if (W == L.T) return qw[t];
    const uint64_t e4 = reinterpret_cast<const uint64_t*>(tabs + L.off_tw4)[(size_t)dmi * L.T + t];
    int s = 0;
#pragma unroll
    for (int j = 0; j < 4; j++) {
        const uint32_t e = (uint32_t)(e4 >> (16 * j)) & 0xFFFF;
        s += (int)(e >> 8) * (int)qw[e & 0xFF];
    }
    return (s + 8) >> 4;
}

// Dual-plane candidate (ccs, dual mode j) from the warp's plane weights: its exact error
// (LLONG_MAX when no colour quant fits), and with phys != nullptr its block and symbolic words.
__device__ __noinline__ long long dual_candidate(const KernelArgs& a, const ExtWarp& ws, int ccs, int j, bool calpha,
                                                 const int* sum, uint8_t (*qw)[32], uint8_t* phys, uint32_t* sym) {
    const uint8_t* tabs = a.tables;
    const TableLayout& L = a.L;
    const int T = L.T;
    const DevBm bm = reinterpret_cast<const DevBm*>(tabs + L.off_dual)[j];
    const DevDm dm = reinterpret_cast<const DevDm*>(tabs + L.off_dm)[bm.dm];
    const int W = dm.W;
    const bool rgb_only = calpha && ccs != 3;
    const int nint = rgb_only ? 6 : 8, cem = rgb_only ? 8 : 12;
    const int avail = 109 - (int)bm.weight_bits;
    int qc = -1;
    for (int q = 20; q >= 4; q--)
        if ((int)ise_bits(nint, q) <= avail) { qc = q; break; }
    if (qc < 0) return LLONG_MAX;
    // decimate and quantise both planes (pass07's rule over [0, 1])
    const float qlm1 = (float)(c_levels_r[bm.quant] - 1);
    const uint8_t* q2u = tabs + L.off_q2u;
    const int qoff = tabs[L.off_q2u_start + bm.quant];
    for (int pl = 0; pl < 2; pl++) {
        const float* wv = pl ? ws.w2 : ws.w1;
        for (int i = 0; i < W; i++) {
            float dw;
            if (W == T) dw = wv[i];
            else {
                float num = 0.0f, den = 0.0f;
                const int n = tabs[L.off_wt_count + bm.dm * 64 + i];
                const int base = dm.wt_base + reinterpret_cast<const uint16_t*>(tabs + L.off_wt_start)[bm.dm * 64 + i];
                for (int k = 0; k < n; k++) {
                    const uint32_t e = reinterpret_cast<const uint16_t*>(tabs + L.off_w2t)[base + k];
                    const float c = (float)(e >> 8) * (1.0f / 16.0f);
                    num = num + c * wv[e & 0xFF];
                    den = den + c;
                }
                dw = num / den;
            }
            const float ix = fminf(fmaxf(dw, 0.0f), 1.0f), ix1 = ix * qlm1;
            const uint32_t wl = f2u(ix1), wh = min(wl + 1, f2u(qlm1));
            const uint32_t li = q2u[qoff + wl], hi = q2u[qoff + wh];
            qw[pl][i] = (uint8_t)(((float)li + (float)hi) < (128.0f * ix) ? hi : li);
        }
    }
    // endpoints per channel: least squares on the channel's plane
    float a1 = 0.0f, b1 = 0.0f, k1 = 0.0f, a2 = 0.0f, b2 = 0.0f, k2 = 0.0f;
    float s0[4] = {0.0f, 0.0f, 0.0f, 0.0f}, s1[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    for (int t = 0; t < T; t++) {
        const float w1 = (float)ext_infill(tabs, L, W, bm.dm, qw[0], t) / 64.0f;
        const float w2 = (float)ext_infill(tabs, L, W, bm.dm, qw[1], t) / 64.0f;
        const float o1 = 1.0f - w1, o2 = 1.0f - w2;
        a1 = a1 + o1 * o1; b1 = b1 + o1 * w1; k1 = k1 + w1 * w1;
        a2 = a2 + o2 * o2; b2 = b2 + o2 * w2; k2 = k2 + w2 * w2;
        const uchar4 x = ws.c8[t];
        const float xv[4] = {(float)x.x, (float)x.y, (float)x.z, (float)x.w};
#pragma unroll
        for (int ch = 0; ch < 4; ch++) {
            const float w = ch == ccs ? w2 : w1, o = ch == ccs ? o2 : o1;
            s0[ch] = s0[ch] + o * xv[ch];
            s1[ch] = s1[ch] + w * xv[ch];
        }
    }
    const uint8_t* cu2u = tabs + L.off_cu2u + (qc - 4) * 512;
    int ue[2][4];
#pragma unroll
    for (int ch = 0; ch < 4; ch++) {
        const float aa = ch == ccs ? a2 : a1, bb = ch == ccs ? b2 : b1, cc = ch == ccs ? k2 : k1;
        const float det = aa * cc - bb * bb;
        float e0, e1;
        if (det > 0.0001f * (aa * cc)) { e0 = (cc * s0[ch] - bb * s1[ch]) / det; e1 = (aa * s1[ch] - bb * s0[ch]) / det; }
        else { e0 = e1 = (float)sum[ch] / (float)T; }
        e0 = fminf(fmaxf(e0, 0.0f), 255.0f);
        e1 = fminf(fmaxf(e1, 0.0f), 255.0f);
        ue[0][ch] = cu2u[(int)rintf(e0) * 2 + 1];
        ue[1][ch] = cu2u[(int)rintf(e1) * 2 + 1];
    }
    if (rgb_only) { ue[0][3] = 255; ue[1][3] = 255; }
    if (ue[1][0] + ue[1][1] + ue[1][2] < ue[0][0] + ue[0][1] + ue[0][2]) {  // the decoder would swap
#pragma unroll
        for (int ch = 0; ch < 4; ch++) { const int t = ue[0][ch]; ue[0][ch] = ue[1][ch]; ue[1][ch] = t; }
        for (int pl = 0; pl < 2; pl++)
            for (int i = 0; i < W; i++) qw[pl][i] = (uint8_t)(64 - qw[pl][i]);
    }
    long long err = 0;
    for (int t = 0; t < T; t++) {
        const int w1 = ext_infill(tabs, L, W, bm.dm, qw[0], t), w2 = ext_infill(tabs, L, W, bm.dm, qw[1], t);
        const uchar4 x = ws.c8[t];
        const int xv[4] = {x.x, x.y, x.z, x.w};
#pragma unroll
        for (int ch = 0; ch < 4; ch++) {
            const int d = xv[ch] - ext_dec8(ext_lerp(ue[0][ch] * 257, ue[1][ch] * 257, ch == ccs ? w2 : w1));
            err += (long long)c_cwi[ch] * (long long)(d * d);
        }
    }
    if (phys) {
        for (int i = 0; i < 108; i++) sym[i] = 0;
        sym[0] = __float_as_uint((float)err * 1e-4f);
        sym[1] = bm.mode_index; sym[2] = 1; sym[5] = (uint32_t)qc; sym[6] = 1u + (uint32_t)ccs; sym[8] = (uint32_t)cem;
        for (int ch = 0; ch < nint / 2; ch++) { sym[12 + 2 * ch] = (uint32_t)ue[0][ch]; sym[13 + 2 * ch] = (uint32_t)ue[1][ch]; }
        for (int i = 0; i < W; i++) { sym[44 + i] = qw[0][i]; sym[76 + i] = qw[1][i]; }
        // physical block: interleaved plane weights, mode, partition count, format, plane-2
        // component below the weights, colour values (single partition)
        const int q = bm.quant;
        const uint8_t* wscr = tabs + L.off_wscr + q * 32;
        const float levels = (float)c_levels_r[q];
        uint8_t wv[64], wbuf[18];
        for (int i = 0; i < 18; i++) wbuf[i] = 0;
        for (int i = 0; i < W; i++) {
            wv[2 * i] = wscr[(int)((((float)qw[0][i]) / 64.0f) * (levels - 1.0f) + 0.5f)];
            wv[2 * i + 1] = wscr[(int)((((float)qw[1][i]) / 64.0f) * (levels - 1.0f) + 0.5f)];
        }
        const uint32_t wbits = ise_bits(2 * W, q);
        encode_ise(L, tabs, q, 2 * W, wv, wbuf, 0);
        for (int i = 0; i < 16; i++) phys[i] = (uint8_t)bitrev8(wbuf[15 - i]);
        write_bits(bm.mode_index, 11, 0, phys);
        write_bits(0, 2, 11, phys);
        write_bits((uint32_t)cem, 4, 13, phys);
        write_bits((uint32_t)ccs, 2, 128 - wbits - 2, phys);
        const uint8_t* cscr = tabs + L.off_cscr + (qc - 4) * 256;
        uint8_t vals[8];
        for (int k = 0; k < nint; k++) vals[k] = cscr[sym[12 + k]];
        encode_ise(L, tabs, qc, nint, vals, phys, 17);
    }
    return err;
}

__global__ void __launch_bounds__(kExtWarps * 32) k_extend(const __grid_constant__ KernelArgs a, int flags) {
    __shared__ ExtWarp wsm[kExtWarps];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    ExtWarp& ws = wsm[warp];
    const int T = a.L.T, bx = a.L.bx, by = a.L.by;
    constexpr unsigned FULL = 0xffffffffu;
    for (int lb = blockIdx.x * kExtWarps + warp; lb < a.nblocks; lb += gridDim.x * kExtWarps) {
        const int blk = chunk_block(a, lb);
        if (blk < 0) continue;
        const BlockSrc src = block_src(a, blk);
        for (int t = lane; t < T; t += 32) ws.c8[t] = src_rgba8(src, bx, t);
        __syncwarp();
        const uchar4 c0 = ws.c8[0];
        bool same = true, opaque = true, const_a = true;
        int sum[4] = {0, 0, 0, 0};
        for (int t = lane; t < T; t += 32) {
            const uchar4 x = ws.c8[t];
            same = same && x.x == c0.x && x.y == c0.y && x.z == c0.z && x.w == c0.w;
            opaque = opaque && x.w == 255;
            const_a = const_a && x.w == c0.w;
            sum[0] += x.x; sum[1] += x.y; sum[2] += x.z; sum[3] += x.w;
        }
        same = __all_sync(FULL, same);
        opaque = __all_sync(FULL, opaque);
        const_a = __all_sync(FULL, const_a);
#pragma unroll
        for (int ch = 0; ch < 4; ch++) sum[ch] = __reduce_add_sync(FULL, sum[ch]);
        uint4* dst = block_dst(a, blk);
        if (same && (flags & 1)) {  // LDR void-extent block of the colour x 257, no extent
            if (lane == 0) {
                *dst = make_uint4(0xFFFFFDFCu, 0xFFFFFFFFu, (uint32_t)c0.x * 0x101u | ((uint32_t)c0.y * 0x101u) << 16,
                                  (uint32_t)c0.z * 0x101u | ((uint32_t)c0.w * 0x101u) << 16);
                if (a.symbolic) {
                    uint32_t* s = a.symbolic + (size_t)blk * 108;
                    for (int i = 0; i < 108; i++) s[i] = 0;
                    s[2] = 1; s[7] = 1; s[12] = c0.x; s[13] = c0.y; s[14] = c0.z; s[15] = c0.w;
                }
            }
            __syncwarp();
            continue;
        }
        if (!(flags & 2)) { __syncwarp(); continue; }
        // exact error of the search's block, decoded
        if (lane == 0) {
            const uint4 v = *dst;
            uint8_t raw[16];
            const uint32_t wv4[4] = {v.x, v.y, v.z, v.w};
            for (int i = 0; i < 16; i++) raw[i] = (uint8_t)(wv4[i >> 2] >> (8 * (i & 3)));
            dec::parse_block(raw, bx, by, ws.kb);
        }
        __syncwarp();
        long long es = 0;
        for (int t = lane; t < T; t += 32) {
            uint16_t v16[4];
            dec::texel16(ws.kb, bx, by, t % bx, t / bx, v16);
            const uchar4 x = ws.c8[t];
            const int xv[4] = {x.x, x.y, x.z, x.w};
#pragma unroll
            for (int ch = 0; ch < 4; ch++) {
                const int d = xv[ch] - (int)dec::to_unorm8(v16[ch]);
                es += (long long)c_cwi[ch] * (long long)(d * d);
            }
        }
        for (int o = 16; o > 0; o >>= 1) es += __shfl_xor_sync(FULL, es, o);
        // dual-plane candidates: plane-2 component outer, block modes inner
        long long best = LLONG_MAX;
        int best_idx = 0x7FFFFFFF;
        const int nd = a.L.ndual;
        for (int pass = 0; pass < 2; pass++) {
            int ccs_lo = 0, ccs_hi = 3, win_ccs = -1, win_j = -1;
            if (pass == 1) {  // the winner's plane weights again, then its encoding
                long long b = best;
                int bi = best_idx;
                for (int o = 16; o > 0; o >>= 1) {
                    const long long ob = __shfl_xor_sync(FULL, b, o);
                    const int oi = __shfl_xor_sync(FULL, bi, o);
                    if (ob < b || (ob == b && oi < bi)) { b = ob; bi = oi; }
                }
                if (!(b < es)) break;  // the search's block stays
                win_ccs = bi / nd; win_j = bi % nd;
                ccs_lo = ccs_hi = win_ccs;
            }
            for (int ccs = ccs_lo; ccs <= ccs_hi; ccs++) {
                if (ccs == 3 && const_a) continue;
                float mu[4];
#pragma unroll
                for (int ch = 0; ch < 4; ch++) mu[ch] = (float)sum[ch] / (float)T;
                if (lane < 4 && lane != ccs) {  // positive-deviation sums along axis `lane`, in texel order
                    float Sx = 0.0f, Sy = 0.0f, Sz = 0.0f, Sw = 0.0f;
                    for (int t = 0; t < T; t++) {
                        const uchar4 x = ws.c8[t];
                        const float d0 = ccs == 0 ? 0.0f : (float)x.x - mu[0], d1 = ccs == 1 ? 0.0f : (float)x.y - mu[1];
                        const float d2 = ccs == 2 ? 0.0f : (float)x.z - mu[2], d3 = ccs == 3 ? 0.0f : (float)x.w - mu[3];
                        const float dl = lane == 0 ? d0 : lane == 1 ? d1 : lane == 2 ? d2 : d3;
                        if (dl > 0.0f) { Sx = Sx + d0; Sy = Sy + d1; Sz = Sz + d2; Sw = Sw + d3; }
                    }
                    ws.S[lane][0] = Sx; ws.S[lane][1] = Sy; ws.S[lane][2] = Sz; ws.S[lane][3] = Sw;
                }
                __syncwarp();
                int bax = -1;
                float bl = 0.0f;
                for (int ax = 0; ax < 4; ax++) {
                    if (ax == ccs) continue;
                    float l = ws.S[ax][0] * ws.S[ax][0];
                    l = l + ws.S[ax][1] * ws.S[ax][1];
                    l = l + ws.S[ax][2] * ws.S[ax][2];
                    l = l + ws.S[ax][3] * ws.S[ax][3];
                    if (l > bl) { bl = l; bax = ax; }
                }
                float dir[4] = {0.0f, 0.0f, 0.0f, 0.0f};
                if (bax >= 0) {
                    const float len = sqrtf(bl);
#pragma unroll
                    for (int ch = 0; ch < 4; ch++) dir[ch] = ws.S[bax][ch] / len;
                }
                float pmin = 1e30f, pmax = -1e30f;
                int vmin = 255, vmax = 0;
                for (int t = lane; t < T; t += 32) {
                    const uchar4 x = ws.c8[t];
                    const float d0 = ccs == 0 ? 0.0f : (float)x.x - mu[0], d1 = ccs == 1 ? 0.0f : (float)x.y - mu[1];
                    const float d2 = ccs == 2 ? 0.0f : (float)x.z - mu[2], d3 = ccs == 3 ? 0.0f : (float)x.w - mu[3];
                    float v = d0 * dir[0];
                    v = v + d1 * dir[1];
                    v = v + d2 * dir[2];
                    v = v + d3 * dir[3];
                    ws.w1[t] = v;
                    pmin = fminf(pmin, v); pmax = fmaxf(pmax, v);
                    const int c = ccs == 0 ? x.x : ccs == 1 ? x.y : ccs == 2 ? x.z : x.w;
                    vmin = min(vmin, c); vmax = max(vmax, c);
                }
                for (int o = 16; o > 0; o >>= 1) {
                    pmin = fminf(pmin, __shfl_xor_sync(FULL, pmin, o)); pmax = fmaxf(pmax, __shfl_xor_sync(FULL, pmax, o));
                    vmin = min(vmin, __shfl_xor_sync(FULL, vmin, o)); vmax = max(vmax, __shfl_xor_sync(FULL, vmax, o));
                }
                for (int t = lane; t < T; t += 32) {
                    const uchar4 x = ws.c8[t];
                    const int c = ccs == 0 ? x.x : ccs == 1 ? x.y : ccs == 2 ? x.z : x.w;
                    ws.w1[t] = pmax > pmin ? (ws.w1[t] - pmin) / (pmax - pmin) : 0.0f;
                    ws.w2[t] = vmax > vmin ? (float)(c - vmin) / (float)(vmax - vmin) : 0.0f;
                }
                __syncwarp();
                if (pass == 0) {
                    for (int j = lane; j < nd; j += 32) {
                        const long long e = dual_candidate(a, ws, ccs, j, opaque, sum, ws.qw[lane], nullptr, nullptr);
                        if (e < best) { best = e; best_idx = ccs * nd + j; }
                    }
                } else if (lane == 0) {
                    uint8_t phys[18];
                    uint32_t sym[108];
                    for (int i = 0; i < 18; i++) phys[i] = 0;
                    dual_candidate(a, ws, win_ccs, win_j, opaque, sum, ws.qw[0], phys, sym);
                    *dst = make_uint4(phys[0] | (phys[1] << 8) | (phys[2] << 16) | ((uint32_t)phys[3] << 24),
                                      phys[4] | (phys[5] << 8) | (phys[6] << 16) | ((uint32_t)phys[7] << 24),
                                      phys[8] | (phys[9] << 8) | (phys[10] << 16) | ((uint32_t)phys[11] << 24),
                                      phys[12] | (phys[13] << 8) | (phys[14] << 16) | ((uint32_t)phys[15] << 24));
                    if (a.symbolic) {
                        uint32_t* s = a.symbolic + (size_t)blk * 108;
                        for (int i = 0; i < 108; i++) s[i] = sym[i];
                    }
                }
                __syncwarp();  // the next plane-2 component overwrites the plane weights
            }
        }
        __syncwarp();
    }
}

}  // namespace

cudaError_t launch_extend(const KernelArgs& a, int flags, cudaStream_t s) {
    if (!(flags & 3)) return cudaSuccess;
    int grid = (a.nblocks + kExtWarps - 1) / kExtWarps;
    if (a.block_list) grid = std::min(grid, kListGridPack);
    if (grid <= 0) return cudaSuccess;
    k_extend<<<grid, kExtWarps * 32, 0, s>>>(a, flags);
    return cudaGetLastError();
}

size_t refine_smem_bytes(const TableLayout& L, int topn) {
    const size_t pbs = (size_t)refine_pbs(L.T, topn);
    const bool u8 = refine_u8(L.T);
    return sizeof(CandSmem) * kRefineThreads + (u8 ? 256 * 4 : 0) + pbs * L.T * (u8 ? 4 : 16) + ((pbs * L.T + 15) & ~(size_t)15) +
           kRefineThreads * 4;
}

size_t refine_smem_bytes(const TableLayout& L) {  // the largest over the refinement top-N
    size_t m = 0;
    for (int topn : {1, 2, 4, 8}) m = std::max(m, refine_smem_bytes(L, topn));
    return m;
}

cudaError_t configure_search_kernels(size_t search_bytes, size_t front_bytes);
constexpr int kMaxConfigDevices = 64;

// The dynamic shared-memory limit is a per-function attribute shared by every
// context and thread of the process; it only ever grows (per device), so
// launches for different footprints may be queued concurrently.
cudaError_t configure_kernels(const TableLayout& L) {
    static std::mutex mu;
    static size_t limit[kMaxConfigDevices][3];
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxConfigDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> g(mu);
    size_t* m = limit[dev];
    const size_t need[3] = {search_smem_bytes(L), front_smem_bytes(L), refine_smem_bytes(L)};
    if (need[0] <= m[0] && need[1] <= m[1] && need[2] <= m[2]) return cudaSuccess;
    for (int i = 0; i < 3; i++) m[i] = std::max(m[i], need[i]);
    e = configure_search_kernels(m[0], m[1]);
    if (e != cudaSuccess) return e;
    for (auto f : {k_refine<1, false>, k_refine<2, false>, k_refine<4, false>, k_refine<8, false>, k_refine<1, true>,
                   k_refine<2, true>, k_refine<4, true>, k_refine<8, true>})
        if ((e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)m[2])) != cudaSuccess) return e;
    return cudaFuncSetAttribute(k_refine_tail, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)refine_tail_smem_bytes(kTailMaxTexels));
}

cudaError_t launch_refine(const KernelArgs& a, cudaStream_t s) {
    const int cpb = refine_cpb(a.topn);
    const int npb = a.nblocks * a.slots, pbs = refine_pbs(a.L.T, cpb);
    int grid = (npb + pbs - 1) / pbs;
    if (a.block_list) grid = std::min(grid, kListGridRefine);
    const size_t smem = refine_smem_bytes(a.L, cpb);
    if (refine_u8(a.L.T)) {
        if (cpb == 1) k_refine<1, true><<<grid, kRefineThreads, smem, s>>>(a);
        else if (cpb == 2) k_refine<2, true><<<grid, kRefineThreads, smem, s>>>(a);
        else if (cpb == 4) k_refine<4, true><<<grid, kRefineThreads, smem, s>>>(a);
        else k_refine<8, true><<<grid, kRefineThreads, smem, s>>>(a);
    } else {
        if (cpb == 1) k_refine<1, false><<<grid, kRefineThreads, smem, s>>>(a);
        else if (cpb == 2) k_refine<2, false><<<grid, kRefineThreads, smem, s>>>(a);
        else if (cpb == 4) k_refine<4, false><<<grid, kRefineThreads, smem, s>>>(a);
        else k_refine<8, false><<<grid, kRefineThreads, smem, s>>>(a);
    }
    return cudaGetLastError();
}

cudaError_t launch_refine_tail(const KernelArgs& a, cudaStream_t s) {
    if (!a.tail || a.L.T > kTailMaxTexels) return cudaSuccess;
    const int grid = std::min((a.tail_cap + kRefineThreads - 1) / kRefineThreads, 148 * kTailCtas);
    k_refine_tail<<<std::max(grid, 1), kRefineThreads, refine_tail_smem_bytes(a.L.T), s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_select_pack(const KernelArgs& a, cudaStream_t s) {
    int grid = (a.nblocks + 127) / 128;
    if (a.block_list) grid = std::min(grid, kListGridPack);
    k_select_pack<<<grid, 128, 0, s>>>(a);
    return cudaGetLastError();
}

}  // namespace astcb200
