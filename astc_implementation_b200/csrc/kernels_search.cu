// Partition search and front-end kernels of the ASTC encoder (sm_100a).
//
//   k_partition_search  passes 001-007 (shaders/pass001..pass007): k-means over
//                       the block's texels, coverage mismatch against every
//                       selected partitioning, the reference's bitonic ordering,
//                       error estimate of 128 candidates, pick of 4.
//                       One warp per (block, partition count).
//   k_front             passes 01-12 (shaders/pass01..pass12) for one
//                       partitioned block per CTA: ideal endpoints, per
//                       decimation-mode weight solving, per block-mode weight
//                       quantisation error, colour-format search, top-8 pick.
//
// Sums whose order the reference leaves to float atomics are taken in ascending
// texel / weight order, each by one thread or lane, so results are bit-identical
// to the CPU oracle (oracle/astc_oracle.cpp), which fixes the same order; integer
// sums, whose order does not matter, may be split or regrouped.
#include <algorithm>

#include "device_math.cuh"
#include "kernels.h"

namespace astcb200 {

using namespace dev;

namespace {

constexpr unsigned FULL = 0xffffffffu;
constexpr float ERR_DEFAULT = 1e37f;
__constant__ int c_levels[21] = {2, 3, 4, 5, 6, 8, 10, 12, 16, 20, 24, 32, 40, 48, 64, 80, 96, 128, 160, 192, 256};
__constant__ int c_steps_for_quant[12] = {2, 3, 4, 5, 6, 8, 10, 12, 16, 20, 24, 32};
__constant__ int c_free_bits[4] = {111, 97, 94, 91};  // pass07:5
// pass10's format-class combinations (i | j << 2 | k << 4 | l << 6) for P = 2, 3, 4: every
// tuple of classes 0..3 whose classes lie within one of each other (the pass's i, j, k, l
// loops with their skips), grouped by the total i + j + k + l and, inside a total, in loop
// order; c_combo_off[P - 2][c] .. [c + 1] delimits total c.
__constant__ uint8_t c_combo[78] = {
    0, 4, 1, 5, 9, 6, 10, 14, 11, 15,                                                      // P = 2
    0, 16, 4, 1, 20, 17, 5, 21, 37, 25, 22, 41, 38, 26, 42, 58, 46, 43, 62, 59, 47, 63,     // P = 3
    0, 64, 16, 4, 1, 80, 68, 20, 65, 17, 5, 84, 81, 69, 21, 85, 149, 101, 89, 86, 165, 153,  // P = 4
    105, 150, 102, 90, 169, 166, 154, 106, 170, 234, 186, 174, 171, 250, 238, 190, 235, 187, 175,
    254, 251, 239, 191, 255};
__constant__ uint8_t c_combo_off[3][14] = {{0, 1, 3, 4, 6, 7, 9, 10, 10, 10, 10, 10, 10, 10},
                                           {10, 11, 14, 17, 18, 21, 24, 25, 28, 31, 32, 32, 32, 32},
                                           {32, 33, 37, 43, 47, 48, 52, 58, 62, 63, 67, 73, 77, 78}};

enum { FMT_LUMINANCE = 0, FMT_LUMINANCE_ALPHA = 4, FMT_RGB_SCALE = 6, FMT_RGB = 8, FMT_RGB_SCALE_ALPHA = 10, FMT_RGBA = 12 };

struct Tabs {
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
    __device__ int bm_order(int j) const { return reinterpret_cast<const uint16_t*>(b + L->off_bm_order)[j]; }
    __device__ const uint8_t* part_texels(int P, int e) const { return b + L->off_part_texel + ((size_t)(P - 2) * 1024 + e) * L->T; }
    __device__ int part_count(int P, int e, int q) const { return b[L->off_part_counts + ((P - 2) * 1024 + e) * 4 + q]; }
    __device__ uint32_t part_seed(int P, int e) const { return reinterpret_cast<const uint32_t*>(b + L->off_part_info)[(P - 2) * 1024 + e]; }
    __device__ uint64_t cov(int P, int e, int q) const { return reinterpret_cast<const uint64_t*>(b + L->off_cov)[((size_t)(P - 2) * 1024 + e) * 4 + q]; }
    __device__ float sin_t(int i) const { return reinterpret_cast<const float*>(b + L->off_sin)[i]; }
    __device__ float cos_t(int i) const { return reinterpret_cast<const float*>(b + L->off_cos)[i]; }
    __device__ int q2u(int i) const { return b[L->off_q2u + i]; }
    __device__ int q2u_start(int q) const { return b[L->off_q2u_start + q]; }
    __device__ int qmt(int row, int bits) const { return reinterpret_cast<const int8_t*>(b + L->off_qmt)[row * 128 + bits]; }
    __device__ float bqe(int i) const { return reinterpret_cast<const float*>(b + L->off_bqe)[i]; }
};

__device__ __forceinline__ float dist_sq(float4 a, float4 b) {
    const float4 d = a - b;
    return dot4(d * d, chan_w());
}

// ============================================================ passes 001-007
constexpr int kSearchWarps = 4;
// Per warp: texels, 1024 sort keys, 128 + 128 candidate errors, k-means assignments, then
// (FIXED semantics) the 128 first keys of the full order and a 132-bin histogram.
constexpr int kSearchWarpBytes = 144 * 16 + 1024 * 8 + 128 * 4 * 2 + 160 + 128 * 8 + 132 * 4;

// FIXED semantics of pass005 (full sort): the first 128 of all 1024 keys m << 32 | i in
// ascending order, into ord.  The mismatch counts m of the sel selected entries are at most
// 128 (the sum of P popcounts of 64-bit words, halved), so a stable counting sort by m in
// index order gives the full order; entries i >= sel (m = 0xFFFFFFFF) keep rank i.
__device__ void full_order(const unsigned long long* key, unsigned long long* ord, uint32_t* hist, uint32_t sel, int lane) {
    for (int b = lane; b < 132; b += 32) hist[b] = 0;
    __syncwarp();
    for (uint32_t i = lane; i < sel; i += 32) atomicAdd(&hist[(uint32_t)(key[i] >> 32)], 1u);
    __syncwarp();
    uint32_t v[5], s = 0;  // exclusive scan of bins 0..128, five per lane
#pragma unroll
    for (int j = 0; j < 5; j++) { const int b = lane * 5 + j; v[j] = b < 129 ? hist[b] : 0u; s += v[j]; }
    uint32_t incl = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) { const uint32_t t = __shfl_up_sync(FULL, incl, o); if (lane >= o) incl += t; }
    uint32_t run = incl - s;
    __syncwarp();
#pragma unroll
    for (int j = 0; j < 5; j++) { const int b = lane * 5 + j; if (b < 129) hist[b] = run; run += v[j]; }
    __syncwarp();
    const uint32_t lt = (1u << lane) - 1u;
    const uint32_t end = sel > 128u ? sel : 128u;
    for (uint32_t base = 0; base < end; base += 32) {
        const uint32_t i = base + lane;
        const unsigned long long k = key[i];
        const uint32_t m = (uint32_t)(k >> 32);
        const bool selected = i < sel;
        const uint32_t grp = __match_any_sync(FULL, selected ? m : 0xFFFFFFFFu);
        const uint32_t rank = selected ? hist[m] + __popc(grp & lt) : i;
        if (rank < 128u) ord[rank] = k;
        __syncwarp();
        if (selected && 31 - __clz(grp) == lane) hist[m] += __popc(grp);
        __syncwarp();
    }
    __syncwarp();
}

template <int P>
__device__ void search_one(const KernelArgs& a, int blk, int lb, uint8_t* ws, int lane) {
    const Tabs tb{a.tables, &a.L};
    const int T = a.L.T;
    float4* px = reinterpret_cast<float4*>(ws);
    unsigned long long* key = reinterpret_cast<unsigned long long*>(ws + 144 * 16);
    float* eu = reinterpret_cast<float*>(ws + 144 * 16 + 1024 * 8);
    float* es = eu + 128;
    uint8_t* asg = reinterpret_cast<uint8_t*>(es + 128);
    unsigned long long* ord_buf = reinterpret_cast<unsigned long long*>(ws + 144 * 16 + 1024 * 8 + 128 * 4 * 2 + 160);
    uint32_t* hist = reinterpret_cast<uint32_t*>(ord_buf + 128);
    const BlockSrc src = block_src(a, blk);
    for (int t = lane; t < T; t += 32) px[t] = src_texel(src, a.L.bx, t);
    __syncwarp();

    // pass001: farthest-point initial centres; ties pick the highest texel index
    float4 c[P];
    c[0] = px[145897 % T];
    float dist[5];
#pragma unroll
    for (int j = 0; j < 5; j++) { const int t = lane + 32 * j; dist[j] = t < T ? dist_sq(c[0], px[t]) : 0.0f; }
#pragma unroll
    for (int pp = 1; pp < P; pp++) {
        uint32_t mx = 0;
#pragma unroll
        for (int j = 0; j < 5; j++) if (lane + 32 * j < T) mx = max(mx, fbits(dist[j]));
        mx = __reduce_max_sync(FULL, mx);
        int idx = -1;
#pragma unroll
        for (int j = 0; j < 5; j++) if (lane + 32 * j < T && fbits(dist[j]) == mx) idx = lane + 32 * j;
        idx = __reduce_max_sync(FULL, idx);
        c[pp] = px[idx];
        if (pp < P - 1) {
#pragma unroll
            for (int j = 0; j < 5; j++) { const int t = lane + 32 * j; if (t < T) dist[j] = fminf(dist[j], dist_sq(c[pp], px[t])); }
        }
    }
    // passes 002/003, four iterations
    uint32_t as[5];
    for (int it = 0; it < 4; it++) {
#pragma unroll
        for (int j = 0; j < 5; j++) {
            const int t = lane + 32 * j;
            as[j] = 0;
            if (t < T) {
                float best = 1e30f;
#pragma unroll
                for (int q = 0; q < P; q++) { const float d = dist_sq(px[t], c[q]); if (d < best) { best = d; as[j] = q; } }
            }
        }
        bool problem = false;
#pragma unroll
        for (int q = 0; q < P; q++) {
            int n = 0;
#pragma unroll
            for (int j = 0; j < 5; j++) n += __popc(__ballot_sync(FULL, lane + 32 * j < T && as[j] == (uint32_t)q));
            if (n == 0) problem = true;
        }
        if (problem && lane < P) as[0] = lane;
#pragma unroll
        for (int q = 0; q < P; q++) {
            uint32_t n = 0, s0 = 0, s1 = 0, s2 = 0, s3 = 0;
#pragma unroll
            for (int j = 0; j < 5; j++) {
                const int t = lane + 32 * j;
                if (t < T && as[j] == (uint32_t)q) {
                    n++; s0 += f2u(px[t].x); s1 += f2u(px[t].y); s2 += f2u(px[t].z); s3 += f2u(px[t].w);
                }
            }
            n = __reduce_add_sync(FULL, n);
            s0 = __reduce_add_sync(FULL, s0); s1 = __reduce_add_sync(FULL, s1);
            s2 = __reduce_add_sync(FULL, s2); s3 = __reduce_add_sync(FULL, s3);
            if (n > 0) {
                const float fc = (float)n;
                c[q] = make_float4((float)s0 / fc, (float)s1 / fc, (float)s2 / fc, (float)s3 / fc);
            } else {
                c[q] = mk(0.0f);
            }
        }
    }
#pragma unroll
    for (int j = 0; j < 5; j++) { const int t = lane + 32 * j; if (t < T) asg[t] = (uint8_t)as[j]; }
    __syncwarp();
    // pass004: k-means bitmaps over the 64 k-means texels, mismatch per partitioning
    uint64_t km[P];
    {
        const int k0 = asg[a.L.kmeans[lane]], k1 = asg[a.L.kmeans[lane + 32]];
#pragma unroll
        for (int q = 0; q < P; q++) {
            const uint32_t lo = __ballot_sync(FULL, k0 == q), hi = __ballot_sync(FULL, k1 == q);
            km[q] = (uint64_t)lo | ((uint64_t)hi << 32);
        }
    }
    const uint32_t sel = a.L.count_selected[P - 1];
    for (int i = lane; i < 1024; i += 32) {
        uint32_t m = 0xFFFFFFFFu;
        if ((uint32_t)i < sel) {
            uint32_t p[P][P];
#pragma unroll
            for (int x = 0; x < P; x++)
#pragma unroll
                for (int y = 0; y < P; y++) p[x][y] = __popcll(km[x] ^ tb.cov(P, i, y));
            if (P == 2) {
                m = min(p[0][0] + p[1][1], p[0][1] + p[1][0]) / 2;
            } else if (P == 3) {
                const uint32_t v0 = min(p[1][1] + p[2][2], p[1][2] + p[2][1]) + p[0][0];
                const uint32_t v1 = min(p[1][0] + p[2][2], p[1][2] + p[2][0]) + p[0][1];
                const uint32_t v2 = min(p[1][0] + p[2][1], p[1][1] + p[2][0]) + p[0][2];
                m = min(v0, min(v1, v2)) / 2;
            } else {
                const uint32_t mx23 = min(p[2][2] + p[3][3], p[2][3] + p[3][2]);
                const uint32_t mx13 = min(p[2][1] + p[3][3], p[2][3] + p[3][1]);
                const uint32_t mx12 = min(p[2][1] + p[3][2], p[2][2] + p[3][1]);
                const uint32_t mx03 = min(p[2][0] + p[3][3], p[2][3] + p[3][0]);
                const uint32_t mx02 = min(p[2][0] + p[3][2], p[2][2] + p[3][0]);
                const uint32_t mx01 = min(p[2][1] + p[3][0], p[2][0] + p[3][1]);
                const uint32_t v0 = p[0][0] + min(p[1][1] + mx23, min(p[1][2] + mx13, p[1][3] + mx12));
                const uint32_t v1 = p[0][1] + min(p[1][0] + mx23, min(p[1][2] + mx03, p[1][3] + mx02));
                const uint32_t v2 = p[0][2] + min(p[1][1] + mx03, min(p[1][0] + mx13, p[1][3] + mx01));
                const uint32_t v3 = p[0][3] + min(p[1][1] + mx02, min(p[1][2] + mx01, p[1][0] + mx12));
                m = min(v0, min(v1, min(v2, v3))) / 2;
            }
        }
        key[i] = ((unsigned long long)m << 32) | (uint32_t)i;
    }
    __syncwarp();
    // pass005: the reference's bitonic network run by 256 invocations (a partial sort); FIXED
    // semantics: the full order
    const unsigned long long* ord = key;
    if (a.fixed) {
        full_order(key, ord_buf, hist, sel, lane);
        ord = ord_buf;
    }
    for (unsigned k = 2; k <= 1024 && !a.fixed; k <<= 1)
        for (unsigned j = k >> 1; j > 0; j >>= 1) {
#pragma unroll
            for (int r = 0; r < 8; r++) {
                const unsigned l = lane + 32 * r, partner = l ^ j;
                if (partner > l) {
                    const bool asc = (l & k) == 0;
                    const unsigned long long x = key[l], y = key[partner];
                    if ((x > y) == asc) { key[l] = y; key[partner] = x; }
                }
            }
            __syncwarp();
        }
    // pass006: error estimate of the first 128 ordered partitionings.  The
    // shader keeps avg/dir in per-invocation arrays, so texel t only sees its
    // own partition's average/direction when t < P and its partition is t.
    float wie = T <= 20 ? 0.03f : T <= 31 ? 0.04f : T <= 41 ? 0.05f : 0.055f;
    wie = wie * wie;
    const float4 cw = chan_w();
    uint32_t u_all = 0;  // sum over all texels of f2u(|x|^2 weighted), the line error of a zero direction
    for (int t = lane; t < T; t += 32) { const float4 x = px[t]; u_all += f2u(dot4(x * x, cw)); }
    for (int o = 16; o > 0; o >>= 1) u_all += __shfl_xor_sync(FULL, u_all, o);
    for (int r = 0; r < 4; r++) {
        const int cand = lane + 32 * r;
        const int e = (int)(uint32_t)ord[cand];
        const uint8_t* row = tb.part_texels(P, e);
        uint32_t cnt[P], sm[P][4];
#pragma unroll
        for (int q = 0; q < P; q++) { cnt[q] = 0; sm[q][0] = sm[q][1] = sm[q][2] = sm[q][3] = 0; }
        for (int t = 0; t < T; t++) {
            const int p = row[t];
            const float4 x = px[t];
            const uint32_t u0 = f2u(x.x), u1 = f2u(x.y), u2 = f2u(x.z), u3 = f2u(x.w);
#pragma unroll
            for (int q = 0; q < P; q++) if (p == q) { cnt[q]++; sm[q][0] += u0; sm[q][1] += u1; sm[q][2] += u2; sm[q][3] += u3; }
        }
        float4 tavg[P], tdir[P];
#pragma unroll
        for (int q = 0; q < P; q++) {
            const float fc = (float)cnt[q];
            tavg[q] = fc > 0.0f ? make_float4((float)sm[q][0] / fc, (float)sm[q][1] / fc, (float)sm[q][2] / fc, (float)sm[q][3] / fc) : mk(0.0f);
        }
#pragma unroll
        for (int q = 0; q < P; q++) {
            uint32_t ax[4][4];
#pragma unroll
            for (int u = 0; u < 4; u++) ax[u][0] = ax[u][1] = ax[u][2] = ax[u][3] = 0;
            for (int t = 0; t < T; t++) {
                if (row[t] != q) continue;
                const float4 av = (a.fixed || t == q) ? tavg[q] : mk(0.0f);
                const float4 d = px[t] - av;
                const uint32_t d0 = (uint32_t)f2i(d.x), d1 = (uint32_t)f2i(d.y), d2 = (uint32_t)f2i(d.z), d3 = (uint32_t)f2i(d.w);
                if (d.x > 0.0f) { ax[0][0] += d0; ax[0][1] += d1; ax[0][2] += d2; ax[0][3] += d3; }
                if (d.y > 0.0f) { ax[1][0] += d0; ax[1][1] += d1; ax[1][2] += d2; ax[1][3] += d3; }
                if (d.z > 0.0f) { ax[2][0] += d0; ax[2][1] += d1; ax[2][2] += d2; ax[2][3] += d3; }
                if (d.w > 0.0f) { ax[3][0] += d0; ax[3][1] += d1; ax[3][2] += d2; ax[3][3] += d3; }
            }
            float4 s[4];
#pragma unroll
            for (int u = 0; u < 4; u++) s[u] = make_float4((float)(int32_t)ax[u][0], (float)(int32_t)ax[u][1], (float)(int32_t)ax[u][2], (float)(int32_t)ax[u][3]);
            float4 best = s[0];
            float mp = dot4(s[0], s[0]);
#pragma unroll
            for (int u = 1; u < 4; u++) { const float pr = dot4(s[u], s[u]); if (pr > mp) { mp = pr; best = s[u]; } }
            tdir[q] = normalize4(best);
        }
        // Every texel but those t < P of partition t sees a zero average and direction: its
        // projection is 0, its line error |x|^2 (weighted) and its scale error NaN (the zero
        // direction's normalisation), so f2u gives 0xFFFFFFFF.  The integer sums take those
        // terms for every texel at once (u_all, -T) and the loop corrects the few texels
        // that see their partition's own average and direction; integer sums do not depend
        // on their order.
        uint32_t usum = u_all, ssum = 0u - (uint32_t)T;
        int32_t lmin[P], lmax[P];
#pragma unroll
        for (int q = 0; q < P; q++) { lmin[q] = 2147483647; lmax[q] = -2147483647; }
        if (a.fixed) {  // every texel sees its partition's average and direction
            float4 sdir[P];
#pragma unroll
            for (int q = 0; q < P; q++) sdir[q] = normalize4(tavg[q]);
            usum = 0u; ssum = 0u;
            for (int t = 0; t < T; t++) {
                const int p = row[t];
                float4 av = tavg[0], ud = tdir[0], sd = sdir[0];
#pragma unroll
                for (int q = 1; q < P; q++) if (p == q) { av = tavg[q]; ud = tdir[q]; sd = sdir[q]; }
                const float4 x = px[t];
                const float up = dot4(x, ud);
                const float4 uproj = av + ud * dot4(x - av, ud);
                const float4 udiff = x - uproj;
                usum += f2u(dot4(udiff * udiff, cw));
                const float4 sproj = sd * dot4(x, sd);
                const float4 sdiff = x - sproj;
                ssum += f2u(dot4(sdiff * sdiff, cw));
                const int32_t upi = f2i(up * 4096.0f);
#pragma unroll
                for (int q = 0; q < P; q++) if (p == q) { lmin[q] = min(lmin[q], upi); lmax[q] = max(lmax[q], upi); }
            }
        }
#pragma unroll
        for (int t = 0; t < P && !a.fixed; t++) {
            if (row[t] != t) continue;
            const float4 av = tavg[t], ud = tdir[t];
            const float4 x = px[t];
            usum -= f2u(dot4(x * x, cw));
            ssum += 1u;
            const float up = dot4(x, ud);
            const float4 uproj = av + ud * dot4(x - av, ud);
            const float4 udiff = x - uproj;
            const float ud2 = dot4(udiff * udiff, cw);
            const float4 sd = normalize4(av);
            const float4 sproj = sd * dot4(x, sd);
            const float4 sdiff = x - sproj;
            const float sd2 = dot4(sdiff * sdiff, cw);
            usum += f2u(ud2);
            ssum += f2u(sd2);
            const int32_t upi = f2i(up * 4096.0f);
            lmin[t] = min(lmin[t], upi); lmax[t] = max(lmax[t], upi);
        }
#pragma unroll
        for (int q = 0; q < P; q++)  // the partition has a texel of projection 0
            if (!a.fixed && tb.part_count(P, e, q) > (row[q] == q ? 1 : 0)) { lmin[q] = min(lmin[q], 0); lmax[q] = max(lmax[q], 0); }
        float tu = (float)usum, ts = (float)ssum;
#pragma unroll
        for (int q = 0; q < P; q++) {
            const float mn = (float)lmin[q] / 4096.0f, mxv = (float)lmax[q] / 4096.0f;
            const float ll = fmaxf(mxv - mn, 1e-7f);
            const float ew = (float)tb.part_count(P, e, q) * wie;
            tu = tu + ew * (ll * ll);
            const float4 a0 = (q == 0 || a.fixed) ? tavg[q] : mk(0.0f);
            ts = ts + ew * dot4(a0, a0);
        }
        eu[cand] = tu;
        es[cand] = ts;
    }
    __syncwarp();
    // pass007: best 4 by each error, interleaved and deduplicated; the rank is
    // used as the table entry (REF-BUG-4, pass007:93,156)
    if (lane == 0) {
        uint32_t bui[4] = {0, 0, 0, 0}, bsi[4] = {0, 0, 0, 0};
        float bue[4] = {1e30f, 1e30f, 1e30f, 1e30f}, bse[4] = {1e30f, 1e30f, 1e30f, 1e30f};
        for (int i = 0; i < 128; i++) {
            const float u = eu[i], s = es[i];
            if (u < bue[3]) {
                bue[3] = u; bui[3] = i;
                for (int j = 3; j > 0; j--)
                    if (bue[j] < bue[j - 1]) { float te = bue[j]; bue[j] = bue[j - 1]; bue[j - 1] = te; uint32_t ti = bui[j]; bui[j] = bui[j - 1]; bui[j - 1] = ti; }
            }
            if (s < bse[3]) {
                bse[3] = s; bsi[3] = i;
                for (int j = 3; j > 0; j--)
                    if (bse[j] < bse[j - 1]) { float te = bse[j]; bse[j] = bse[j - 1]; bse[j - 1] = te; uint32_t ti = bsi[j]; bsi[j] = bsi[j - 1]; bsi[j - 1] = ti; }
            }
        }
        uint32_t fin[4] = {0, 0, 0, 0};
        int emitted = 0;
        for (int i = 0; i < 8 && emitted < 4; i++) {
            const uint32_t idx = (i & 1) ? bsi[i >> 1] : bui[i >> 1];
            bool seen = false;
            for (int j = 0; j < emitted; j++) seen |= fin[j] == idx;
            if (!seen) fin[emitted++] = idx;
        }
        uint16_t* out = a.picks[lb].v + (P - 2) * 5;
        // FIXED semantics: the table entry the candidate was evaluated for
        for (int i = 0; i < 4; i++) out[i] = (uint16_t)(a.fixed && i < emitted ? (uint32_t)ord[fin[i]] : fin[i]);
        out[4] = (uint16_t)emitted;
    }
}

__global__ void __launch_bounds__(kSearchWarps * 32) k_partition_search(const __grid_constant__ KernelArgs a) {
    extern __shared__ __align__(16) uint8_t smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    uint8_t* ws = smem + warp * kSearchWarpBytes;
    const int nb = list_blocks(a);
    // P-major items: a CTA's warps share P; one pass for a chunk, a grid-stride loop over a block list
    for (int item = blockIdx.x * kSearchWarps + warp; item < nb * 3; item += gridDim.x * kSearchWarps) {
        const int lb = item % nb, P = item / nb + 2;
        const int blk = chunk_block(a, lb);
        if (P == 2) search_one<2>(a, blk, lb, ws, lane);
        else if (P == 3) search_one<3>(a, blk, lb, ws, lane);
        else search_one<4>(a, blk, lb, ws, lane);
        if (a.work && lane == 0) atomicAdd(a.work + 10 + (P - 2), 1ull);
        __syncwarp();
    }
}

// ============================================================ passes 01-12
// One CTA of NT threads per partitioned block: 128 for the full search; the proposal
// search, whose partitioned blocks evaluate few block modes, may use 64 or 32 so that more
// of them are resident per SM.  Every value is computed by the same thread sequence
// whatever NT is (loops only spread independent items), so results do not depend on it.

struct FrontLayout {
    int px, w, wes, tp, dec, lo, hi, scratch, bm_err, bm_bits, ccr_tot, ccr_q, ccr_fmt, qf, misc, dml, bml, total;
};

// Scratch of passes 02-05 per half-warp: the pass03 table indices [64], angular offsets
// [16], pass05 keys [16] (u64) and minidx [16].  pass02's infilled weights (T floats per
// half-warp) go to pass07's buffer, unused between pass08's sums and pass07.
constexpr int kDmScratchHalf = 64 * 4 + 16 * 4 + 16 * 8 + 16 * 4;
constexpr int kDmScratchPerWarp = 2 * kDmScratchHalf;

struct FrontMisc {
    float4 avg[4], dir[4], ep0[4], ep1[4];
    float mn[4], mx[4], lsq[4];
    float min_cutoff;
    uint32_t is_const, gray, calpha;
    uint32_t ece_can_offset[4], ece_can_bc[4];
    float p9[4][4];  // pass09 inputs per partition: rre, are, brgb, ba
    float sxyz[4][3][4];  // pass08: per partition, sums of the deviations along r, g, b (w = 0)
    float acc[4][5];      // pass08: per partition, the five encoding-choice error sums
    float4 axes[4][4];    // pass08: per partition, ub, ua, sb, la
    float cerr[4][21][4];
    uint8_t cfmt[4][21][4];
    float combo_err[21][13];
    uint8_t combo_fmt[21][13][4];
    int top[kNumCand];
    int ncand;
    int nlive;  // block modes in the proposal search's list
};

// pass07's buffer in floats, before pass02 also the texel channels and projections,
// then pass08's error terms (5 x Tp; Tp = T rounded up to 4).  The full search's
// pass07 takes one thread per mode (max_w x nt); the proposal search's (`list`) works on
// groups of kListGroup modes (max_w + Tp each), so its launches need less shared memory
// and more of its CTAs fit on an SM.
constexpr int kListGroup = 16;
__host__ __device__ inline int front_layout_qf_floats(int T, int max_w, int nt, bool list) {
    const int Tp = (T + 3) & ~3;
    int f = list ? kListGroup * (max_w + Tp) : max_w * nt;
    if (f < 5 * Tp) f = 5 * Tp;
    if (f < (nt / 32) * 2 * T) f = (nt / 32) * 2 * T;  // pass02's infill, two modes per warp
    return f;
}
__host__ __device__ inline int take16(int& o, int bytes) { const int r = o; o = (o + bytes + 15) & ~15; return r; }
__host__ __device__ inline FrontLayout front_layout(int T, int ndm, int nbm, int max_w, int nt, bool list) {
    FrontLayout f;
    int o = 0;
    f.px = take16(o, T * 16);
    f.w = take16(o, T * 4);
    f.wes = take16(o, T * 4);
    f.tp = take16(o, T);
    f.dec = take16(o, ndm * 64 * 4);
    f.lo = take16(o, ndm * 8 * 4);
    f.hi = take16(o, ndm * 8 * 4);
    f.scratch = take16(o, (nt / 32) * kDmScratchPerWarp);
    f.bm_err = take16(o, nbm * 4);
    f.bm_bits = take16(o, nbm * 4);
    f.ccr_tot = take16(o, nbm * 4);
    f.ccr_q = take16(o, nbm * 2);
    f.ccr_fmt = take16(o, nbm * 4);
    f.qf = take16(o, front_layout_qf_floats(T, max_w, nt, list) * 4);
    f.misc = take16(o, (int)sizeof(FrontMisc));
    f.dml = take16(o, 16 + ndm * 2);
    f.bml = take16(o, nbm * 2);  // the proposal search's block modes, ascending
    f.total = o;
    return f;
}

// Quantised weight w of block mode bmi given the dm's ideal decimated weights
// (pass06 range rules + pass07:230-275).  Returns the unquantised value on the
// 0..64 scale and writes the rescaled float weight.
struct BmQuant {
    float low, scale, slb, rscale, qlm1;
    int q2u_start, quant;
};
__device__ __forceinline__ BmQuant bm_quant_setup(const Tabs& tb, const DevBm& bm, const float* lo, const float* hi, float min_cutoff) {
    float low = lo[bm.quant < 8 ? bm.quant : 0], high = hi[bm.quant < 8 ? bm.quant : 0];
    if (bm.quant >= 8) { low = 0.0f; high = 0.0f; }  // pass05 never writes slots 8..12 (REF-BUG-5 buffer read as 0)
    if (high > 1.02f * min_cutoff) high = 1.0f;
    if (high <= low) { low = 0.0f; high = 1.0f; }
    BmQuant r;
    r.qlm1 = (float)(c_levels[bm.quant] - 1);
    float rscale = high - low;
    r.scale = 1.0f / rscale;
    r.slb = low * r.scale;
    r.rscale = rscale / 64.0f;
    r.low = low;
    r.q2u_start = tb.q2u_start(bm.quant);
    r.quant = bm.quant;
    return r;
}
__device__ __forceinline__ int bm_quant_weight(const Tabs& tb, const BmQuant& s, float ideal, float* qf) {
    const float ix = clampf(ideal * s.scale - s.slb, 0.0f, 1.0f);
    const float ix1 = ix * s.qlm1;
    const uint32_t wl = f2u(ix1), wh = min(wl + 1, f2u(s.qlm1));
    const int li = tb.q2u(s.q2u_start + wl), hi = tb.q2u(s.q2u_start + wh);
    const bool uh = ((float)li + (float)hi) < (128.0f * ix);
    const int v = uh ? hi : li;
    *qf = (float)v * s.rscale + s.low;
    return v;
}

// pass02 of one decimation mode by a half-warp (lane gl of 16): the ideal decimated
// weights dw, then for decimated modes the infill and the one-step correction.  Every lane
// of the warp takes the syncs (both halves run this together, each on its own mode).
__device__ __forceinline__ void pass02_mode(const Tabs& tb, int T, int m, const DevDm& dmi, int W, bool act, int gl, float* inf,
                                            const float* iw, const float* wes, bool is_const, float* dw) {
    if (W == T || !act) {
        for (int w = gl; w < W; w += 16) dw[w] = iw[w];
    } else {
        for (int w = gl; w < W; w += 16) {
            const int n = tb.wt_count(m, w);
            float v = 0.0f;
            if (n) {
                const int base = dmi.wt_base + tb.wt_start(m, w);
                float ws = 0.0f, tc = 1e-10f;
                for (int j = 0; j < n; j++) {
                    const uint32_t e = tb.w2t(base + j);
                    const int t = e & 0xFF;
                    const float cwt = ((float)(e >> 8) * (1.0f / 16.0f)) * wes[is_const ? 0 : t];
                    ws = ws + iw[t] * cwt;
                    tc = tc + cwt;
                }
                v = ws / tc;
            }
            dw[w] = v;
        }
    }
    const bool decim = act && W != T;
    __syncwarp();
    if (decim) {
        for (int t = gl; t < T; t += 16) {
            // the texel's entries in list order; padding entries add dw[0] * 0, which never changes v
            const uint64_t e4 = tb.tw4(m, t);
            float v = 0.0f;
#pragma unroll
            for (int j = 0; j < 4; j++) { const uint32_t e = (uint32_t)(e4 >> (16 * j)) & 0xFFFF; v = v + dw[e & 0xFF] * ((float)(e >> 8) * (1.0f / 16.0f)); }
            inf[t] = v;
        }
    }
    __syncwarp();
    if (decim) {
        for (int w = gl; w < W; w += 16) {
            const int n = tb.wt_count(m, w), base = dmi.wt_base + tb.wt_start(m, w);
            float e0 = 1e-10f, e1 = 0.0f;
            for (int j = 0; j < n; j++) {
                const uint32_t e = tb.w2t(base + j);
                const int t = e & 0xFF;
                const float c = (float)(e >> 8) * (1.0f / 16.0f);
                const float sc = wes[is_const ? 0 : t] * c;
                e0 = e0 + c * sc;
                e1 = e1 + (inf[t] - iw[t]) * sc;
            }
            dw[w] = dw[w] + clampf((e1 * -16.0f) / e0, -0.25f, 0.25f);
        }
    }
}

// Passes 02-05 for the decimation modes of a partitioned block, a half-warp per mode, two
// modes per warp at a time (passes 03-05 need at most 16 lanes: 16 angular steps at most,
// 12 for every valid mode).  Every lane of a warp runs the same number of loop trips (a
// half without a mode idles), so the warp-wide __syncwarp()s are reached by all of its
// lanes.
template <int kFrontWarps>
__device__ __forceinline__ void dm_passes(const Tabs& tb, int T, const FrontLayout& fl, uint8_t* sm, int ndm_run,
                                          const int16_t* dm_run, const float* iw, const float* wes, bool is_const,
                                          float* dec, float* lov, float* hiv, float* infbuf) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int half = lane >> 4, hl = lane & 15;
    float* inf = infbuf + (warp * 2 + half) * T;
    uint8_t* hs = sm + fl.scratch + warp * kDmScratchPerWarp + half * kDmScratchHalf;
    uint32_t* smp = reinterpret_cast<uint32_t*>(hs);
    float* ang = reinterpret_cast<float*>(hs + 64 * 4);
    float* lh = reinterpret_cast<float*>(hs + 64 * 4 + 16 * 4);  // pass05 keys [16] (u64), minidx [16]
    for (int mb = warp * 2; mb < ndm_run; mb += kFrontWarps * 2) {
        const int mi = mb + half;
        const bool act = mi < ndm_run;
        const int m = act ? (dm_run ? dm_run[mi] : mi) : 0;
        const DevDm dmi = tb.dm(m);
        const int W = act ? (int)dmi.W : 0;
        float* dw = dec + m * 64;
        pass02_mode(tb, T, m, dmi, W, act, hl, inf, iw, wes, is_const, dw);
        __syncwarp();
        for (int w = hl; w < W; w += 16) smp[w] = f2u(rintf(clampf(dw[w], 0.0f, 1.0f) * (1024.0f - 1.0f)));
        __syncwarp();
        // pass03: angular offsets
        if (act) {
            // table values fetched four at a time, then summed in weight order
            float ax = 0.0f, ay = 0.0f;
            int j = 0;
            for (; j + 4 <= W; j += 4) {
                float c[4], sn[4];
#pragma unroll
                for (int u = 0; u < 4; u++) { const int k = smp[j + u] * 16 + hl; c[u] = tb.cos_t(k); sn[u] = tb.sin_t(k); }
#pragma unroll
                for (int u = 0; u < 4; u++) { ax = ax + c[u]; ay = ay + sn[u]; }
            }
            for (; j < W; j++) { const int k = smp[j] * 16 + hl; ax = ax + tb.cos_t(k); ay = ay + tb.sin_t(k); }
            ang[hl] = atan2_search(ay, ax) * (1.0f / (2.0f * 3.14159265358979323846f));
        }
        __syncwarp();
        // pass04 + pass05: lane i < S evaluates angular step i (rounding error and cut
        // errors over the weights) and offers its candidates to the weight spans the
        // sequential scan of pass05 would update with them: span sp takes e, sp - 1 takes
        // e + cl and then e + ch, sp - 2 takes e + cl + ch, each only when strictly below the
        // span's best so far (initially 1e37), steps in ascending order.  That scan keeps,
        // per span, the first minimum in this order, which is the smallest key
        //   error bits << 32 | step << 2 | order within the step << 1 | low-cut flag:
        // errors are sums of non-negative products (never -0.0f, NaN or 1e37), so their
        // bit patterns order like their values.  Only spans 0..15 are read (q <= 7 needs
        // span c_steps_for_quant[q] <= 12; S <= 12 for every valid decimation mode).
        const int S = act ? (int)dmi.max_angular_steps : 0;
        unsigned long long* best = reinterpret_cast<unsigned long long*>(lh);  // [16]
        float* lmin = lh + 32;                                                 // [16] minidx per step
        best[hl] = ~0ull;
        __syncwarp();
        if (hl < S) {
            float mnw = 3.4e38f, mxw = -3.4e38f;
            for (int j = 0; j < W; j++) { const float v = dw[j]; if (v < mnw) mnw = v; if (v > mxw) mxw = v; }
            const float rcp = (float)(hl + 1), off = ang[hl];
            const float minidx = rintf(mnw * rcp - off), maxidx = rintf(mxw * rcp - off);
            float ev = 0.0f, cl = 0.0f, ch = 0.0f;
            for (int j = 0; j < W; j++) {
                const float sv = dw[j] * rcp - off, r = rintf(sv), d = sv - r;
                ev = ev + d * d;
                cl = cl + (r == minidx ? 1.0f - (2.0f * d) : 0.0f);
                ch = ch + (r == maxidx ? 1.0f + (2.0f * d) : 0.0f);
            }
            const int sp = min(max(f2i((maxidx - minidx) + 1.0f), 2), (int)dmi.max_quant_steps + 3);
            const float ss = 1.0f / rcp, esc = ss * ss;
            const float e = ev * esc, ecl0 = cl * esc, ech0 = ch * esc;
            const float ecl = e + ecl0, ech = e + ech0, eclh = (e + ecl0) + ech0;
            lmin[hl] = minidx;
            const unsigned long long ik = (unsigned long long)hl << 2;
            if (sp < 16 && e < 1e37f) atomicMin(&best[sp], ((unsigned long long)__float_as_uint(e) << 32) | ik);
            if (sp - 1 < 16 && ecl < 1e37f) atomicMin(&best[sp - 1], ((unsigned long long)__float_as_uint(ecl) << 32) | ik | 1ull);
            if (sp - 1 < 16 && ech < 1e37f) atomicMin(&best[sp - 1], ((unsigned long long)__float_as_uint(ech) << 32) | ik | 2ull);
            if (sp - 2 < 16 && eclh < 1e37f) atomicMin(&best[sp - 2], ((unsigned long long)__float_as_uint(eclh) << 32) | ik | 1ull);
        }
        __syncwarp();
        // pass05: low/high value per quant level from the best step of its span (step 0
        // and no low cut when no candidate got below 1e37)
        if (act && hl < 8) {
            const int q = hl;
            float lo_v = 0.0f, hi_v = 0.0f;
            if (q <= (int)dmi.max_quant_level) {
                const int qs = c_steps_for_quant[q];
                const unsigned long long k = best[qs];
                const int bsi = k == ~0ull ? 0 : (int)(((uint32_t)k) >> 2);
                const float lwi = lmin[bsi] + ((k != ~0ull && (k & 1ull)) ? 1.0f : 0.0f);
                const float hwi = (lwi + (float)qs) - 1.0f;
                const float step = 1.0f / (1.0f + (float)bsi);
                const float off = ang[bsi];
                lo_v = (off + lwi) * step;
                hi_v = (off + hwi) * step;
            }
            lov[m * 8 + q] = lo_v;
            hiv[m * 8 + q] = hi_v;
        }
        __syncwarp();
    }
}

// Code of the full search only (every block mode) is kept out of line, so that the
// proposal search's path through the front stays compact in the instruction cache (the
// front stalls on instruction fetch).
// pass07 over every block mode, one thread per mode.
template <int kFrontThreads>
__device__ __noinline__ void pass07_all_modes(const Tabs& tb, int T, int P, int nbm, const float* lov, const float* hiv,
                                              float min_cutoff, const float* dec, float* qfs, const float* iw,
                                              const float* wes, bool is_const, float* bm_err, int* bm_bits) {
    const int tid = threadIdx.x;
    // one thread per mode; neighbouring threads get modes of the same decimation
    for (int j = tid; j < nbm; j += kFrontThreads) {
        const int i = tb.bm_order(j);
        const DevBm bm = tb.bm(i);
        const int bc = c_free_bits[P - 1] - (int)bm.weight_bits;
        if (bm.quant > 11 || bc <= 0) { bm_err[i] = 1e38f; bm_bits[i] = 0; continue; }
        const DevDm dmi = tb.dm(bm.dm);
        const BmQuant s = bm_quant_setup(tb, bm, lov + bm.dm * 8, hiv + bm.dm * 8, min_cutoff);
        const float* dw = dec + bm.dm * 64;
        for (int w = 0; w < dmi.W; w++) { float qf; bm_quant_weight(tb, s, dw[w], &qf); qfs[w * kFrontThreads + tid] = qf; }
        float err = 0.0f;
        for (int t = 0; t < T; t++) {
            const uint64_t e4 = tb.tw4(bm.dm, t);
            float v = 0.0f;
#pragma unroll
            for (int j = 0; j < 4; j++) { const uint32_t e = (uint32_t)(e4 >> (16 * j)) & 0xFFFF; v = v + qfs[(e & 0xFF) * kFrontThreads + tid] * ((float)(e >> 8) * (1.0f / 16.0f)); }
            const float d = v - iw[t];
            err = err + (d * d) * wes[is_const ? 0 : t];
        }
        bm_err[i] = err;
        bm_bits[i] = bc;
    }
}

// P1: the instance for partitioned blocks of one partition only (the proposal pass's P = 1
// list), with P a constant the compiler folds into every loop bound and branch.
template <int NT, bool P1>
__device__ void front_body(const KernelArgs& a, const int P_arg, int lb, int blk, int slot_in_block, uint32_t entry, uint8_t* sm) {
    constexpr int kFrontThreads = NT, kFrontWarps = NT / 32;
    const int P = P1 ? 1 : P_arg;
    const Tabs tb{a.tables, &a.L};
    const int T = a.L.T, ndm = a.L.ndm, nbm = a.L.nbm;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const FrontLayout fl = front_layout(T, ndm, nbm, a.L.max_w, NT, a.bm_mask != nullptr);
    float4* px = reinterpret_cast<float4*>(sm + fl.px);
    float* iw = reinterpret_cast<float*>(sm + fl.w);
    float* wes = reinterpret_cast<float*>(sm + fl.wes);
    uint8_t* tp = sm + fl.tp;
    float* dec = reinterpret_cast<float*>(sm + fl.dec);
    float* lov = reinterpret_cast<float*>(sm + fl.lo);
    float* hiv = reinterpret_cast<float*>(sm + fl.hi);
    float* bm_err = reinterpret_cast<float*>(sm + fl.bm_err);
    int* bm_bits = reinterpret_cast<int*>(sm + fl.bm_bits);
    float* ccr_tot = reinterpret_cast<float*>(sm + fl.ccr_tot);
    uint8_t* ccr_q = sm + fl.ccr_q;
    uint8_t* ccr_fmt = sm + fl.ccr_fmt;
    float* qfs = reinterpret_cast<float*>(sm + fl.qf);
    FrontMisc& M = *reinterpret_cast<FrontMisc*>(sm + fl.misc);
    const float4 cw = chan_w();
    // Partition bytes of texels t..t+3 (t a multiple of 4 below Tp) and of texel t < T.  With one
    // partition they are known, 0 for the block's texels and 0xFF (no partition) for the
    // padding ones, and are not read from shared memory.
    auto tp4 = [&](int t) -> uint32_t {
        if constexpr (P1) {
            uint32_t q = 0;
#pragma unroll
            for (int j = 0; j < 4; j++) q |= (t + j < T ? 0u : 0xFFu) << (8 * j);
            return q;
        } else {
            return *reinterpret_cast<const uint32_t*>(tp + t);
        }
    };
    auto tp1 = [&](int t) -> int {
        if constexpr (P1) return 0;
        else return tp[t];
    };

    // Per-partition sums over the texels are taken in ascending texel order, as the
    // oracle does, by one lane per (partition, channel or term) over the whole block:
    // texels of other partitions add +0.0f.  Every such sum starts at +0.0f and adds
    // terms that are never -0.0f, so it is never -0.0f and adding +0.0f leaves it
    // unchanged: the result is the member-only sum.  The lanes read four texels per
    // step (the block padded to Tp texels whose partition byte matches none).
    const int Tp = (T + 3) & ~3;
    float* pxc = qfs;           // [4][Tp] texel channels, until pass01 ends
    float* prj = qfs + 4 * Tp;  // [Tp] projections on the partition's direction, until iw is set
    float* terms = qfs;         // [5][Tp] pass08 error terms, until they are summed
    // Side work goes to the other warps first (role 0 is warp 1's lane 0); warp 0 takes
    // pass01's chain.  With one warp, roles are its lanes.
    const int role = (tid + kFrontThreads - 32) % kFrontThreads;

    const uint8_t* prow = P > 1 ? tb.part_texels(P, entry) : nullptr;
    const BlockSrc src = block_src(a, blk);
    for (int t = tid; t < Tp; t += kFrontThreads) {
        float4 v = mk(0.0f);
        uint8_t q = 0xFF;
        if (t < T) { v = src_texel(src, a.L.bx, t); q = P > 1 ? prow[t] : 0; px[t] = v; }
        pxc[t] = v.x; pxc[Tp + t] = v.y; pxc[2 * Tp + t] = v.z; pxc[3 * Tp + t] = v.w;
        tp[t] = q;
    }
    __syncthreads();
    // ---------------- pass01: per-partition average, direction, projections
    // lane 4p + c of warp 0 takes partition p, channel c (lanes 16-31 repeat 0-15); all four
    // partitions are computed whatever P is (empty ones feed is_const and min_cutoff)
    const int gp = (lane >> 2) & 3, gc = lane & 3;
    float avg_c = 0.0f;
    if (warp == 0) {
        const float* v = pxc + gc * Tp;
        float s = 0.0f;
        int n = 0;
        for (int t = 0; t < Tp; t += 4) {
            const float4 x = *reinterpret_cast<const float4*>(v + t);
            const uint32_t q = tp4(t);
            const bool m0 = (int)(q & 0xFF) == gp, m1 = (int)((q >> 8) & 0xFF) == gp;
            const bool m2 = (int)((q >> 16) & 0xFF) == gp, m3 = (int)(q >> 24) == gp;
            s = s + (m0 ? x.x : 0.0f); s = s + (m1 ? x.y : 0.0f);
            s = s + (m2 ? x.z : 0.0f); s = s + (m3 ? x.w : 0.0f);
            n += (int)m0 + (int)m1 + (int)m2 + (int)m3;
        }
        const float cnt = (float)n;  // the oracle's count of 1.0f additions, exact
        avg_c = cnt > 0.0f ? s / cnt : 0.0f;
        if (lane < 16) reinterpret_cast<float*>(&M.avg[gp])[gc] = avg_c;
    }
    __syncthreads();
    if (warp == 0) {
        const float* v = pxc + gc * Tp;
        float dd = 0.0f;
        for (int t = 0; t < Tp; t += 4) {
            const float4 x = *reinterpret_cast<const float4*>(v + t);
            const uint32_t q = tp4(t);
            const float p0 = fmaxf(x.x - avg_c, 0.0f), p1 = fmaxf(x.y - avg_c, 0.0f);
            const float p2 = fmaxf(x.z - avg_c, 0.0f), p3 = fmaxf(x.w - avg_c, 0.0f);
            dd = dd + ((int)(q & 0xFF) == gp ? p0 * p0 : 0.0f);
            dd = dd + ((int)((q >> 8) & 0xFF) == gp ? p1 * p1 : 0.0f);
            dd = dd + ((int)((q >> 16) & 0xFF) == gp ? p2 * p2 : 0.0f);
            dd = dd + ((int)(q >> 24) == gp ? p3 * p3 : 0.0f);
        }
        const int g0 = lane & ~3;
        const float4 avg = make_float4(__shfl_sync(FULL, avg_c, g0), __shfl_sync(FULL, avg_c, g0 + 1),
                                       __shfl_sync(FULL, avg_c, g0 + 2), __shfl_sync(FULL, avg_c, g0 + 3));
        const float4 d = normalize4(make_float4(__shfl_sync(FULL, dd, g0), __shfl_sync(FULL, dd, g0 + 1),
                                                __shfl_sync(FULL, dd, g0 + 2), __shfl_sync(FULL, dd, g0 + 3)));
        if (lane < 16 && gc == 0) M.dir[gp] = d;
        __syncwarp();
        for (int t = lane; t < Tp; t += 32) {
            float pr = 0.0f;
            if (t < T) { const int p = tp1(t); pr = dot4(px[t] - M.avg[p], M.dir[p]); }
            prj[t] = pr;
        }
        __syncwarp();
        // range of the projections, taken in texel order as the oracle does
        float mn = 1e10f, mx = -1e10f;
        for (int t = 0; t < Tp; t += 4) {
            const float4 x = *reinterpret_cast<const float4*>(prj + t);
            const uint32_t q = tp4(t);
            if ((int)(q & 0xFF) == gp) { mn = fminf(mn, x.x); mx = fmaxf(mx, x.x); }
            if ((int)((q >> 8) & 0xFF) == gp) { mn = fminf(mn, x.y); mx = fmaxf(mx, x.y); }
            if ((int)((q >> 16) & 0xFF) == gp) { mn = fminf(mn, x.z); mx = fmaxf(mx, x.z); }
            if ((int)(q >> 24) == gp) { mn = fminf(mn, x.w); mx = fmaxf(mx, x.w); }
        }
        if (mn >= mx) { mn = 0.0f; mx = 1e-7f; }
        const float len = mx - mn;
        const float lsq = len * len;
        float4 e0 = avg, e1 = avg;
        if (!(d.x == 0.0f && d.y == 0.0f && d.z == 0.0f && d.w == 0.0f)) { e0 = avg + d * mn; e1 = avg + d * mx; }
        if (lane < 16 && gc == 0) { M.lsq[gp] = lsq; M.mn[gp] = mn; M.mx[gp] = mx; M.ep0[gp] = e0; M.ep1[gp] = e1; }
        // min_cutoff: the smallest (1 - ep0) / ((ep1 - ep0) + 1e-9) above 0.5 over partitions and
        // channels (10 when none); lane 4p + c computes partition p, channel c, and the minimum
        // of these values (never NaN, never 0) does not depend on the order it is taken in
        const float e0c = comp(e0, gc), e1c = comp(e1, gc);
        const float epc = (1.0f - e0c) / ((e1c - e0c) + 1e-9f);
        float me = (lane < 16 && epc > 0.5f) ? epc : 10.0f;
        for (int o = 16; o > 0; o >>= 1) me = fminf(me, __shfl_xor_sync(FULL, me, o));
        const float l1 = __shfl_sync(FULL, lsq, 4), l2 = __shfl_sync(FULL, lsq, 8), l3 = __shfl_sync(FULL, lsq, 12);
        if (lane == 0) { M.min_cutoff = me; M.is_const = (l1 == lsq && l2 == lsq && l3 == lsq) ? 1u : 0u; }
    }
    // pass08, first part (needs only the averages): role 9p + 3s + c sums channel c of the
    // deviations from the average over the texels of partition p whose channel s is above it
    for (int v = role; v < 9 * P; v += kFrontThreads) {
        const int p = v / 9, s = (v / 3) % 3, c = v % 3;
        const float as = comp(M.avg[p], s), ac = comp(M.avg[p], c);
        const float* xs = pxc + s * Tp;
        const float* xc = pxc + c * Tp;
        float sum = 0.0f;
        for (int t = 0; t < Tp; t += 4) {
            const float4 vs = *reinterpret_cast<const float4*>(xs + t), vc = *reinterpret_cast<const float4*>(xc + t);
            const uint32_t q = tp4(t);
            sum = sum + (((int)(q & 0xFF) == p && vs.x - as > 0.0f) ? vc.x - ac : 0.0f);
            sum = sum + (((int)((q >> 8) & 0xFF) == p && vs.y - as > 0.0f) ? vc.y - ac : 0.0f);
            sum = sum + (((int)((q >> 16) & 0xFF) == p && vs.z - as > 0.0f) ? vc.z - ac : 0.0f);
            sum = sum + (((int)(q >> 24) == p && vs.w - as > 0.0f) ? vc.w - ac : 0.0f);
        }
        M.sxyz[p][s][c] = sum;
    }
    if (warp == kFrontWarps - 1) {
        bool gray = true, same_a = true;
        for (int t = lane; t < T; t += 32) {
            gray = gray && px[t].x == px[t].y && px[t].x == px[t].z;
            same_a = same_a && px[t].w == px[0].w;
        }
        gray = __all_sync(FULL, gray);
        same_a = __all_sync(FULL, same_a);
        if (lane == 0) { M.gray = gray; M.calpha = same_a; }
    }
    __syncthreads();
    const bool is_const = M.is_const != 0;
    const float ew = (((cw.x + cw.y) + cw.z) + cw.w) / 4.0f;
    for (int t = tid; t < T; t += kFrontThreads) {
        const int p = tp1(t);
        const float span = fmaxf(M.mx[p] - M.mn[p], 1e-6f);
        iw[t] = clampf((prj[t] - M.mn[p]) / span, 0.0f, 1.0f);
        wes[t] = M.lsq[p] * ew;
    }
    // pass08, second part: the encoding-choice axes of partition p (role p)
    for (int p = role; p < P; p += kFrontThreads) {
        const float4 sx = make_float4(M.sxyz[p][0][0], M.sxyz[p][0][1], M.sxyz[p][0][2], 0.0f);
        const float4 sy = make_float4(M.sxyz[p][1][0], M.sxyz[p][1][1], M.sxyz[p][1][2], 0.0f);
        const float4 sz = make_float4(M.sxyz[p][2][0], M.sxyz[p][2][1], M.sxyz[p][2][2], 0.0f);
        const float pxx = dot4(sx, sx), pyy = dot4(sy, sy), pzz = dot4(sz, sz);
        float4 bv = sx; float bs = pxx;
        if (pyy > bs) { bv = sy; bs = pyy; }
        if (pzz > bs) { bv = sz; bs = pzz; }
        float4 avg = M.avg[p]; avg.w = 0.0f;
        const float4 ub = normalize4(bv);
        const float4 lbv = normalize4(make_float4(1.0f, 1.0f, 1.0f, 0.0f));
        M.axes[p][0] = ub;
        M.axes[p][1] = avg - ub * dot4(avg, ub);
        M.axes[p][2] = normalize4(avg);
        M.axes[p][3] = avg - lbv * dot4(avg, lbv);
        const float4 e0 = M.ep0[p], e1 = M.ep1[p];
        const float lim = 0.12f * 65536.0f;
        M.ece_can_offset[p] = fabsf(e1.x - e0.x) < lim && fabsf(e1.y - e0.y) < lim && fabsf(e1.z - e0.z) < lim;
        M.ece_can_bc[p] = (M.gray && M.calpha) ? 0 : 1;
        // pass09 inputs of this partition; the 4 x 21 cells are filled later, one per role
        const float ps = (float)(P == 1 ? T : tb.part_count(P, entry, p));
        const float4 e0h = vmax(e0 - mk(65535.0f), mk(0.0f)), e1h = vmax(e1 - mk(65535.0f), mk(0.0f));
        const float4 e0l = vmin(e0, mk(0.0f)), e1l = vmin(e1, mk(0.0f));
        const float4 sre = ((e0l * e0l + e1l * e1l) + e0h * e0h) + e1h * e1h;
        M.p9[p][0] = (dot3(sre, cw) * 0.5f) * ps;
        M.p9[p][1] = ((sre.w * cw.w) * 0.5f) * ps;
        M.p9[p][2] = ((cw.x + cw.y) + cw.z) * ps;
        M.p9[p][3] = cw.w * ps;
    }

    // Block-mode subset of the proposal search: only its modes and their
    // decimation modes are evaluated; the others never become candidates.
    const uint64_t* bmm = a.bm_mask ? a.bm_mask + ((size_t)lb * 4 + (P - 1)) * kMaskWords : nullptr;
    uint32_t* flags = reinterpret_cast<uint32_t*>(sm + fl.dml);  // 4 words: one bit per decimation mode
    int16_t* list = reinterpret_cast<int16_t*>(sm + fl.dml + 16);
    if (bmm && tid < 4) flags[tid] = 0;
    __syncthreads();
    int16_t* blist = reinterpret_cast<int16_t*>(sm + fl.bml);
    if (bmm) {
        for (int i = tid; i < nbm; i += kFrontThreads)
            if ((bmm[i >> 6] >> (i & 63)) & 1) { const int d = tb.bm(i).dm; atomicOr(&flags[d >> 5], 1u << (d & 31)); }
        if (warp == 0) {  // the masked block modes in ascending order: each 32-bit half word is its own ballot
            int n = 0;
            for (int i0 = 0; i0 < nbm; i0 += 32) {
                uint32_t b = (uint32_t)(bmm[i0 >> 6] >> (i0 & 63));
                if (nbm - i0 < 32) b &= (1u << (nbm - i0)) - 1u;
                if ((b >> lane) & 1u) blist[n + __popc(b & ((1u << lane) - 1u))] = (int16_t)(i0 + lane);
                n += __popc(b);
            }
            if (lane == 0) M.nlive = n;
        }
    }
    // pass08 error terms of every texel against its partition's axes
    for (int t = tid; t < Tp; t += kFrontThreads) {
        float t0 = 0.0f, t1 = 0.0f, t2 = 0.0f, t3 = 0.0f, t4 = 0.0f;
        if (t < T) {
            const int p = tp1(t);
            const float4 ub = M.axes[p][0], ua = M.axes[p][1], sb = M.axes[p][2], la = M.axes[p][3];
            const float4 lbv = normalize4(make_float4(1.0f, 1.0f, 1.0f, 0.0f));
            float4 rgb = px[t]; rgb.w = 0.0f;
            const float ad = px[t].w - 65536.0f;
            t0 = (ad * ad) * cw.w;
            const float4 du = (ua + ub * dot3(rgb, ub)) - rgb;
            t1 = dot3(du * du, cw);
            const float4 ds = sb * dot3(rgb, sb) - rgb;
            t2 = dot3(ds * ds, cw);
            const float4 dl = (la + lbv * dot3(rgb, lbv)) - rgb;
            t3 = dot3(dl * dl, cw);
            const float4 dn = lbv * dot3(rgb, lbv) - rgb;
            t4 = dot3(dn * dn, cw);
        }
        terms[t] = t0; terms[Tp + t] = t1; terms[2 * Tp + t] = t2; terms[3 * Tp + t] = t3; terms[4 * Tp + t] = t4;
    }
    __syncthreads();
    // the decimation modes to run (warp 0): the decimated ones first, whose pass02 makes them
    // the longest, so that the warps taking them in turn finish closer together; pass08
    // sums (role 5p + k)
    if (bmm && warp == 0) {
        int n = 0;
        for (int pass = 0; pass < 2; pass++)
            for (int d0 = 0; d0 < ndm; d0 += 32) {
                const int d = d0 + lane;
                const bool f = d < ndm && ((flags[d >> 5] >> (d & 31)) & 1) && ((tb.dm(d).W == T) == (pass == 1));
                const uint32_t b = __ballot_sync(FULL, f);
                if (f) list[n + __popc(b & ((1u << lane) - 1))] = (int16_t)d;
                n += __popc(b);
            }
        __syncwarp();
        if (lane == 0) flags[0] = n;  // the flags are no longer needed
    }
    for (int v = role; v < 5 * P; v += kFrontThreads) {
        const int p = v / 5, k = v % 5;
        const float* x = terms + k * Tp;
        float s = 0.0f;
        for (int t = 0; t < Tp; t += 4) {
            const float4 y = *reinterpret_cast<const float4*>(x + t);
            const uint32_t q = tp4(t);
            s = s + ((int)(q & 0xFF) == p ? y.x : 0.0f); s = s + ((int)((q >> 8) & 0xFF) == p ? y.y : 0.0f);
            s = s + ((int)((q >> 16) & 0xFF) == p ? y.z : 0.0f); s = s + ((int)(q >> 24) == p ? y.w : 0.0f);
        }
        M.acc[p][k] = s;
    }
    __syncthreads();
    const int ndm_run = bmm ? (int)flags[0] : ndm;
    const int16_t* dm_run = bmm ? list : nullptr;
    // ---------------- pass09: colour error per partition, quant level and integer count
    // (role 21p + q; runs beside passes 02-05, which do not read it)
    for (int c = role; c < P * 21; c += kFrontThreads) {
        const int p = c / 21, q = c % 21;
        if (q < 4) {
            for (int j = 0; j < 4; j++) M.cerr[p][q][j] = ERR_DEFAULT;
            M.cfmt[p][q][0] = FMT_LUMINANCE; M.cfmt[p][q][1] = FMT_RGB_SCALE; M.cfmt[p][q][2] = FMT_RGB; M.cfmt[p][q][3] = FMT_RGBA;
            continue;
        }
        const int i = q - 4;
        const float rre = M.p9[p][0], are = M.p9[p][1], brgb = M.p9[p][2], ba = M.p9[p][3];
        const bool cbc = M.ece_can_bc[p] == 1, coe = M.ece_can_offset[p] == 1;
        const float bcrgba = cbc ? 0.625f : 1.0f, oergba = coe ? 0.5f : 1.0f, bcrgb = cbc ? 0.5f : 1.0f, oergb = coe ? 0.25f : 1.0f;
        const float acc0 = M.acc[p][0], acc1 = M.acc[p][1], acc2 = M.acc[p][2], acc4 = M.acc[p][4];
        const float rgbs_e = (acc2 - acc1) * 0.7f, lum_e = (acc4 - acc1) * 3.0f, ad_e = acc0 * 3.0f;
        const float orgba = q >= 19 ? 1.0f : oergba, orgb = q >= 19 ? 1.0f : oergb;
        const float bq = tb.bqe(i);
        const float qrgb = brgb * bq, qrgba = (brgb + ba) * bq;
        M.cerr[p][q][3] = (((qrgba * bcrgba) * orgba) + rre) + are; M.cfmt[p][q][3] = FMT_RGBA;
        const float full = (((qrgb * bcrgb) * orgb) + rre) + ad_e;
        const float rgbsa = ((qrgba + rgbs_e) + rre) + are;
        if (rgbsa < full) { M.cerr[p][q][2] = rgbsa; M.cfmt[p][q][2] = FMT_RGB_SCALE_ALPHA; }
        else { M.cerr[p][q][2] = full; M.cfmt[p][q][2] = FMT_RGB; }
        const float lrgbs = ((qrgb + rre) + ad_e) + rgbs_e;
        const float la_e = ((qrgba + rre) + are) + lum_e;
        if (lrgbs < la_e) { M.cerr[p][q][1] = lrgbs; M.cfmt[p][q][1] = FMT_RGB_SCALE; }
        else { M.cerr[p][q][1] = la_e; M.cfmt[p][q][1] = FMT_LUMINANCE_ALPHA; }
        M.cerr[p][q][0] = ((qrgb + rre) + ad_e) + lum_e; M.cfmt[p][q][0] = FMT_LUMINANCE;
    }

    // ---------------- passes 02-05
    dm_passes<kFrontWarps>(tb, T, fl, sm, ndm_run, dm_run, iw, wes, is_const, dec, lov, hiv, qfs);
    __syncthreads();

    // ---------------- pass07: weight quantisation error per block mode
    const int nlist = bmm ? M.nlive : nbm;  // block modes evaluated: the list, or all of them
    if (!bmm) pass07_all_modes<kFrontThreads>(tb, T, P, nbm, lov, hiv, M.min_cutoff, dec, qfs, iw, wes, is_const, bm_err, bm_bits);
    // ---------------- pass10: best format combination per quant level and integer total
    // One item per (quant level, integer total), beside pass07 (role-indexed): the format
    // combinations with that total, in the order the one-thread loops visit them (i, j, k, l
    // ascending, each format class within one of the others), so the first minimum is the same.
    if (P > 1) {
        const int NC = P == 2 ? 7 : P == 3 ? 10 : 13;
        for (int it = role; it < 17 * NC; it += kFrontThreads) {
            const int q = 4 + it / NC, c = it - (it / NC) * NC;
            float be = ERR_DEFAULT;
            uint32_t bf = 0;
            for (int o = c_combo_off[P - 2][c]; o < c_combo_off[P - 2][c + 1]; o++) {
                const uint32_t cb = c_combo[o];
                const int i = cb & 3, j = (cb >> 2) & 3, k = (cb >> 4) & 3, l = cb >> 6;
                float e;
                if (P == 2) e = fminf(M.cerr[0][q][i] + M.cerr[1][q][j], 1e10f);
                else if (P == 3) e = fminf((M.cerr[0][q][i] + M.cerr[1][q][j]) + M.cerr[2][q][k], 1e10f);
                else e = fminf(((M.cerr[0][q][i] + M.cerr[1][q][j]) + M.cerr[2][q][k]) + M.cerr[3][q][l], 1e10f);
                if (e < be) { be = e; bf = cb; }
            }
            M.combo_err[q][c] = be;
            uint8_t* f = M.combo_fmt[q][c];
            f[0] = M.cfmt[0][q][bf & 3]; f[1] = M.cfmt[1][q][(bf >> 2) & 3];
            f[2] = P > 2 ? M.cfmt[2][q][(bf >> 4) & 3] : 0;
            f[3] = P > 3 ? M.cfmt[3][q][bf >> 6] : 0;
        }
    }
    if (bmm) {
        // The proposal search's few block modes, in groups that fit the buffer: the quantised
        // weights (one thread per mode and weight), the error terms (one per mode and
        // texel), then each mode's sum in texel order (padding texels add +0.0f to a sum of
        // non-negative terms).  Each value is the one-thread-per-mode loop's.
        const int mw = a.L.max_w;
        const int qf_floats = front_layout_qf_floats(T, mw, kFrontThreads, true);
        const int G = qf_floats / (mw + Tp);
        float* qw = qfs;           // [G][mw]
        float* et = qfs + G * mw;  // [G][Tp]
        for (int g0 = 0; g0 < nlist; g0 += G) {
            const int g = min(G, nlist - g0);
            for (int it = tid; it < g * mw; it += kFrontThreads) {
                const int k = it / mw, w = it - k * mw;
                const DevBm bm = tb.bm(blist[g0 + k]);
                const int bc = c_free_bits[P - 1] - (int)bm.weight_bits;
                if (bm.quant > 11 || bc <= 0 || w >= (int)tb.dm(bm.dm).W) continue;
                const BmQuant s = bm_quant_setup(tb, bm, lov + bm.dm * 8, hiv + bm.dm * 8, M.min_cutoff);
                float qf;
                bm_quant_weight(tb, s, dec[bm.dm * 64 + w], &qf);
                qw[k * mw + w] = qf;
            }
            __syncthreads();
            for (int it = tid; it < g * Tp; it += kFrontThreads) {
                const int k = it / Tp, t = it - k * Tp;
                const DevBm bm = tb.bm(blist[g0 + k]);
                const int bc = c_free_bits[P - 1] - (int)bm.weight_bits;
                float term = 0.0f;
                if (t < T && !(bm.quant > 11 || bc <= 0)) {
                    const uint64_t e4 = tb.tw4(bm.dm, t);
                    const float* qk = qw + k * mw;
                    float v = 0.0f;
#pragma unroll
                    for (int j = 0; j < 4; j++) { const uint32_t e = (uint32_t)(e4 >> (16 * j)) & 0xFFFF; v = v + qk[e & 0xFF] * ((float)(e >> 8) * (1.0f / 16.0f)); }
                    const float d = v - iw[t];
                    term = (d * d) * wes[is_const ? 0 : t];
                }
                et[k * Tp + t] = term;
            }
            __syncthreads();
            // (the next group's first phase writes only qw, which this one does not read)
            for (int k = tid; k < g; k += kFrontThreads) {
                const int i = blist[g0 + k];
                const DevBm bm = tb.bm(i);
                const int bc = c_free_bits[P - 1] - (int)bm.weight_bits;
                if (bm.quant > 11 || bc <= 0) { bm_err[i] = 1e38f; bm_bits[i] = 0; continue; }
                const float* x = et + k * Tp;
                float err = 0.0f;
                for (int t = 0; t < Tp; t += 4) {
                    const float4 y = *reinterpret_cast<const float4*>(x + t);
                    err = err + y.x; err = err + y.y; err = err + y.z; err = err + y.w;
                }
                bm_err[i] = err;
                bm_bits[i] = bc;
            }
        }
    }
    __syncthreads();
    // ---------------- pass11: best colour combination per block mode
    for (int k = tid; k < nlist; k += kFrontThreads) {
        const int i = bmm ? blist[k] : k;
        const float werr = bm_err[i];
        uint8_t* fm = ccr_fmt + i * 4;
        if (werr >= ERR_DEFAULT) { ccr_tot[i] = ERR_DEFAULT; ccr_q[i * 2] = ccr_q[i * 2 + 1] = 0; fm[0] = fm[1] = fm[2] = fm[3] = 0; continue; }
        const int bits = bm_bits[i];
        int best_i = 0;
        float best_e = ERR_DEFAULT;
        if (P == 1) {
            for (int ic = 1; ic <= 4; ic++) {
                const int ql = tb.qmt(ic, bits);
                if (ql < 4) continue;
                const float e = M.cerr[0][ql][ic - 1];
                if (e < best_e) { best_e = e; best_i = ic; }
            }
            const int fql = tb.qmt(best_i, bits);
            fm[0] = fql >= 4 ? M.cfmt[0][fql][best_i - 1] : FMT_LUMINANCE;
            fm[1] = fm[2] = fm[3] = 0;
            ccr_q[i * 2] = ccr_q[i * 2 + 1] = (uint8_t)fql;
        } else {
            const int hi = P == 2 ? 8 : 9, modb = P == 2 ? 2 : P == 3 ? 5 : 8;
            for (int ic = P; ic <= hi; ic++) {
                const int ql = tb.qmt(ic, bits);
                if (ql < 4) break;
                const float e = M.combo_err[ql][ic - P];
                if (e < best_e) { best_e = e; best_i = ic; }
            }
            const int fql = tb.qmt(best_i, bits), fqlm = tb.qmt(best_i, bits + modb);
            for (int k = 0; k < 4; k++) fm[k] = fql >= 4 ? M.combo_fmt[fql][best_i - P][k] : 0;
            ccr_q[i * 2] = (uint8_t)fql; ccr_q[i * 2 + 1] = (uint8_t)fqlm;
        }
        ccr_tot[i] = best_e + werr;
    }
    __syncthreads();
    // ---------------- pass12: the 8 best trials (first minimum wins ties)
    // warp 0 picks them in order: each round the (error, index)-smallest mode after the
    // previous pick -- the order in which counting, for every mode, the modes ranked
    // before it would place them
    if (warp == 0 && bmm && nlist <= 32) {
        // up to 32 listed modes, one per lane: a usable mode's pick position is the number
        // of usable modes before it in (error, index) order
        const int i = lane < nlist ? blist[lane] : 0x7FFFFFFF;
        const float e = lane < nlist ? ccr_tot[i] : ERR_DEFAULT;
        const bool ok = e < ERR_DEFAULT;
        int rank = 0;
        for (int j = 0; j < nlist; j++) {
            const float ej = __shfl_sync(FULL, e, j);
            const int ij = __shfl_sync(FULL, i, j);
            rank += (ej < ERR_DEFAULT && (ej < e || (ej == e && ij < i))) ? 1 : 0;
        }
        const int nok = __popc(__ballot_sync(FULL, ok));
        if (ok && rank < kNumCand) M.top[rank] = i;
        if (lane >= nok && lane < kNumCand) M.top[lane] = -1;
    } else if (warp == 0) {
        float pv = 0.0f;
        int pi = -1;
        for (int r = 0; r < kNumCand; r++) {
            float be = 3.4e38f;
            int bi = 0x7FFFFFFF;
            for (int k = lane; k < nlist; k += 32) {
                const int i = bmm ? blist[k] : k;
                const float e = ccr_tot[i];
                if (!(e < ERR_DEFAULT)) continue;
                if (r > 0 && !(e > pv || (e == pv && i > pi))) continue;
                if (e < be || (e == be && i < bi)) { be = e; bi = i; }
            }
            for (int o = 16; o > 0; o >>= 1) {
                const float oe = __shfl_xor_sync(0xFFFFFFFFu, be, o);
                const int oi = __shfl_xor_sync(0xFFFFFFFFu, bi, o);
                if (oe < be || (oe == be && oi < bi)) { be = oe; bi = oi; }
            }
            if (bi == 0x7FFFFFFF) {  // fewer than kNumCand usable modes
                if (lane >= r && lane < kNumCand) M.top[lane] = -1;
                break;
            }
            if (lane == 0) M.top[r] = bi;
            pv = be; pi = bi;
        }
    }
    __syncthreads();
    PBRec& rec = a.pbrec[(size_t)lb * a.slots + slot_in_block];
    if (a.work && tid == 0) {
        int nbm_run = nbm;
        if (bmm) {
            nbm_run = 0;
            for (int w = 0; w < kMaskWords; w++) {
                const int lo = w * 64;
                if (lo >= nbm) break;
                const uint64_t valid = nbm - lo >= 64 ? ~0ull : ((1ull << (nbm - lo)) - 1);
                nbm_run += __popcll(bmm[w] & valid);
            }
        }
        atomicAdd(a.work + (P - 1), 1ull);
        atomicAdd(a.work + 4, (unsigned long long)ndm_run);
        atomicAdd(a.work + 5, (unsigned long long)nbm_run);
    }
    if (tid == 0) {
        int n = 0;
        while (n < a.topn && M.top[n] >= 0) n++;
        M.ncand = n;
        rec.P = P; rec.entry = entry; rec.ncand = n;
        rec.seed = P > 1 ? tb.part_seed(P, entry) : 0;
    }
    if (tid < 4) { rec.avg[tid] = M.avg[tid]; rec.ep0[tid] = M.ep0[tid]; rec.ep1[tid] = M.ep1[tid]; }
    __syncthreads();
    // candidate initial state: the trial's quantised weights (REF-BUG-6: only
    // floor(W/4)*4 weights are packed by pass07, the rest read as 0; FIXED semantics: all W)
    const int ncand = M.ncand;
    for (int k = tid >> 3; k < ncand; k += kFrontThreads / 8) {
        const int i = M.top[k];
        const DevBm bm = tb.bm(i);
        const DevDm dmi = tb.dm(bm.dm);
        CandInit& c = rec.c[k];
        if ((tid & 7) == 0) {
            c.bm = (uint16_t)i; c.ql = ccr_q[i * 2]; c.qlm = ccr_q[i * 2 + 1];
            for (int f = 0; f < 4; f++) c.fmt[f] = ccr_fmt[i * 4 + f];
        }
        const BmQuant s = bm_quant_setup(tb, bm, lov + bm.dm * 8, hiv + bm.dm * 8, M.min_cutoff);
        const int packed_w = a.fixed ? dmi.W : (dmi.W / 4) * 4;
        for (int w = tid & 7; w < 64; w += 8) {
            int v = 0;
            if (w < packed_w) { float qf; v = bm_quant_weight(tb, s, dec[bm.dm * 64 + w], &qf); }
            c.qw[w] = (uint8_t)v;
        }
    }
}

// Resident CTAs of 128 threads the register budget is sized for (the proposal search's
// compact layout lets that many fit in shared memory for the small footprints).
constexpr int kFrontMinBlocks128 = 8;
template <int NT, bool P1>
__global__ void __launch_bounds__(NT, kFrontMinBlocks128 * 128 / NT > 32 ? 32 : kFrontMinBlocks128 * 128 / NT) k_front(const __grid_constant__ KernelArgs a) {
    extern __shared__ __align__(16) uint8_t smem[];
    // Items: every slot of every block in slot-major order (co-resident CTAs work on the
    // same partition count), or the proposal pass's work list grouped by partition count.
    const int nb = list_blocks(a);
    const int items = a.pb_list ? pb_total(a) : nb * a.slots;
    for (int li = blockIdx.x; li < items; li += gridDim.x) {
        int k, lb;
        if (a.pb_list) pb_item(a, li, lb, k);
        else { k = li / nb; lb = li % nb; }
        const int blk = chunk_block(a, lb);
        int P = 1, entry = 0;
        bool present = true;
        if (k > 0 && a.prop) {
            const PropPicks& pp = a.prop[lb];
            present = k - 1 < (int)pp.n;
            const int v = present ? pp.v[k - 1] : 0;
            P = 2 + (v >> 10); entry = v & 1023;
        } else if (k > 0) {
            P = 2 + (k - 1) / 4;
            const uint16_t* pk = a.picks[lb].v + (P - 2) * 5;
            const int i = (k - 1) % 4;
            present = i < pk[4];
            entry = present ? pk[i] : 0;
        }
        if (!present) {
            if (threadIdx.x == 0) { PBRec& rec = a.pbrec[(size_t)lb * a.slots + k]; rec.P = P; rec.ncand = 0; rec.entry = 0; rec.seed = 0; }
            continue;  // uniform across the CTA
        }
        front_body<NT, P1>(a, P, lb, blk, k, entry, smem);
        __syncthreads();  // the next item reuses shared memory
    }
}

}  // namespace

size_t search_smem_bytes(const TableLayout&) { return (size_t)kSearchWarps * kSearchWarpBytes; }
size_t front_smem_bytes(const TableLayout& L, int nt, bool list) { return (size_t)front_layout(L.T, L.ndm, L.nbm, L.max_w, nt, list).total; }

// front_bytes: the 128-thread layout, the largest of the three.
cudaError_t configure_search_kernels(size_t search_bytes, size_t front_bytes) {
    cudaError_t e = cudaFuncSetAttribute(k_partition_search, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)search_bytes);
    // the largest shared-memory carveout: occupancy of the front is bounded by shared memory
    for (auto f : {k_front<128, false>, k_front<64, false>, k_front<32, false>, k_front<128, true>, k_front<64, true>,
                   k_front<32, true>}) {
        if (e == cudaSuccess) e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)front_bytes);
        if (e == cudaSuccess) e = cudaFuncSetAttribute(f, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    }
    return e;
}

cudaError_t launch_partition_search(const KernelArgs& a, cudaStream_t s) {
    const int items = a.nblocks * 3;
    int grid = (items + kSearchWarps - 1) / kSearchWarps;
    if (a.block_list) grid = std::min(grid, kListGridSearch);
    k_partition_search<<<grid, kSearchWarps * 32, search_smem_bytes(a.L), s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_front(const KernelArgs& a, cudaStream_t s) {
    const int nt = a.front_threads == 32 || a.front_threads == 64 ? a.front_threads : 128;
    int grid = a.nblocks * a.slots;
    if (a.block_list) grid = std::min(grid, kListGridFront * (128 / nt));
    const size_t smem = front_smem_bytes(a.L, nt, a.bm_mask != nullptr);
    auto go = [&](const KernelArgs& k, bool p1) {
        if (nt == 32) { if (p1) k_front<32, true><<<grid, 32, smem, s>>>(k); else k_front<32, false><<<grid, 32, smem, s>>>(k); }
        else if (nt == 64) { if (p1) k_front<64, true><<<grid, 64, smem, s>>>(k); else k_front<64, false><<<grid, 64, smem, s>>>(k); }
        else { if (p1) k_front<128, true><<<grid, 128, smem, s>>>(k); else k_front<128, false><<<grid, 128, smem, s>>>(k); }
    };
    if (a.pb_list && a.pb_from == 0 && a.pb_to == 0) {
        // the proposal pass's work lists: P = 1 by its own instance, then P = 2..4
        KernelArgs k1 = a, k2 = a;
        k1.pb_from = 0; k1.pb_to = 1;
        k2.pb_from = 1; k2.pb_to = 4;
        go(k1, true);
        go(k2, false);
    } else {
        go(a, false);
    }
    return cudaGetLastError();
}

}  // namespace astcb200
