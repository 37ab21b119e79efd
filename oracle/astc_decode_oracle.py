"""Texels of an encoded block reconstructed from its SymbolicBlock -- TEST INFRASTRUCTURE.

An independent check of the library's ASTC decoder (astc_implementation_b200/csrc/
decode_block.cuh, compiled for the host and the GPU): instead of parsing the 128 physical
bits, it starts from the encoder's symbolic result (code/astc.h:639-655, 108 u32 words:
[1] block mode, [2] partition count, [3] partition seed, [8..11] endpoint formats,
[12 + 8p ..] partition p's endpoint values on the 0..255 scale, [44 ..] weights on the
0..64 scale; for the library's optional encodings [6] = 1 + the plane-2 component of a
dual-plane block, whose plane-2 weights are at [76 ..], and [7] = 1 for a void-extent block,
whose colour is [12..15]) and applies the ASTC specification's decoding steps to those values:

  * block-mode fields (weight grid size and weight range) from the 11 mode bits
    (Khronos Data Format Specification 1.3, ASTC section "Block Mode");
  * the weight grid infilled to texels with the specification's fixed-point bilinear
    weights (section "Weight Infill");
  * LDR colour endpoint modes 0, 1, 4, 5, 6, 8, 9, 10, 12, 13 with bit transfer and blue
    contraction (section "LDR Endpoint Decoding");
  * 16-bit interpolation of the endpoints expanded as e * 257, then the library's 8-bit
    output rule (round to nearest of the 16-bit value / 257).

Partition assignments come from the partition tables of the CPU oracle (oracle/liboracle,
pinned to the reference's own init_partition_tables), not from the decoder's hash.  Only
tests import this module.
"""
import numpy as np


def block_mode_grid(bm):
    """(grid_x, grid_y, weight quant index, dual plane) of an 11-bit 2D block mode; None if
    reserved or void-extent."""
    if bm & 3:
        r = ((bm >> 4) & 1) | ((bm & 3) << 1)
        a = (bm >> 5) & 3
        sel = (bm >> 2) & 3
        if sel == 0:
            gx, gy = ((bm >> 7) & 3) + 4, a + 2
        elif sel == 1:
            gx, gy = ((bm >> 7) & 3) + 8, a + 2
        elif sel == 2:
            gx, gy = a + 2, ((bm >> 7) & 3) + 8
        elif (bm >> 8) & 1:
            gx, gy = ((bm >> 7) & 1) + 2, a + 2
        else:
            gx, gy = a + 2, ((bm >> 7) & 1) + 6
        h, d = (bm >> 9) & 1, (bm >> 10) & 1
    else:
        if (bm & 0xF) == 0:
            return None
        r = ((bm >> 4) & 1) | (((bm >> 2) & 3) << 1)
        a = (bm >> 5) & 3
        h, d = (bm >> 9) & 1, (bm >> 10) & 1
        sel = (bm >> 7) & 3
        if sel == 0:
            gx, gy = 12, a + 2
        elif sel == 1:
            gx, gy = a + 2, 12
        elif sel == 2:
            gx, gy = a + 6, ((bm >> 9) & 3) + 6
            h = d = 0
        else:
            if a == 0:
                gx, gy = 6, 10
            elif a == 1:
                gx, gy = 10, 6
            else:
                return None
    if r < 2:
        return None
    return gx, gy, (r - 2) + 6 * h, d


def infill_weights(bx, by, gx, gy, grid):
    """Per-texel weights (0..64) from a gx x gy grid of 0..64 weights (row-major)."""
    ds = (1024 + bx // 2) // (bx - 1)
    dt = (1024 + by // 2) // (by - 1)
    out = np.zeros(bx * by, np.int64)

    def g(i):
        return int(grid[i]) if i < gx * gy else 0

    for t in range(by):
        for s in range(bx):
            gs = (ds * s * (gx - 1) + 32) >> 6
            gt = (dt * t * (gy - 1) + 32) >> 6
            js, fs, jt, ft = gs >> 4, gs & 0xF, gt >> 4, gt & 0xF
            w11 = (fs * ft + 8) >> 4
            w10, w01 = ft - w11, fs - w11
            w00 = 16 - fs - ft + w11
            v0 = js + jt * gx
            p = g(v0) * w00 + g(v0 + 1) * w01 + g(v0 + gx) * w10 + g(v0 + gx + 1) * w11
            out[t * bx + s] = (p + 8) >> 4
    return out


def _bit_transfer_signed(a, b):
    b = (b >> 1) | (a & 0x80)
    a = (a >> 1) & 0x3F
    if a & 0x20:
        a -= 0x40
    return a, b


def _blue_contract(c):
    r, g, b, a = c
    return [(r + b) >> 1, (g + b) >> 1, b, a]


def _clamp(c):
    return [min(255, max(0, int(x))) for x in c]


def endpoints(cem, v):
    """LDR endpoint pair (e0, e1), each [r, g, b, a] in 0..255, of mode `cem` from its
    unquantised values v (0..255)."""
    v = [int(x) for x in v]
    if cem == 0:
        return [v[0]] * 3 + [255], [v[1]] * 3 + [255]
    if cem == 1:
        l0 = (v[0] >> 2) | (v[1] & 0xC0)
        l1 = min(l0 + (v[1] & 0x3F), 255)
        return [l0] * 3 + [255], [l1] * 3 + [255]
    if cem == 4:
        return [v[0]] * 3 + [v[2]], [v[1]] * 3 + [v[3]]
    if cem == 5:
        b0, a0 = _bit_transfer_signed(v[1], v[0])
        b2, a2 = _bit_transfer_signed(v[3], v[2])
        return _clamp([a0] * 3 + [a2]), _clamp([a0 + b0] * 3 + [a2 + b2])
    if cem in (6, 10):
        alpha0, alpha1 = (v[4], v[5]) if cem == 10 else (255, 255)
        return [(v[0] * v[3]) >> 8, (v[1] * v[3]) >> 8, (v[2] * v[3]) >> 8, alpha0], [v[0], v[1], v[2], alpha1]
    if cem in (8, 12):
        alpha0, alpha1 = (v[6], v[7]) if cem == 12 else (255, 255)
        c0 = [v[0], v[2], v[4], alpha0]
        c1 = [v[1], v[3], v[5], alpha1]
        if v[1] + v[3] + v[5] >= v[0] + v[2] + v[4]:
            return c0, c1
        return _blue_contract(c1), _blue_contract(c0)
    if cem in (9, 13):
        b0, a0 = _bit_transfer_signed(v[1], v[0])
        b1, a1 = _bit_transfer_signed(v[3], v[2])
        b2, a2 = _bit_transfer_signed(v[5], v[4])
        if cem == 13:
            b3, a3 = _bit_transfer_signed(v[7], v[6])
        else:
            b3, a3 = 0, 255
        c0 = [a0, a1, a2, a3]
        c1 = [a0 + b0, a1 + b1, a2 + b2, a3 + b3]
        if b0 + b1 + b2 >= 0:
            return _clamp(c0), _clamp(c1)
        return _clamp(_blue_contract(c1)), _clamp(_blue_contract(c0))
    raise ValueError("not an LDR endpoint mode the encoder emits: %d" % cem)


class PartitionTables:
    """Texel -> partition maps by (partition count, seed), from the CPU oracle's tables."""

    def __init__(self, orc, bx, by):
        import ctypes
        p = lambda a: a.ctypes.data_as(ctypes.c_void_p)
        self.pinfo = np.zeros((3073, 150), np.uint32)
        cov = [np.zeros((1024, k), np.uint64) for k in (2, 3, 4)]
        km = np.zeros(64, np.uint32)
        self.packed = np.zeros((3, 1024), np.uint16)
        assert orc.orc_partitions(bx, by, p(self.pinfo), p(cov[0]), p(cov[1]), p(cov[2]), p(km), p(self.packed)) == 0
        self.T = bx * by

    def of_texel(self, pc, seed):
        row = self.pinfo[(pc - 2) * 1024 + int(self.packed[pc - 2, seed])]
        assert int(row[1]) == seed  # the encoder names partitionings by their table entry's seed
        return row[6:6 + self.T].astype(np.int64)


def block_texels(sym, bx, by, parts):
    """(bx*by, 4) uint8 texels of one block from its SymbolicBlock words."""
    if int(sym[7]):  # void extent: the colour as 16-bit UNORM (x 257), back to 8 bits
        return np.tile(np.array([((int(v) * 257) * 255 + 32767) // 65535 for v in sym[12:16]], np.uint8), (bx * by, 1))
    g = block_mode_grid(int(sym[1]) & 2047)
    dual = int(sym[6]) > 0
    assert g is not None and g[3] == (1 if dual else 0), "plane count of the block mode"
    gx, gy = g[0], g[1]
    w = infill_weights(bx, by, gx, gy, sym[44:44 + gx * gy])
    w2 = infill_weights(bx, by, gx, gy, sym[76:76 + gx * gy]) if dual else w
    ccs = int(sym[6]) - 1 if dual else -1
    pc = int(sym[2])
    tp = parts.of_texel(pc, int(sym[3])) if pc > 1 else np.zeros(bx * by, np.int64)
    out = np.zeros((bx * by, 4), np.uint8)
    eps = []
    for p in range(pc):
        cem = int(sym[8 + p])
        n = 2 * (cem >> 2) + 2
        eps.append(endpoints(cem, sym[12 + 8 * p:12 + 8 * p + n]))
    for t in range(bx * by):
        e0, e1 = eps[tp[t]]
        for c in range(4):
            c0, c1 = e0[c] * 257, e1[c] * 257
            wt = int(w2[t]) if c == ccs else int(w[t])
            v16 = (c0 * (64 - wt) + c1 * wt + 32) >> 6
            out[t, c] = (v16 + 128) // 257
    return out


def image_from_symbolic(sym, bx, by, width, height, parts):
    """(height, width, 4) uint8 image from the SymbolicBlocks of its blocks (raster order)."""
    nbx = (width + bx - 1) // bx
    img = np.zeros((height, width, 4), np.uint8)
    for i, s in enumerate(sym):
        x0, y0 = (i % nbx) * bx, (i // nbx) * by
        tex = block_texels(s, bx, by, parts).reshape(by, bx, 4)
        h, w = min(by, height - y0), min(bx, width - x0)
        img[y0:y0 + h, x0:x0 + w] = tex[:h, :w]
    return img
