// ASTC LDR block decoder (host), written from the ASTC specification.
// The reference has no decoder; this one measures quality (PSNR) and checks
// that every block the encoder emits decodes as the encoder intended.  The block
// decoding itself (decode_block.cuh) is shared with the device decoder.
#include <cstdint>
#include <cstring>

#include "astcb200.h"
#include "decode_block.cuh"
#include "tables.h"

using namespace astcb200;

extern "C" int astcb200_decode(uint32_t bx, uint32_t by, uint32_t dx, uint32_t dy, const uint8_t* blocks, size_t len, uint8_t* out) {
    if (!blocks || !out || !astcb200::valid_footprint((int)bx, (int)by) || dx == 0 || dy == 0) return ASTCB200_BAD_ARG;
    const uint32_t nbx = (dx + bx - 1) / bx, nby = (dy + by - 1) / by;
    if (len < (size_t)nbx * nby * 16) return ASTCB200_BAD_ARG;
    dec::Block k;
    for (uint32_t j = 0; j < nby; j++)
        for (uint32_t i = 0; i < nbx; i++) {
            dec::parse_block(blocks + ((size_t)j * nbx + i) * 16, (int)bx, (int)by, k);
            for (uint32_t y = 0; y < by; y++)
                for (uint32_t x = 0; x < bx; x++) {
                    const uint32_t px = i * bx + x, py = j * by + y;
                    if (px >= dx || py >= dy) continue;
                    uint16_t t[4];
                    dec::texel16(k, (int)bx, (int)by, (int)x, (int)y, t);
                    for (int c = 0; c < 4; c++) out[((size_t)py * dx + px) * 4 + c] = dec::to_unorm8(t[c]);
                }
        }
    return ASTCB200_OK;
}
