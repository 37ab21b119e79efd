"""The oracle's optional encodings beyond the reference's (void-extent and single-partition
dual-plane blocks, orc_set_extensions) on the CPU: every block decodes (library decoder) to
the specification's reconstruction from its symbolic result, the choices are the ones the
exact-error rule makes, and dual plane raises quality on textures whose alpha does not follow
their colour."""
import contextlib
import os
import sys

import numpy as np
import pytest

import _libs
import astc_implementation_b200 as ab
from astc_implementation_b200 import synth

sys.path.insert(0, os.path.join(_libs.REPO, "oracle"))
import astc_decode_oracle as ado  # noqa: E402


@contextlib.contextmanager
def oracle_mode(ext, fixed=False):
    orc = _libs.oracle()
    pe, pf = orc.orc_set_extensions(ext), orc.orc_set_semantics(1 if fixed else 0)
    try:
        yield
    finally:
        orc.orc_set_extensions(pe)
        orc.orc_set_semantics(pf)


def encode(img, bx, by):
    h, w = img.shape[:2]
    n = ((w + bx - 1) // bx) * ((h + by - 1) // by)
    out = np.zeros(n * 16, np.uint8)
    sym = np.zeros((n, 108), np.uint32)
    assert _libs.oracle().orc_encode(_libs.ptr(np.ascontiguousarray(img)), w, h, bx, by, 0, _libs.ptr(out), _libs.ptr(sym)) == 0
    return out, sym


def texture(w, h, seed):
    img = synth.make_texture(w, h, seed)
    img[2:18, 3:21] = [12, 34, 56, 200]  # one colour: void-extent blocks
    return img


def test_extensions_default_off():
    orc = _libs.oracle()
    assert orc.orc_set_extensions(0) == 0
    img = texture(40, 30, 2)
    a = encode(img, 4, 4)
    with oracle_mode(0):
        b = encode(img, 4, 4)
    assert np.array_equal(a[0], b[0]) and (a[1][:, 6:8] == 0).all()


@pytest.mark.parametrize("fixed", [False, True])
@pytest.mark.parametrize("bx,by", [(4, 4), (6, 6), (8, 5), (12, 12)])
def test_extended_blocks_decode_to_their_reconstruction(bx, by, fixed):
    w, h = 5 * bx + 3, 4 * by + 2
    img = texture(w, h, 400 + bx)
    with oracle_mode(3, fixed):
        out, sym = encode(img, bx, by)
    parts = ado.PartitionTables(_libs.oracle(), bx, by)
    assert np.array_equal(ab.decode(bx, by, w, h, out), ado.image_from_symbolic(sym, bx, by, w, h, parts))
    assert (sym[:, 6] > 0).any()  # dual-plane blocks were chosen
    # every void-extent block is a block of one colour, and every such block is one
    nbx = (w + bx - 1) // bx
    tex = synth.texel_blocks(img, bx, by)
    const = np.array([np.all(t == t[0]) for t in tex])
    assert np.array_equal(sym[:, 7] == 1, const)


def test_void_extent_block_bytes():
    img = np.zeros((8, 8, 4), np.uint8)
    img[:] = [1, 128, 255, 77]
    with oracle_mode(1):
        out, sym = encode(img, 4, 4)
    blk = out[:16]
    assert list(blk[:8]) == [0xFC, 0xFD, 0xFF, 0xFF, 0xFF, 0xFF, 0xFF, 0xFF]
    assert list(blk[8:]) == [1, 1, 128, 128, 255, 255, 77, 77]
    assert np.array_equal(ab.decode(4, 4, 8, 8, out), img)


@pytest.mark.parametrize("bx,by", [(4, 4), (6, 6)])
def test_dual_plane_raises_quality(bx, by):
    """The generator's right half has noise alpha unrelated to the colour: dual plane with
    alpha on the second plane fits it, and an extended block is only chosen when its decoded
    error is lower, so no block gets worse."""
    img = synth.make_texture(96, 64, 9)
    with oracle_mode(0, True):
        base, bsym = encode(img, bx, by)
    with oracle_mode(2, True):
        ext, esym = encode(img, bx, by)
    p0 = ab.psnr(ab.decode(bx, by, 96, 64, base), img)
    p1 = ab.psnr(ab.decode(bx, by, 96, 64, ext), img)
    assert p1 > p0 + 0.2, (p0, p1)
    dual = esym[:, 6] > 0
    assert dual.any() and np.array_equal(esym[~dual], bsym[~dual])
    assert (esym[dual, 6] == 4).sum() > 0  # alpha on the second plane
