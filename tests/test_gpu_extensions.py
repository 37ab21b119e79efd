"""The optional encodings on the GPU (ASTCB200_FLAG_VOID_EXTENT, ASTCB200_FLAG_DUAL_PLANE):
bit for bit against the oracle's extensions (orc_set_extensions) in both semantics, through
the full search and the proposal search; every block decodes to the specification's
reconstruction from its symbolic result; dual plane raises quality."""
import contextlib
import os
import sys

import numpy as np
import pytest

import _libs
import astc_implementation_b200 as ab
from astc_implementation_b200 import proposal, synth

sys.path.insert(0, os.path.join(_libs.REPO, "oracle"))
import astc_decode_oracle as ado  # noqa: E402

pytestmark = pytest.mark.gpu


@contextlib.contextmanager
def oracle_mode(ext, fixed):
    orc = _libs.oracle()
    pe, pf = orc.orc_set_extensions(ext), orc.orc_set_semantics(1 if fixed else 0)
    try:
        yield
    finally:
        orc.orc_set_extensions(pe)
        orc.orc_set_semantics(pf)


def oracle_encode(img, bx, by, iters=6):
    h, w = img.shape[:2]
    n = ((w + bx - 1) // bx) * ((h + by - 1) // by)
    out = np.zeros((n, 16), np.uint8)
    sym = np.zeros((n, 108), np.uint32)
    assert _libs.oracle().orc_encode_iters(_libs.ptr(np.ascontiguousarray(img)), w, h, bx, by, 0, iters, _libs.ptr(out),
                                           _libs.ptr(sym)) == 0
    return out, sym


def texture(w, h, seed):
    img = synth.make_texture(w, h, seed)
    img[1:13, 2:17] = [200, 100, 50, 255]  # one colour: void-extent blocks
    return img


@pytest.mark.parametrize("fixed", [False, True])
@pytest.mark.parametrize("bx,by", [(4, 4), (6, 6), (8, 5), (12, 12)])
def test_extensions_bit_exact_against_oracle(bx, by, fixed):
    w, h = 7 * bx + 3, 5 * by + 2
    img = texture(w, h, 600 + bx * 16 + by)
    enc = ab.ASTCEncoder(device=0, fixed=fixed, void_extent=True, dual_plane=True)
    enc.secondaryInit(w, h, bx, by)
    sym = enc.encode_symbolic(img)
    out = enc.encode(img).reshape(-1, 16)
    enc.close()
    with oracle_mode(3, fixed):
        ref_out, ref_sym = oracle_encode(img, bx, by)
    assert np.array_equal(sym, ref_sym)
    assert np.array_equal(out, ref_out)
    assert (sym[:, 6] > 0).any() and (sym[:, 7] > 0).any()
    parts = ado.PartitionTables(_libs.oracle(), bx, by)
    assert np.array_equal(ab.decode(bx, by, w, h, out.reshape(-1)), ado.image_from_symbolic(sym, bx, by, w, h, parts))


def test_void_extent_only():
    img = texture(48, 40, 7)
    enc = ab.ASTCEncoder(device=0, void_extent=True)
    enc.secondaryInit(48, 40, 4, 4)
    sym = enc.encode_symbolic(img)
    out = enc.encode(img)
    enc.close()
    with oracle_mode(1, False):
        ref_out, ref_sym = oracle_encode(img, 4, 4)
    assert np.array_equal(sym, ref_sym) and np.array_equal(out.reshape(-1, 16), ref_out)
    assert (sym[:, 7] > 0).any() and not (sym[:, 6] > 0).any()


@pytest.mark.parametrize("bx,by,topn,iters,fb", [(4, 4, 8, 6, 6), (6, 6, 3, 6, 3)])
def test_extensions_after_the_proposal_search(bx, by, topn, iters, fb):
    """The extensions follow the proposal search too: proposal-search blocks equal the FIXED
    oracle restricted to the GPU's selection with the extensions, the others its full search."""
    w, h = 11 * bx + 3, 7 * by + 2
    img = texture(w, h, 190 + bx)
    enc = ab.ASTCEncoder(device=0, fixed=True, void_extent=True, dual_plane=True)
    enc.secondaryInit(w, h, bx, by)
    enc.set_proposal_net(proposal.load_weights(bx, by))
    enc.set_pruning(True, reroute_error=0.0)
    sym = enc.encode_symbolic(img)
    blocks = enc.encode(img).reshape(-1, 16)
    route, picks, masks = enc.proposal_selection(img)
    enc.close()
    n = picks.shape[0]
    r_out = np.zeros((n, 16), np.uint8)
    r_sym = np.zeros((n, 108), np.uint32)
    found = np.zeros(n, np.uint8)
    with oracle_mode(3, True):
        assert _libs.oracle().orc_encode_restricted(_libs.ptr(img), w, h, bx, by, 0, _libs.ptr(np.ascontiguousarray(picks)),
                                                    _libs.ptr(np.ascontiguousarray(masks)), topn, iters, _libs.ptr(r_out),
                                                    _libs.ptr(r_sym), _libs.ptr(found)) == 0
        f_out, f_sym = oracle_encode(img, bx, by, iters=fb)
    prop = (route == 0) & found.astype(bool)
    assert prop.sum() > 0.5 * n
    assert np.array_equal(sym[prop], r_sym[prop]) and np.array_equal(blocks[prop], r_out[prop])
    assert np.array_equal(sym[~prop], f_sym[~prop]) and np.array_equal(blocks[~prop], f_out[~prop])


@pytest.mark.parametrize("bx,by", [(4, 4), (6, 6)])
def test_dual_plane_raises_quality(bx, by):
    imgs = [synth.make_texture(256, 256, s) for s in (7, 8)]
    res = {}
    for dual in (False, True):
        enc = ab.ASTCEncoder(device=0, fixed=True, dual_plane=dual)
        enc.secondaryInit(256, 256, bx, by)
        res[dual] = np.mean([ab.psnr(ab.decode(bx, by, 256, 256, enc.encode(im)), im) for im in imgs])
        enc.close()
    assert res[True] > res[False] + 0.1, res
