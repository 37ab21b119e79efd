"""FIXED semantics on the GPU (ASTCB200_FLAG_FIXED_SEMANTICS): the CUDA encoder against the
oracle's FIXED mode, bit for bit, at every footprint and on the edge cases the REF tests
cover; the proposal search with FIXED semantics against the restricted FIXED oracle."""
import contextlib

import numpy as np
import pytest

import _libs
import astc_implementation_b200 as ab
from astc_implementation_b200 import proposal, synth

pytestmark = pytest.mark.gpu


@contextlib.contextmanager
def fixed_oracle():
    prev = _libs.oracle().orc_set_semantics(1)
    try:
        yield
    finally:
        _libs.oracle().orc_set_semantics(prev)


def oracle_encode(img, bx, by, iters=6):
    h, w = img.shape[:2]
    n = ((w + bx - 1) // bx) * ((h + by - 1) // by)
    out = np.zeros((n, 16), np.uint8)
    sym = np.zeros((n, 108), np.uint32)
    with fixed_oracle():
        assert _libs.oracle().orc_encode_iters(_libs.ptr(np.ascontiguousarray(img)), w, h, bx, by, 0, iters,
                                               _libs.ptr(out), _libs.ptr(sym)) == 0
    return out, sym


@pytest.fixture(scope="module")
def enc():
    e = ab.ASTCEncoder(device=0, fixed=True)
    e.init()
    yield e
    e.close()


def gpu_encode(enc, img, bx, by):
    h, w = img.shape[:2]
    enc.secondaryInit(w, h, bx, by)
    sym = enc.encode_symbolic(img)
    out = enc.encode(img).reshape(-1, 16)
    return out, sym


def test_config1_256_seed0_4x4_bit_exact(enc):
    img = synth.make_texture(256, 256, 0)
    out, sym = gpu_encode(enc, img, 4, 4)
    ref_out, ref_sym = oracle_encode(img, 4, 4)
    assert np.array_equal(sym, ref_sym)
    assert np.array_equal(out, ref_out)
    ref = ab.ASTCEncoder(device=0)  # REF semantics on the same image
    ref.secondaryInit(256, 256, 4, 4)
    ref_blocks = ref.encode(img)
    ref.close()
    p_fixed = ab.psnr(ab.decode(4, 4, 256, 256, out.reshape(-1)), img)
    p_ref = ab.psnr(ab.decode(4, 4, 256, 256, ref_blocks), img)
    assert p_fixed > p_ref + 1.0


@pytest.mark.parametrize("bx,by", _libs.FOOTPRINTS)
def test_every_footprint_bit_exact(enc, bx, by):
    w, h = 5 * bx + 3, 3 * by + 1  # ragged edges
    img = synth.make_texture(w, h, 300 + bx * 16 + by)
    out, sym = gpu_encode(enc, img, bx, by)
    ref_out, ref_sym = oracle_encode(img, bx, by)
    assert np.array_equal(sym, ref_sym)
    assert np.array_equal(out, ref_out)


def test_6x6_medium_bit_exact(enc):
    img = synth.make_texture(192, 132, 9)
    out, sym = gpu_encode(enc, img, 6, 6)
    ref_out, ref_sym = oracle_encode(img, 6, 6)
    assert np.array_equal(sym, ref_sym) and np.array_equal(out, ref_out)


@pytest.mark.parametrize("w,h", [(1, 1), (3, 5), (17, 13)])
def test_tiny_images(enc, w, h):
    img = synth.make_texture(24, 24, 4)[:h, :w].copy()
    for bx, by in [(4, 4), (6, 6), (12, 12)]:
        out, sym = gpu_encode(enc, img, bx, by)
        ref_out, ref_sym = oracle_encode(img, bx, by)
        assert np.array_equal(sym, ref_sym) and np.array_equal(out, ref_out)


@pytest.mark.parametrize("kind", ["black", "white", "gray", "noise"])
def test_degenerate_and_noise_blocks(enc, kind):
    rng = np.random.default_rng(3)
    img = np.zeros((24, 20, 4), np.uint8)
    if kind == "white":
        img[:] = 255
    elif kind == "gray":
        v = rng.integers(0, 256, (24, 20), dtype=np.uint8)
        img[..., 0] = img[..., 1] = img[..., 2] = v
        img[..., 3] = 255
    elif kind == "noise":
        img = rng.integers(0, 256, (24, 20, 4), dtype=np.uint8)
    for bx, by in [(4, 4), (6, 6), (8, 5)]:
        out, sym = gpu_encode(enc, img, bx, by)
        ref_out, ref_sym = oracle_encode(img, bx, by)
        assert np.array_equal(sym, ref_sym) and np.array_equal(out, ref_out)


def test_batch_fixed_equals_single_images():
    tex = [(synth.make_texture(37, 29, 3), 4, 4), (synth.make_texture(50, 44, 4), 6, 6), (synth.make_texture(20, 21, 5), 8, 8)]
    enc = ab.ASTCEncoder(device=0, fixed=True)
    outs = enc.encode_batch(tex)
    for (img, bx, by), o in zip(tex, outs):
        ref_out, _ = oracle_encode(img, bx, by)
        assert np.array_equal(o.reshape(-1, 16), ref_out)
    enc.close()


@pytest.mark.parametrize("bx,by,topn,iters,fb", [(4, 4, 8, 6, 3), (6, 6, 3, 6, 3)])
def test_proposal_search_fixed_bit_exact_against_restricted_oracle(bx, by, topn, iters, fb):
    """The proposal search with FIXED semantics and the footprint's tuned settings: every
    proposal-search block equals the FIXED oracle restricted to the GPU's selection; every
    other block equals the FIXED full search with the fallback's iteration count.  The image
    is large enough that refinement CTAs hand their last candidates to the tail pass."""
    net = proposal.load_weights(bx, by)
    w, h = 40 * bx + 3, 24 * by + 2
    img = synth.make_texture(w, h, 190 + bx)
    enc = ab.ASTCEncoder(device=0, fixed=True, stage_timing=True)
    enc.secondaryInit(w, h, bx, by)
    enc.set_proposal_net(net)
    enc.set_pruning(True, reroute_error=0.0)
    sym = enc.encode_symbolic(img)
    blocks = enc.encode(img).reshape(-1, 16)
    tail = int(enc.work_counters()[13])
    route, picks, masks = enc.proposal_selection(img)
    enc.close()
    n = picks.shape[0]
    r_out = np.zeros((n, 16), np.uint8)
    r_sym = np.zeros((n, 108), np.uint32)
    found = np.zeros(n, np.uint8)
    with fixed_oracle():
        assert _libs.oracle().orc_encode_restricted(_libs.ptr(img), w, h, bx, by, 0, _libs.ptr(np.ascontiguousarray(picks)),
                                                    _libs.ptr(np.ascontiguousarray(masks)), topn, iters, _libs.ptr(r_out),
                                                    _libs.ptr(r_sym), _libs.ptr(found)) == 0
    f_out, f_sym = oracle_encode(img, bx, by, iters=fb)
    prop = (route == 0) & found.astype(bool)
    assert prop.sum() > 0.5 * n
    assert np.array_equal(sym[prop], r_sym[prop]) and np.array_equal(blocks[prop], r_out[prop])
    assert np.array_equal(sym[~prop], f_sym[~prop]) and np.array_equal(blocks[~prop], f_out[~prop])
    assert tail > 0  # candidates finished by k_refine_tail are among those compared
