"""The CPU oracle on its own: determinism, edge cases, quality sanity."""
import numpy as np
import pytest

import _libs
import astc_implementation_b200 as ab
from astc_implementation_b200 import synth


def _encode(img, bx, by, threads=0):
    h, w = img.shape[:2]
    n = ((w + bx - 1) // bx) * ((h + by - 1) // by)
    out = np.zeros(n * 16, np.uint8)
    sym = np.zeros((n, 108), np.uint32)
    assert _libs.oracle().orc_encode(_libs.ptr(np.ascontiguousarray(img)), w, h, bx, by, threads, _libs.ptr(out), _libs.ptr(sym)) == 0
    return out, sym


def test_thread_count_does_not_change_results():
    img = synth.make_texture(40, 36, 3)
    a = _encode(img, 4, 4, 1)
    b = _encode(img, 4, 4, 8)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


@pytest.mark.parametrize("w,h", [(1, 1), (3, 5), (17, 13)])
def test_small_and_ragged_images(w, h):
    img = synth.make_texture(max(w, 2), max(h, 2), 11)[:h, :w]
    for bx, by in [(4, 4), (6, 6), (12, 12)]:
        out, sym = _encode(img, bx, by)
        assert (sym[:, 2] >= 1).all()
        dec = ab.decode(bx, by, w, h, out)
        assert dec.shape == (h, w, 4)


@pytest.mark.parametrize("value", [0, 77, 255])
def test_constant_blocks(value):
    img = np.full((16, 16, 4), value, np.uint8)
    out, sym = _encode(img, 4, 4)
    dec = ab.decode(4, 4, 16, 16, out)
    assert np.abs(dec.astype(int) - value).max() <= 1


def test_grayscale_and_constant_alpha_block():
    img = synth.make_texture(16, 16, 5)
    img[:, :, 1] = img[:, :, 0]
    img[:, :, 2] = img[:, :, 0]
    img[:, :, 3] = 255
    out, sym = _encode(img, 4, 4)
    assert ab.psnr(ab.decode(4, 4, 16, 16, out), img) > 30.0


def test_partition_search_returns_reference_rank_entries():
    img = synth.make_texture(8, 8, 2)
    tex = synth.texel_blocks(img, 4, 4)[0]
    for P in (2, 3, 4):
        ent = np.zeros(4, np.uint32)
        n = _libs.oracle().orc_partition_search(4, 4, _libs.ptr(np.ascontiguousarray(tex)), P, _libs.ptr(ent))
        assert 1 <= n <= 4
        # the rank among the first 128 ordered candidates is used as the table entry
        assert all((P - 2) * 1024 <= e < (P - 2) * 1024 + 128 for e in ent[:n])


def _restricted(img, bx, by, picks, masks, topn, iters):
    h, w = img.shape[:2]
    n = picks.shape[0]
    out = np.zeros((n, 16), np.uint8)
    sym = np.zeros((n, 108), np.uint32)
    found = np.zeros(n, np.uint8)
    rc = _libs.oracle().orc_encode_restricted(_libs.ptr(np.ascontiguousarray(img)), w, h, bx, by, 0, _libs.ptr(picks),
                                              _libs.ptr(masks), topn, iters, _libs.ptr(out), _libs.ptr(sym), _libs.ptr(found))
    assert rc == 0
    return out, sym, found.astype(bool)


@pytest.mark.parametrize("bx,by", [(4, 4), (6, 6)])
def test_restricted_search_with_every_candidate_is_the_full_search(bx, by):
    """The proposal search's checker, given P = 1, every partitioning the partition search
    emits (in partition-count order), all block modes, 8 trials and 6 iterations, is the
    full search block for block."""
    img = synth.make_texture(3 * bx + 1, 2 * by + 3, 23)
    tex = synth.texel_blocks(img, bx, by)
    n = tex.shape[0]
    picks = np.zeros((n, 18), np.uint16)
    for i in range(n):
        v = []
        for P in (2, 3, 4):
            ent = np.zeros(4, np.uint32)
            k = _libs.oracle().orc_partition_search(bx, by, _libs.ptr(np.ascontiguousarray(tex[i])), P, _libs.ptr(ent))
            v += [int(e) for e in ent[:k]]
        picks[i, 0] = len(v)
        picks[i, 2:2 + len(v)] = v
    masks = np.full((n, 16), np.iinfo(np.uint64).max, np.uint64)
    full_out, full_sym = _encode(img, bx, by)
    out, sym, found = _restricted(img, bx, by, picks, masks, 8, 6)
    assert found.all()
    assert np.array_equal(sym, full_sym) and np.array_equal(out, full_out.reshape(n, 16))
    # fewer candidates never beat the full search; with none at all nothing is found
    picks_p1 = np.zeros_like(picks)
    _, sym1, found1 = _restricted(img, bx, by, picks_p1, masks, 2, 3)
    assert found1.all() and (sym1[:, 0].view(np.float32) >= full_sym[:, 0].view(np.float32)).all()
    picks_none = picks_p1.copy()
    picks_none[:, 1] = 1
    _, _, found0 = _restricted(img, bx, by, picks_none, masks, 2, 3)
    assert not found0.any()


def test_restricted_search_rejects_bad_candidates():
    img = synth.make_texture(8, 8, 1)
    picks = np.zeros((4, 18), np.uint16)
    masks = np.zeros((4, 16), np.uint64)
    out = np.zeros((4, 16), np.uint8)
    found = np.zeros(4, np.uint8)
    orc = _libs.oracle()
    args = lambda pk, topn, iters, bx=4: (_libs.ptr(img), 8, 8, bx, bx, 1, _libs.ptr(pk), _libs.ptr(masks), topn, iters,
                                          _libs.ptr(out), None, _libs.ptr(found))
    assert orc.orc_encode_restricted(*args(picks, 9, 3)) == -1       # topn above 8
    assert orc.orc_encode_restricted(*args(picks, 2, 0)) == -1       # no refinement
    bad = picks.copy()
    bad[0, 0], bad[0, 2] = 1, (3 << 10)                               # P = 5
    assert orc.orc_encode_restricted(*args(bad, 2, 3)) == -1
    bad[0, 2] = 1023                                                  # entry beyond the selected ones
    assert orc.orc_encode_restricted(*args(bad, 2, 3)) == -1
    assert orc.orc_encode_restricted(*args(picks, 2, 3, bx=12)) == -1  # more than 256 block modes


def test_full_search_iteration_count():
    """orc_encode_iters with the reference's 6 iterations is orc_encode; with fewer, every block's
    error is at least the 6-iteration one (the first iterations are the same, and each candidate
    keeps its best-so-far)."""
    img = synth.make_texture(21, 14, 41)
    h, w = img.shape[:2]
    full_out, full_sym = _encode(img, 4, 4)
    n = full_sym.shape[0]
    for iters in (6, 3, 1):
        out = np.zeros((n, 16), np.uint8)
        sym = np.zeros((n, 108), np.uint32)
        assert _libs.oracle().orc_encode_iters(_libs.ptr(img), w, h, 4, 4, 0, iters, _libs.ptr(out), _libs.ptr(sym)) == 0
        if iters == 6:
            assert np.array_equal(sym, full_sym) and np.array_equal(out, full_out.reshape(n, 16))
        else:
            assert (sym[:, 0].view(np.float32) >= full_sym[:, 0].view(np.float32)).all()


def test_front_candidates_are_well_formed():
    """orc_front_candidates (passes 01-12 of one partitioned block, the GPU stage test's
    checker): 1..8 candidates with distinct valid trial block modes, colour quant levels of
    at least 4, and partition 0's average finite (its endpoints are NaN for a block with no
    direction, as the shader's normalisation of a zero vector gives)."""
    orc = _libs.oracle()
    img = synth.make_texture(24, 24, 11)
    for bx, by in [(4, 4), (6, 6)]:
        c = np.zeros(13, np.uint32)
        orc.orc_counts(bx, by, _libs.ptr(c))
        nbm = int(c[1])
        tex = synth.texel_blocks(img, bx, by)
        for b in range(3):
            for P, entry in [(1, 0), (2, 5), (3, 17)]:
                ep = np.zeros(48, np.float32)
                cands = np.zeros((8, 71), np.uint32)
                n = orc.orc_front_candidates(bx, by, _libs.ptr(np.ascontiguousarray(tex[b])), P, entry, _libs.ptr(ep), _libs.ptr(cands))
                assert 1 <= n <= 8
                bms = [int(v) for v in cands[:n, 0]]
                assert len(set(bms)) == n and all(m < nbm for m in bms)
                assert all(int(v) >= 4 for v in cands[:n, 1])
                assert np.all(np.isfinite(ep.reshape(4, 3, 4)[0, 0]))
