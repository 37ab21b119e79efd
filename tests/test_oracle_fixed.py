"""The oracle's FIXED semantics (the reference's deterministic shader bugs repaired) on the CPU:
the pass005 order against a numpy restatement of both sorts, pass007's entries, the kept
tail weights, and quality against the REF semantics."""
import contextlib

import numpy as np
import pytest

import _libs
import astc_implementation_b200 as ab
from astc_implementation_b200 import synth


@contextlib.contextmanager
def semantics(fixed):
    prev = _libs.oracle().orc_set_semantics(1 if fixed else 0)
    try:
        yield
    finally:
        _libs.oracle().orc_set_semantics(prev)


def _encode(img, bx, by, threads=0):
    h, w = img.shape[:2]
    n = ((w + bx - 1) // bx) * ((h + by - 1) // by)
    out = np.zeros((n, 16), np.uint8)
    sym = np.zeros((n, 108), np.uint32)
    assert _libs.oracle().orc_encode(_libs.ptr(np.ascontiguousarray(img)), w, h, bx, by, threads, _libs.ptr(out),
                                     _libs.ptr(sym)) == 0
    return out, sym


def _order(tex, bx, by, P):
    mism = np.zeros(1024, np.uint32)
    order = np.zeros(128, np.uint32)
    sel = _libs.oracle().orc_partition_order(bx, by, _libs.ptr(np.ascontiguousarray(tex)), P, _libs.ptr(mism), _libs.ptr(order))
    assert sel > 0
    return sel, mism, order


def _partial_bitonic(score):
    """shaders/pass005_partition_ordering.wgsl:66-88 with 256 invocations: only pairs whose
    lower index is below 256 are compared."""
    s = [int(v) for v in score]
    idx = list(range(1024))
    k = 2
    while k <= 1024:
        j = k // 2
        while j > 0:
            for l in range(256):
                p = l ^ j
                if p > l:
                    asc = (l & k) == 0
                    sw = s[l] > s[p] or (s[l] == s[p] and idx[l] > idx[p])
                    if sw == asc:
                        s[l], s[p] = s[p], s[l]
                        idx[l], idx[p] = idx[p], idx[l]
            j //= 2
        k *= 2
    return np.array(idx[:128], np.uint32)


def test_default_semantics_is_ref():
    orc = _libs.oracle()
    assert orc.orc_set_semantics(0) == 0
    assert orc.orc_set_semantics(1) == 0
    assert orc.orc_set_semantics(0) == 1


@pytest.mark.parametrize("bx,by", [(4, 4), (6, 6), (8, 5)])
def test_pass005_order_ref_partial_fixed_full(bx, by):
    img = synth.make_texture(4 * bx, 2 * by, 71 + bx)
    tex = synth.texel_blocks(img, bx, by)
    for b in range(0, tex.shape[0], 3):
        for P in (2, 3, 4):
            with semantics(False):
                sel, mism, ref_order = _order(tex[b], bx, by, P)
            with semantics(True):
                sel2, mism2, fix_order = _order(tex[b], bx, by, P)
            assert sel == sel2 and np.array_equal(mism, mism2)  # pass004 is the same in both
            assert (mism[:sel] <= 128).all() and (mism[sel:] == 0xFFFFFFFF).all()
            assert np.array_equal(ref_order, _partial_bitonic(mism))
            full = np.lexsort((np.arange(1024), mism))[:128]  # ascending score, then index
            assert np.array_equal(fix_order, full)


def test_pass007_entries_fixed_come_from_the_order():
    """REF emits ranks 0..127 as table entries (REF-BUG-4); FIXED emits entries of the order."""
    img = synth.make_texture(24, 16, 5)
    tex = synth.texel_blocks(img, 4, 4)
    saw_difference = False
    for b in range(tex.shape[0]):
        for P in (2, 3, 4):
            with semantics(True):
                _, _, order = _order(tex[b], 4, 4, P)
                ent = np.zeros(4, np.uint32)
                n = _libs.oracle().orc_partition_search(4, 4, _libs.ptr(np.ascontiguousarray(tex[b])), P, _libs.ptr(ent))
            assert 1 <= n <= 4 and len(set(ent[:n].tolist())) == n
            local = ent[:n] - (P - 2) * 1024
            assert np.isin(local, order).all()
            with semantics(False):
                ent_ref = np.zeros(4, np.uint32)
                n_ref = _libs.oracle().orc_partition_search(4, 4, _libs.ptr(np.ascontiguousarray(tex[b])), P, _libs.ptr(ent_ref))
            ranks = ent_ref[:n_ref] - (P - 2) * 1024
            assert (ranks < 128).all()
            saw_difference |= not np.array_equal(np.sort(local), np.sort(ranks))
    assert saw_difference


def test_fixed_keeps_tail_weights():
    """Block modes with W % 4 != 0 weights: REF's candidates start with the tail weights at 0
    (REF-BUG-6); in FIXED some chosen blocks of such modes have non-zero tail weights."""
    img = synth.make_texture(60, 60, 12)
    with semantics(True):
        _, sym = _encode(img, 6, 6)
    tails = 0
    for s in sym:  # [44 + i]: weight i on the 0..64 scale
        nz = np.nonzero(s[44:108])[0]
        if len(nz) and (nz.max() + 1) % 4 != 0:
            tails += 1
    assert tails > 0


def test_fixed_is_deterministic_and_thread_invariant():
    img = synth.make_texture(40, 36, 3)
    with semantics(True):
        a = _encode(img, 4, 4, 1)
        b = _encode(img, 4, 4, 8)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


@pytest.mark.parametrize("bx,by", [(4, 4), (6, 6)])
def test_fixed_improves_quality(bx, by):
    for seed in (1, 2):
        img = synth.make_texture(96, 96, seed)
        with semantics(False):
            ref, _ = _encode(img, bx, by)
        with semantics(True):
            fix, _ = _encode(img, bx, by)
        p_ref = ab.psnr(ab.decode(bx, by, 96, 96, ref.reshape(-1)), img)
        p_fix = ab.psnr(ab.decode(bx, by, 96, 96, fix.reshape(-1)), img)
        assert p_fix > p_ref + 1.0, (seed, p_ref, p_fix)


@pytest.mark.parametrize("w,h", [(1, 1), (3, 5), (17, 13)])
def test_fixed_small_and_ragged_images(w, h):
    img = synth.make_texture(max(w, 2), max(h, 2), 11)[:h, :w].copy()
    with semantics(True):
        for bx, by in [(4, 4), (6, 6), (12, 12)]:
            out, sym = _encode(img, bx, by)
            assert (sym[:, 2] >= 1).all()
            assert ab.decode(bx, by, w, h, out.reshape(-1)).shape == (h, w, 4)
