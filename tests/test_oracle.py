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
