"""The library's ASTC decoder against an independent reconstruction from the encoder's
symbolic blocks (oracle/astc_decode_oracle.py, written from the ASTC specification): the
host build of the decoder on the CPU oracle's output, at every footprint, in both search
semantics.  (tests/test_gpu_decoder.py checks the GPU build against the same reconstruction.)"""
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
def semantics(fixed):
    prev = _libs.oracle().orc_set_semantics(1 if fixed else 0)
    try:
        yield
    finally:
        _libs.oracle().orc_set_semantics(prev)


def oracle_encode(img, bx, by):
    h, w = img.shape[:2]
    n = ((w + bx - 1) // bx) * ((h + by - 1) // by)
    out = np.zeros(n * 16, np.uint8)
    sym = np.zeros((n, 108), np.uint32)
    assert _libs.oracle().orc_encode(_libs.ptr(np.ascontiguousarray(img)), w, h, bx, by, 0, _libs.ptr(out), _libs.ptr(sym)) == 0
    return out, sym


def test_block_mode_fields_match_the_oracles_tables():
    """The restated block-mode decoding gives every valid mode's weight range and plane count
    as the oracle's tables (pinned to the reference's decode_block_mode_2d) do."""
    orc = _libs.oracle()
    for bx, by in [(4, 4), (6, 6), (12, 12)]:
        c = np.zeros(13, np.uint32)
        orc.orc_counts(bx, by, _libs.ptr(c))
        nbm = int(c[1])
        bmi = np.zeros(2048, np.uint32)
        bms = np.zeros((max(nbm, 1), 5), np.uint32)
        orc.orc_block_modes(bx, by, _libs.ptr(bmi), _libs.ptr(bms))
        for mode, _, quant, _, dual in bms[:nbm]:
            g = ado.block_mode_grid(int(mode))
            assert g is not None and g[2] == quant and g[3] == dual


@pytest.mark.parametrize("fixed", [False, True])
@pytest.mark.parametrize("bx,by", _libs.FOOTPRINTS)
def test_host_decoder_matches_symbolic_reconstruction(bx, by, fixed):
    w, h = 4 * bx + 3, 3 * by + 2  # ragged edges
    img = synth.make_texture(w, h, 500 + bx * 16 + by)
    with semantics(fixed):
        out, sym = oracle_encode(img, bx, by)
    parts = ado.PartitionTables(_libs.oracle(), bx, by)
    ref = ado.image_from_symbolic(sym, bx, by, w, h, parts)
    assert np.array_equal(ab.decode(bx, by, w, h, out), ref)


def test_every_endpoint_mode_is_covered():
    """Across a few textures, colour and grayscale, every LDR endpoint mode the encoder emits
    is exercised, and every block decodes to its reconstruction."""
    seen = set()
    parts = {}
    for seed, (bx, by) in enumerate([(4, 4), (6, 6), (8, 5), (5, 4)]):
        for gray in (False, True):
            img = synth.make_texture(48, 40, 600 + seed)
            img[:, ::3, 3] = 255 - img[:, ::3, 3]
            if gray:  # luminance and luminance-alpha endpoints
                img[..., 1] = img[..., 2] = img[..., 0]
                img[:20, :, 3] = 255
            out, sym = oracle_encode(img, bx, by)
            for s in sym:
                seen.update(int(s[8 + p]) for p in range(int(s[2])))
            if (bx, by) not in parts:
                parts[(bx, by)] = ado.PartitionTables(_libs.oracle(), bx, by)
            assert np.array_equal(ab.decode(bx, by, 48, 40, out), ado.image_from_symbolic(sym, bx, by, 48, 40, parts[(bx, by)]))
    assert {0, 4, 6, 8, 9, 10, 12, 13} <= seen, seen


@pytest.mark.parametrize("cem,vals,e0,e1", [
    (1, [200, 0xC5], [50 | 0xC0] * 3 + [255], [min(255, (50 | 0xC0) + 5)] * 3 + [255]),
    (8, [10, 20, 30, 40, 50, 60], [10, 30, 50, 255], [20, 40, 60, 255]),
    (8, [20, 10, 40, 30, 60, 50], [(10 + 50) >> 1, (30 + 50) >> 1, 50, 255], [(20 + 60) >> 1, (40 + 60) >> 1, 60, 255]),
    (6, [100, 200, 50, 128], [50, 100, 25, 255], [100, 200, 50, 255]),
])
def test_endpoint_decoding_known_answers(cem, vals, e0, e1):
    """Hand-worked examples of the specification's endpoint rules: luminance delta, RGB direct
    with and without blue contraction, RGB scale."""
    a, b = ado.endpoints(cem, vals)
    assert a == e0 and b == e1
