"""Integer and constant tables: the oracle's and the product's, against the
reference's own compiled code (digests in tests/golden) and its WGSL text."""
import hashlib

import numpy as np
import pytest

import _libs
import astc_implementation_b200 as ab


def _golden_digests():
    g = _libs.golden_tables()
    return dict(zip(list(g["digest_names"]), g["digests"]))


@pytest.mark.parametrize("bx,by", _libs.FOOTPRINTS)
def test_oracle_footprint_tables_match_reference(bx, by):
    gold = _golden_digests()
    got = _libs.footprint_digests(_libs.oracle(), "orc_", bx, by)
    bad = [k for k, v in got.items() if gold[k] != v]
    assert not bad, bad


@pytest.mark.parametrize("bx,by", _libs.FOOTPRINTS)
def test_product_footprint_tables_match_reference(bx, by):
    gold = _golden_digests()
    got = _libs.footprint_digests(ab.load_library(), "astcb200_tables_", bx, by)
    bad = [k for k, v in got.items() if gold[k] != v]
    assert not bad, bad


def test_angular_tables_match_reference():
    gold = _golden_digests()
    for lib, fn in [(_libs.oracle(), "orc_angular"), (ab.load_library(), "astcb200_tables_angular")]:
        s = np.zeros(16384, np.float32)
        c = np.zeros(16384, np.float32)
        getattr(lib, fn)(_libs.ptr(s), _libs.ptr(c))
        assert hashlib.sha256(s.tobytes()).hexdigest() == gold["angular:sin"]
        assert hashlib.sha256(c.tobytes()).hexdigest() == gold["angular:cos"]


def test_constant_tables_match_reference_sources():
    g = _libs.golden_tables()
    P = _libs.ptr
    q2u = np.zeros(142, np.int32); qmt = np.zeros((10, 128), np.int32); cu = np.zeros((17, 512), np.int32)
    pn = np.zeros((12, 65), np.int32); bqe = np.zeros(17, np.float32); tr = np.zeros(243, np.uint8)
    qu = np.zeros(125, np.uint8); ws = np.zeros((12, 32), np.uint8); cs = np.zeros((17, 256), np.uint8)
    _libs.oracle().orc_const_tables(P(q2u), P(qmt), P(cu), P(pn), P(bqe), P(tr), P(qu), P(ws), P(cs))
    assert np.array_equal(q2u, g["quant_to_unquant"])
    assert np.array_equal(qmt, g["quant_mode_table"])
    assert np.array_equal(cu, g["color_unquant_to_uquant"])
    assert np.array_equal(pn, g["prev_next_values"])
    assert np.array_equal(bqe, g["baseline_quant_error"])
    assert np.array_equal(tr, g["integer_of_trits"].ravel())
    assert np.array_equal(qu, g["integer_of_quints"].ravel())
    assert np.array_equal(ws, g["weight_scramble"])
    assert np.array_equal(cs, g["color_scramble"])


@pytest.mark.parametrize("bx,by,ndm,nbm", [(4, 4, 6, 53), (6, 6, 22, 198), (8, 8, 46, 339), (12, 12, 84, 521)])
def test_trial_mode_counts(bx, by, ndm, nbm):
    nd = np.zeros(1, np.uint32); nb = np.zeros(1, np.uint32)
    _libs.oracle().orc_trial_modes(bx, by, _libs.ptr(nd), None, _libs.ptr(nb), None)
    assert (int(nd[0]), int(nb[0])) == (ndm, nbm)


def test_oracle_tables_match_live_reference_build():
    ref = _libs.ref_lib()
    if ref is None:
        pytest.skip("oracle/_ref not built (needs the reference checkout)")
    for bx, by in [(4, 4), (6, 6), (12, 12), (10, 5)]:
        assert _libs.footprint_digests(ref, "astcref_", bx, by) == _libs.footprint_digests(_libs.oracle(), "orc_", bx, by)


def test_colour_quant_table_non_decreasing():
    """The refinement's endpoint quantisation search (k_refine, Packer::quant_rgb) finds the
    stop of the reference's nudge loop by bisection, which needs every level's colour
    quantise-unquantise table to be non-decreasing in its index."""
    cu = _libs.golden_tables()["color_unquant_to_uquant"]
    assert cu.shape == (17, 512)
    assert (np.diff(cu.astype(np.int64), axis=1) >= 0).all()


def _nudge_stepwise(tab, c0, c1):
    """The reference's loop (pass14 quantize_rgb): step k uses the endpoints after k nudges."""
    f32 = np.float32
    a = b = None
    for _ in range(4096):
        a = [tab[2 * max(int(np.rint(v)), 0) + (1 if f32(v - f32(max(int(np.rint(v)), 0))) >= f32(-0.1) else 0)] for v in c0]
        c0 = [f32(v - f32(0.2)) for v in c0]
        b = [tab[2 * min(int(np.rint(v)), 255) + (1 if f32(v - f32(min(int(np.rint(v)), 255))) >= f32(-0.1) else 0)] for v in c1]
        c1 = [f32(v + f32(0.2)) for v in c1]
        if sum(a) <= sum(b):
            break
    return a, b


def _nudge_bisect(tab, c0, c1):
    """The same stop found as k_refine does: probes at steps 0, 1, 3, 7, ... then bisection,
    endpoints advanced from an earlier probed step by the loop's own float steps."""
    f32 = np.float32

    def probe(x0, x1):
        a = [tab[2 * max(int(np.rint(v)), 0) + (1 if f32(v - f32(max(int(np.rint(v)), 0))) >= f32(-0.1) else 0)] for v in x0]
        b = [tab[2 * min(int(np.rint(v)), 255) + (1 if f32(v - f32(min(int(np.rint(v)), 255))) >= f32(-0.1) else 0)] for v in x1]
        return sum(a) <= sum(b), a, b

    def advance(x0, x1, n):
        for _ in range(n):
            x0 = [f32(v - f32(0.2)) for v in x0]
            x1 = [f32(v + f32(0.2)) for v in x1]
        return x0, x1

    ok, a, b = probe(c0, c1)
    if ok:
        return a, b
    lo, step = 0, 1
    while True:
        hi = min(lo + step, 4095)
        t0, t1 = advance(c0, c1, hi - lo)
        ok, a, b = probe(t0, t1)
        if ok or hi == 4095:
            break
        c0, c1, lo, step = t0, t1, hi, step * 2
    while hi - lo > 1:
        mid = lo + (hi - lo) // 2
        t0, t1 = advance(c0, c1, mid - lo)
        ok, a, b = probe(t0, t1)
        if ok:
            hi = mid
        else:
            lo, c0, c1 = mid, t0, t1
    c0, c1 = advance(c0, c1, 1)
    _, a, b = probe(c0, c1)
    return a, b


def test_nudge_loop_bisection_matches_stepwise():
    """The bisection's result equals the reference loop's on random endpoints in [0, 255]
    at every quant level, inverted pairs (long loops) and half-step values included."""
    cu = _libs.golden_tables()["color_unquant_to_uquant"]
    rng = np.random.default_rng(11)
    f32 = np.float32
    for i in range(600):
        tab = [int(v) for v in cu[i % 17]]
        c0 = [f32(v) for v in rng.uniform(0, 255, 3)]
        c1 = [f32(v) for v in rng.uniform(0, 255, 3)]
        if i % 3 == 1:  # bright low endpoint, dark high one: hundreds of steps
            c0 = [f32(v) for v in rng.uniform(200, 255, 3)]
            c1 = [f32(v) for v in rng.uniform(0, 40, 3)]
        if i % 5 == 2:
            c0 = [f32(np.floor(v) + 0.5) for v in c0]
        assert _nudge_bisect(tab, c0, c1) == _nudge_stepwise(tab, c0, c1), i
