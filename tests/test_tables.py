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
