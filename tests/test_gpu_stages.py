"""Per-stage parity of the full search: the GPU's partition picks (passes 001-007), the
front's partitioned-block records (pass01's averages and endpoints, pass12's candidates with
their quant levels, formats and quantised weights) and every candidate's best state after the
refinement (passes 13-17) against the CPU oracle, block by block, slot by slot and candidate
by candidate, in both semantics.  The end-to-end parity tests compare only the final blocks,
where a stage error that does not change the winning candidate would stay invisible."""
import numpy as np
import pytest

import _libs
import astc_implementation_b200 as ab
from astc_implementation_b200 import synth

pytestmark = pytest.mark.gpu

FOOTPRINTS = [(4, 4), (6, 6), (8, 5), (10, 6), (12, 12)]


def same_bits(a, b):
    """Bit-identical floats, NaN equal to NaN whatever its payload (the GPU writes the canonical
    NaN, the host CPU its own default): the endpoints of a partition with no texels."""
    a, b = np.asarray(a, np.float32), np.asarray(b, np.float32)
    return bool(np.all((a.view(np.uint32) == b.view(np.uint32)) | (np.isnan(a) & np.isnan(b))))


def oracle_front(bx, by, tex, P, entry):
    ep = np.zeros(48, np.float32)
    cands = np.zeros((8, 71), np.uint32)
    n = _libs.oracle().orc_front_candidates(bx, by, _libs.ptr(np.ascontiguousarray(tex)), P, entry, _libs.ptr(ep),
                                             _libs.ptr(cands))
    assert n >= 0
    return n, ep.reshape(4, 3, 4), cands


@pytest.mark.parametrize("fixed", [False, True])
@pytest.mark.parametrize("bx,by", FOOTPRINTS)
def test_partition_picks_and_front_records_match_the_oracle(bx, by, fixed):
    w, h = 6 * bx + 1, 4 * by + 3  # ragged edges
    img = synth.make_texture(w, h, 700 + bx * 16 + by)
    enc = ab.ASTCEncoder(device=0, fixed=fixed)
    enc.secondaryInit(w, h, bx, by)
    picks, recs, snaps = enc.search_stages(img)
    enc.close()
    tex = synth.texel_blocks(img, bx, by)
    orc = _libs.oracle()
    prev = orc.orc_set_semantics(1 if fixed else 0)
    try:
        n_cands = 0
        for b in range(tex.shape[0]):
            # passes 001-007: up to four table entries per partition count
            slots = [(1, 0)]
            for P in (2, 3, 4):
                ent = np.zeros(4, np.uint32)
                n = orc.orc_partition_search(bx, by, _libs.ptr(np.ascontiguousarray(tex[b])), P, _libs.ptr(ent))
                got = picks[b, (P - 2) * 5:(P - 2) * 5 + 5]
                assert int(got[4]) == n, (b, P)
                expect = [int(e) - (P - 2) * 1024 for e in ent[:n]]
                assert [int(v) for v in got[:n]] == expect, (b, P)
                slots += [(P, e) for e in expect] + [None] * (4 - n)
            # passes 01-12 of every present slot
            for s, item in enumerate(slots):
                r = recs[b, s]
                if item is None:
                    assert int(r["ncand"]) == 0
                    continue
                P, entry = item
                n, ep, cands = oracle_front(bx, by, tex[b], P, entry)
                assert int(r["P"]) == P and int(r["entry"]) == entry and int(r["ncand"]) == n, (b, s)
                for name, k in (("avg", 0), ("ep0", 1), ("ep1", 2)):
                    assert same_bits(r[name], ep[:, k, :]), (b, s, name)
                for k in range(n):
                    c = r["cand"][k]
                    o = cands[k]
                    assert (int(c["bm"]), int(c["ql"]), int(c["qlm"])) == (int(o[0]), int(o[1]), int(o[2])), (b, s, k)
                    assert [int(v) for v in c["fmt"]] == [int(v) for v in o[3:7]], (b, s, k)
                    assert np.array_equal(c["qw"].astype(np.uint32), o[7:71]), (b, s, k)
                # passes 13-17: each candidate's best state after the reference's 6 iterations
                ref = np.zeros((8, 104), np.uint32)
                assert orc.orc_refined_candidates(bx, by, _libs.ptr(np.ascontiguousarray(tex[b])), P, entry, 6, _libs.ptr(ref)) == n
                for k in range(8):
                    g, o = snaps[b, s, k], ref[k]
                    assert int(np.float32(g["err"]).view(np.uint32)) == int(o[0]), (b, s, k, "error")
                    if k >= n:
                        continue
                    assert (int(g["bm"]), int(g["final_q"]), int(g["matched"])) == (int(o[1]), int(o[2]), int(o[3])), (b, s, k)
                    assert [int(v) for v in g["ffmt"]] == [int(v) for v in o[4:8]], (b, s, k)
                    assert np.array_equal(g["packed"].astype(np.uint32), o[8:40]), (b, s, k, "packed")
                    assert np.array_equal(g["qw"].astype(np.uint32), o[40:104]), (b, s, k, "weights")
                n_cands += n
        assert n_cands > 0
    finally:
        orc.orc_set_semantics(prev)
