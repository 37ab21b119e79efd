"""Proposal network: the CPU checker itself (finite differences), label extraction
from the full search's symbolic blocks, class layout and the selection rule."""
import os
import sys

import numpy as np
import pytest

import _libs
from astc_implementation_b200 import proposal, synth

sys.path.insert(0, os.path.join(_libs.REPO, "oracle"))
import mlp_oracle as mo  # noqa: E402


def tiny_problem(seed=0, B=3):
    lay = proposal.Layout(4, 4)
    rng = np.random.default_rng(seed)
    w = proposal.init_weights(lay, seed=seed)
    w["b1"] = rng.normal(0, 0.1, 256).astype(np.float32)
    w["b2"] = rng.normal(0, 0.1, 256).astype(np.float32)
    w["w3"] *= 5.0
    img = synth.make_texture(16, 16, seed + 3)
    x = mo.inputs(mo.block_rgba8(img, 4, 4)[:B], lay.inputs_padded)
    part = np.array([5, lay.part_class(3, 7), lay.p1][:B])
    bm = np.array([3, 10, 0][:B])
    return lay, w, x, part, bm


def test_layout_matches_class_plan():
    for bx, by, nbm in [(4, 4, 53), (6, 6, 198)]:
        lay = proposal.Layout(bx, by)
        cl = mo.Classes(lay.sel3)
        assert lay.inputs == 4 * bx * by and lay.inputs_padded % 16 == 0
        assert lay.nbm == nbm and lay.head_base == cl.head_base and lay.head_stride >= nbm
        assert lay.p1 == cl.p1 == sum(lay.sel3) and lay.part_base == cl.part_base
        assert lay.outputs % 128 == 0 and lay.outputs >= lay.head_base + 4 * lay.head_stride
        assert lay.outputs < lay.head_base + 4 * lay.head_stride + 128  # no more padding than the alignment
        assert all(0 < s <= 1024 for s in lay.sel3)
        c = np.arange(lay.p1)
        v = lay.pick_of(c)
        assert (lay.part_class(2 + (v >> 10), v & 1023) == c).all() and ((v & 1023) < np.array(lay.sel3)[v >> 10]).all()
        assert (lay.head_of(c) == 1 + (v >> 10)).all() and lay.head_of(lay.p1) == 0


def test_bf16_rounding_ties_to_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, 1.0 + 2 ** -9, -2.5], np.float32)
    r = mo.bf16_round(x)
    assert list(r) == [1.0, 1.0, 1.0 + 4 * 2 ** -8, 1.0, -2.5]
    assert np.array_equal(proposal.bf16_round(x), r)


def test_oracle_gradients_match_finite_differences():
    lay, w, x, part, bm = tiny_problem()
    lp, lb, g, _ = mo.loss_and_grads(x, w, part, bm, lay.nbm, lay.head_stride, lay.sel3)
    rng = np.random.default_rng(1)
    W = {k: v.astype(np.float64) for k, v in w.items()}

    def loss(WW):
        a, b, _, _ = mo.loss_and_grads(x, WW, part, bm, lay.nbm, lay.head_stride, lay.sel3)
        return a + b

    for key in ("w1", "b1", "w2", "b2", "w3", "b3"):
        flat = W[key].reshape(-1)
        idx = rng.choice(flat.size, 6, replace=False)
        if key == "w3":  # entries that feed the labelled classes carry most of the gradient
            idx = np.concatenate([idx, [part[0] * 256 + 3, (lay.head_base + 3) * 256 + 5]])
        for i in idx:
            h = 1e-6
            Wp = {k: v.copy() for k, v in W.items()}
            Wm = {k: v.copy() for k, v in W.items()}
            Wp[key].reshape(-1)[i] += h
            Wm[key].reshape(-1)[i] -= h
            fd = (loss(Wp) - loss(Wm)) / (2 * h)
            an = g[key].reshape(-1)[i]
            assert abs(fd - an) <= 1e-6 + 1e-5 * abs(an), (key, i, fd, an)


def test_oracle_softmax_gradient_sums_to_zero():
    lay, w, x, part, bm = tiny_problem(seed=4)
    _, _, _, dz = mo.loss_and_grads(x, w, part, bm, lay.nbm, lay.head_stride, lay.sel3)
    assert np.allclose(dz[:, : lay.p1 + 1].sum(axis=1), 0.0, atol=1e-12)
    assert np.all(dz[:, lay.p1 + 1: lay.head_base] == 0.0)  # padding before the heads
    heads = lay.head_of(part)
    for i in range(len(part)):
        h0 = lay.head_base + heads[i] * lay.head_stride
        assert abs(dz[i, h0: h0 + lay.nbm].sum()) < 1e-12
        other = np.delete(np.arange(lay.head_base, lay.outputs), np.arange(h0 - lay.head_base, h0 - lay.head_base + lay.nbm))
        assert np.all(dz[i, other] == 0.0)


def test_labels_from_full_search_symbolic_blocks():
    img = synth.make_texture(48, 40, 21)
    n = 12 * 10
    sym = np.zeros((n, 108), np.uint32)
    out = np.zeros((n, 16), np.uint8)
    assert _libs.oracle().orc_encode(_libs.ptr(img), 48, 40, 4, 4, 0, _libs.ptr(out), _libs.ptr(sym)) == 0
    part, bm, ok = proposal.labels_from_symbolic(sym, 4, 4)
    lay = proposal.Layout(4, 4)
    assert ok.all()
    assert (part >= 0).all() and (part <= lay.p1).all()
    assert ((part == lay.p1) == (sym[:, 2] == 1)).all()
    v = lay.pick_of(part[part != lay.p1])
    assert (2 + (v >> 10) == sym[part != lay.p1, 2]).all()
    assert (bm >= 0).all() and (bm < lay.nbm).all()
    modes = proposal._trial_modes(4, 4)
    assert (modes[bm] == sym[:, 1]).all()
    assert len(set(part.tolist())) > 3


def test_oracle_select_rule():
    lay = proposal.Layout(4, 4)
    z = np.full(lay.outputs, -30.0)
    z[lay.p1] = 0.0
    z[lay.part_class(2, 17)] = 1.0  # P=2 entry 17, the best
    z[lay.part_class(3, 3)] = 0.5   # P=3 entry 3
    z[lay.head_base] = 50.0          # a block-mode logit: never a partition class
    conf, picks, modes = mo.select(z, lay.sel3, 4, 0.99, 0.5, 2, lay.nbm, lay.head_stride)
    assert conf and picks[:2] == [lay.part_class(2, 17), lay.part_class(3, 3)]
    assert all(len(m) == 2 for m in modes)
    conf, picks, _ = mo.select(z, lay.sel3, 4, 0.5, 0.5, 2, lay.nbm, lay.head_stride)
    assert picks == [lay.part_class(2, 17)]  # P=1 (0.27) + entry 17 (0.72) reaches the coverage
    conf, _, _ = mo.select(np.zeros(lay.outputs), lay.sel3, 4, 0.9, 0.5, 2, lay.nbm, lay.head_stride)
    assert not conf  # flat logits: five classes of ~1100 carry almost nothing
