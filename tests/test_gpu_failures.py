"""Failure paths on the GPU, made to fire without faulting or hanging anything: the host
wait's timeout on a long encode, and the network kernel's bounded mbarrier waits given a
limit too small for the work in flight.  After each, the same context encodes correctly."""
import numpy as np
import pytest

import _libs
import astc_implementation_b200 as ab
from astc_implementation_b200 import proposal, synth

pytestmark = pytest.mark.gpu


def oracle_encode(img, bx, by):
    h, w = img.shape[:2]
    n = ((w + bx - 1) // bx) * ((h + by - 1) // by)
    out = np.zeros(n * 16, np.uint8)
    assert _libs.oracle().orc_encode(_libs.ptr(np.ascontiguousarray(img)), w, h, bx, by, 0, _libs.ptr(out), None) == 0
    return out


def test_host_timeout_then_context_still_correct():
    big = synth.make_texture(2048, 2048, 1)  # the full search takes a few hundred ms here
    small = synth.make_texture(64, 48, 2)
    enc = ab.ASTCEncoder(device=0, timeout_ms=1)
    enc.secondaryInit(2048, 2048, 4, 4)
    out = np.full(enc.numBlocks * 16, 0xAB, np.uint8)
    with pytest.raises(ab.ASTCError) as e:
        enc.encode(big, out)
    assert e.value.status == ab.TIMEOUT
    enc.set_timeout(0)
    # the next call queues behind the timed-out work and waits for both
    enc.secondaryInit(64, 48, 4, 4)
    assert np.array_equal(enc.encode(small), oracle_encode(small, 4, 4))
    # the timed-out call's blocks went to the context's staging, never to the caller's buffer
    assert (out == 0xAB).all()
    enc.secondaryInit(2048, 2048, 4, 4)
    again = enc.encode(big)
    enc.close()
    fresh = ab.ASTCEncoder(device=0)
    fresh.secondaryInit(2048, 2048, 4, 4)
    assert np.array_equal(again, fresh.encode(big))
    fresh.close()


def test_host_timeout_pinned_output_is_written_later():
    """With pinned host buffers the timed-out call's copy stays queued and lands once the work
    completes; a later call on the context returns only after that."""
    import torch
    img = synth.make_texture(1024, 1024, 3)
    enc = ab.ASTCEncoder(device=0, timeout_ms=1)
    enc.secondaryInit(1024, 1024, 4, 4)
    pin_in = torch.from_numpy(img.reshape(-1)).pin_memory()
    pin_out = torch.full((enc.numBlocks * 16,), 0xAB, dtype=torch.uint8).pin_memory()
    with pytest.raises(ab.ASTCError) as e:
        enc.encode(pin_in.numpy(), pin_out.numpy())
    assert e.value.status == ab.TIMEOUT
    enc.set_timeout(0)
    ref = enc.encode(img)  # returns after the earlier work and its copy
    assert np.array_equal(pin_out.numpy(), ref)
    enc.close()


def test_inference_wait_limit_gives_up_then_recovers():
    bx = by = 4
    img = synth.make_texture(512, 512, 5)
    lay = proposal.Layout(bx, by)
    enc = ab.ASTCEncoder(device=0)
    enc.set_proposal_net(proposal.load_weights(bx, by))
    enc.secondaryInit(512, 512, bx, by)
    z_ok = enc.proposal_logits(img, lay.outputs)
    enc.set_inference_wait_limit(1)  # one non-blocking poll: every CTA finds its copies or MMAs in flight
    with pytest.raises(ab.ASTCError) as e:
        enc.proposal_logits(img, lay.outputs)
    assert e.value.status == ab.TIMEOUT
    enc.set_inference_wait_limit(0)
    z = enc.proposal_logits(img, lay.outputs)
    assert np.array_equal(z, z_ok)
    enc.set_pruning(True)
    blocks = enc.encode(img)
    assert enc.pruning_stats()[0] > 0
    enc.close()
    again = ab.ASTCEncoder(device=0)
    again.set_proposal_net(proposal.load_weights(bx, by))
    again.set_pruning(True)
    again.secondaryInit(512, 512, bx, by)
    assert np.array_equal(blocks, again.encode(img))
    again.close()


def test_inference_wait_limit_rejects_bad_values():
    enc = ab.ASTCEncoder(device=0)
    with pytest.raises(ab.ASTCError):
        enc.set_inference_wait_limit(1 << 31)
    enc.close()
