"""The GPU decoder (astcb200_decode_device / astcb200_decode_error_device): against an
independent reconstruction of every block the GPU encoder emits from its symbolic result
(oracle/astc_decode_oracle.py, written from the ASTC specification), at every footprint,
in both search semantics and for the proposal search; against the host decoder for
void-extent blocks and arbitrary bytes (reserved modes and HDR blocks decode to the error
colour); and the same squared-error sums as a host computation."""
import os
import sys

import numpy as np
import pytest

import _libs
import astc_implementation_b200 as ab
from astc_implementation_b200 import proposal, synth

sys.path.insert(0, os.path.join(_libs.REPO, "oracle"))
import astc_decode_oracle as ado  # noqa: E402

pytestmark = pytest.mark.gpu

FOOTPRINTS = [(4, 4), (5, 4), (5, 5), (6, 5), (6, 6), (8, 5), (8, 6), (8, 8), (10, 5), (10, 6), (10, 8), (10, 10),
              (12, 10), (12, 12)]


def gpu_decode(bx, by, w, h, blocks):
    import torch
    d_blk = torch.from_numpy(np.ascontiguousarray(blocks).reshape(-1)).cuda()
    d_out = torch.zeros(w * h * 4, dtype=torch.uint8, device="cuda")
    s = torch.cuda.current_stream()
    ab.decode_device(bx, by, w, h, d_blk.data_ptr(), d_out.data_ptr(), s.cuda_stream)
    torch.cuda.synchronize()
    return d_out.cpu().numpy().reshape(h, w, 4)


def gpu_sse(bx, by, w, h, blocks, ref):
    import torch
    d_blk = torch.from_numpy(np.ascontiguousarray(blocks).reshape(-1)).cuda()
    d_ref = torch.from_numpy(np.ascontiguousarray(ref).reshape(-1)).cuda()
    d_sse = torch.full((4,), 12345, dtype=torch.int64, device="cuda")  # overwritten, not added to
    s = torch.cuda.current_stream()
    ab.decode_error_device(bx, by, w, h, d_blk.data_ptr(), d_ref.data_ptr(), d_sse.data_ptr(), s.cuda_stream)
    torch.cuda.synchronize()
    return d_sse.cpu().numpy().astype(np.uint64)


def host_sse(a, b):
    d = a.astype(np.int64) - b.astype(np.int64)
    return (d * d).reshape(-1, 4).sum(axis=0).astype(np.uint64)


@pytest.mark.parametrize("bx,by", FOOTPRINTS)
def test_decoder_matches_host_on_encoded_blocks(bx, by):
    w, h = 7 * bx + 3, 5 * by + 2  # ragged edges
    img = synth.make_texture(w, h, 300 + bx * 16 + by)
    n = ((w + bx - 1) // bx) * ((h + by - 1) // by)
    blocks = np.zeros((n, 16), np.uint8)
    assert _libs.oracle().orc_encode(_libs.ptr(img), w, h, bx, by, 0, _libs.ptr(blocks), None) == 0
    host = ab.decode(bx, by, w, h, blocks)
    assert np.array_equal(gpu_decode(bx, by, w, h, blocks), host)
    sse = gpu_sse(bx, by, w, h, blocks, img)
    assert np.array_equal(sse, host_sse(host, img))
    assert abs(ab.psnr_from_sse(sse, w, h) - ab.psnr(host, img)) < 1e-9


@pytest.mark.parametrize("fixed", [False, True])
@pytest.mark.parametrize("bx,by", FOOTPRINTS)
def test_decoder_matches_symbolic_reconstruction_of_gpu_encodes(bx, by, fixed):
    """GPU encode -> GPU decode equals the texels the specification gives for the encoder's
    own symbolic blocks (endpoints, weights, partitioning), for every block."""
    w, h = 6 * bx + 5, 4 * by + 3
    img = synth.make_texture(w, h, 700 + bx * 16 + by)
    enc = ab.ASTCEncoder(device=0, fixed=fixed)
    enc.secondaryInit(w, h, bx, by)
    sym = enc.encode_symbolic(img)
    blocks = enc.encode(img)
    enc.close()
    ref = ado.image_from_symbolic(sym, bx, by, w, h, ado.PartitionTables(_libs.oracle(), bx, by))
    assert np.array_equal(gpu_decode(bx, by, w, h, blocks), ref)


@pytest.mark.parametrize("bx,by", [(4, 4), (6, 6)])
def test_decoder_matches_symbolic_reconstruction_of_proposal_search(bx, by):
    w, h = 40 * bx + 1, 30 * by + 2
    img = synth.make_texture(w, h, 800 + bx)
    enc = ab.ASTCEncoder(device=0)
    enc.set_proposal_net(proposal.load_weights(bx, by))
    enc.set_pruning(True)
    enc.secondaryInit(w, h, bx, by)
    sym = enc.encode_symbolic(img)
    blocks = enc.encode(img)
    assert enc.pruning_stats()[0] > 0
    enc.close()
    ref = ado.image_from_symbolic(sym, bx, by, w, h, ado.PartitionTables(_libs.oracle(), bx, by))
    assert np.array_equal(gpu_decode(bx, by, w, h, blocks), ref)


@pytest.mark.parametrize("bx,by", [(4, 4), (6, 6), (8, 5), (12, 12)])
def test_decoder_matches_host_on_arbitrary_bytes(bx, by):
    rng = np.random.default_rng(bx * 100 + by)
    w, h = 40 * bx, 30 * by
    n = 40 * 30
    blocks = rng.integers(0, 256, (n, 16), dtype=np.uint8)
    ve = rng.random(n) < 0.2  # void-extent blocks, LDR and HDR
    blocks[ve, 0] = 0xFC
    blocks[ve, 1] = (blocks[ve, 1] & 0xFC) | 0x01
    host = ab.decode(bx, by, w, h, blocks)
    gpu = gpu_decode(bx, by, w, h, blocks)
    assert np.array_equal(gpu, host)
    magenta = (host == np.array([255, 0, 255, 255], np.uint8)).all(axis=2)
    assert magenta.any() and (~magenta).any()  # both error and valid blocks occur
    ref = rng.integers(0, 256, (h, w, 4), dtype=np.uint8)
    assert np.array_equal(gpu_sse(bx, by, w, h, blocks, ref), host_sse(host, ref))


def test_decoder_argument_errors():
    with pytest.raises(ab.ASTCError):
        ab.decode_device(7, 7, 16, 16, 1 << 20, 1 << 20)
    with pytest.raises(ab.ASTCError):
        ab.decode_device(4, 4, 0, 16, 1 << 20, 1 << 20)
    with pytest.raises(ab.ASTCError):
        ab.decode_device(4, 4, 16, 16, 1 << 20, (1 << 20) + 1)  # unaligned image
