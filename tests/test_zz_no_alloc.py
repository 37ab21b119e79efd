"""The allocation-free entry point (astcb200_encode_noalloc).

Some callers cannot allocate device memory: an engine whose own allocator owns the
whole device heap, a plug-in inside a process with a fixed allocation policy.  For
them the library keeps a fixed 52 MiB array in device memory (intermediates and the
tables of the footprints used) and encodes at most 2048 blocks per call into buffers
the caller already owns.  This file is collected last so that a run stopping at the
first failure has run every other test first.
"""
import numpy as np
import pytest

import astc_implementation_b200 as ab
from astc_implementation_b200 import synth

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("w,h,bx,by", [(160, 96, 4, 4), (90, 66, 6, 6)])
def test_noalloc_matches_regular_entry_twice(w, h, bx, by):
    import torch
    img = synth.make_texture(w, h, 21)
    enc = ab.ASTCEncoder(device=0)
    enc.secondaryInit(w, h, bx, by)
    d_in = torch.from_numpy(img.reshape(-1)).cuda()
    ref = torch.zeros(enc.numBlocks * 16, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    enc.encode_device(d_in.data_ptr(), ref.data_ptr(), stream)
    torch.cuda.synchronize()
    expected = ref.cpu().numpy()
    assert expected.any()
    for _ in range(2):  # the second call reuses the scratch left by the first
        out = torch.full((enc.numBlocks * 16,), 0xAA, dtype=torch.uint8, device="cuda")
        ab.encode_noalloc(0, d_in.data_ptr(), w, h, bx, by, out.data_ptr(), stream)
        torch.cuda.synchronize()
        assert np.array_equal(out.cpu().numpy(), expected)  # bit-exact, the encoder's tolerance
    enc.close()


def test_noalloc_rejects_oversized_request():
    import torch
    d = torch.zeros(16, dtype=torch.uint8, device="cuda")
    with pytest.raises(ab.ASTCError) as e:
        ab.encode_noalloc(0, d.data_ptr(), 1024, 1024, 4, 4, d.data_ptr())
    assert e.value.status == ab.TOO_LARGE


def test_noalloc_allocates_nothing_after_set_up():
    """Once a device and its footprints are set up, calls with other images of those
    footprints leave the device's free memory unchanged, and still match the regular
    entry point."""
    import torch
    cases = [(160, 96, 4, 4, 31), (90, 66, 6, 6, 32), (150, 100, 4, 4, 33), (84, 72, 6, 6, 34)]
    enc = ab.ASTCEncoder(device=0)
    stream = torch.cuda.current_stream().cuda_stream
    ins, outs, expected = [], [], []
    for w, h, bx, by, seed in cases:
        img = synth.make_texture(w, h, seed)
        enc.secondaryInit(w, h, bx, by)
        d_in = torch.from_numpy(img.reshape(-1)).cuda()
        ref = torch.zeros(enc.numBlocks * 16, dtype=torch.uint8, device="cuda")
        enc.encode_device(d_in.data_ptr(), ref.data_ptr(), stream)
        ins.append(d_in)
        outs.append(torch.full((enc.numBlocks * 16,), 0xAA, dtype=torch.uint8, device="cuda"))
        expected.append(ref)
    torch.cuda.synchronize()
    expected = [e.cpu().numpy() for e in expected]
    for (w, h, bx, by, _), d_in, out in zip(cases[:2], ins[:2], outs[:2]):  # set-up: device, 4x4, 6x6
        ab.encode_noalloc(0, d_in.data_ptr(), w, h, bx, by, out.data_ptr(), stream)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info(0)[0]
    for (w, h, bx, by, _), d_in, out in zip(cases[2:], ins[2:], outs[2:]):
        ab.encode_noalloc(0, d_in.data_ptr(), w, h, bx, by, out.data_ptr(), stream)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info(0)[0] == free0
    for out, exp in zip(outs, expected):
        assert np.array_equal(out.cpu().numpy(), exp)
    enc.close()
