"""Batched encoding (astcb200_encode_batch*, autotuner, mip downsampler) on the GPU.

Every texture of a batch must get exactly the blocks a single-image encode gives
it (which the parity tests pin to the oracle), whatever the mix of sizes and
footprints, the launch configuration and whether the CUDA graph is replayed.
"""
import numpy as np
import pytest

import _libs
import astc_implementation_b200 as ab
from astc_implementation_b200 import synth

pytestmark = pytest.mark.gpu

# ragged sizes, three footprints, 1x1 and sub-block textures included
MIXED = [((37, 19), (4, 4)), ((64, 64), (6, 6)), ((100, 53), (8, 8)), ((5, 3), (4, 4)),
         ((1, 1), (6, 6)), ((130, 70), (4, 4)), ((23, 41), (8, 8)), ((48, 30), (6, 6))]


def textures(seed0):
    return [(synth.make_texture(w, h, seed0 + i), bx, by) for i, ((w, h), (bx, by)) in enumerate(MIXED)]


@pytest.fixture(scope="module")
def enc():
    e = ab.ASTCEncoder(device=0)
    e.init()
    yield e
    e.close()


def single(enc, img, bx, by):
    h, w = img.shape[:2]
    enc.secondaryInit(w, h, bx, by)
    return enc.encode(img)


def test_batch_equals_single_image_encodes(enc):
    tex = textures(500)
    outs = enc.encode_batch(tex)
    st = enc.last_stats
    assert st.blocks == sum(o.size // 16 for o in outs) and st.launches > 0
    assert st.h2d_bytes == sum(img.size for img, _, _ in tex)
    for (img, bx, by), out in zip(tex, outs):
        assert np.array_equal(out, single(enc, img, bx, by)), (img.shape, bx, by)


def test_batch_matches_oracle_small():
    tex = [(synth.make_texture(21, 13, 7), 4, 4), (synth.make_texture(14, 9, 8), 6, 6)]
    e = ab.ASTCEncoder(device=0)
    outs = e.encode_batch(tex)
    e.close()
    for (img, bx, by), out in zip(tex, outs):
        h, w = img.shape[:2]
        n = ((w + bx - 1) // bx) * ((h + by - 1) // by)
        ref = np.zeros((n, 16), np.uint8)
        assert _libs.oracle().orc_encode(_libs.ptr(np.ascontiguousarray(img)), w, h, bx, by, 0, _libs.ptr(ref), None) == 0
        assert np.array_equal(out.reshape(n, 16), ref)


def test_graph_replay_with_new_contents(enc):
    a, b = textures(600), textures(700)  # same shape, different texels
    enc.encode_batch(a)
    outs = enc.encode_batch(b)  # replays the graph captured for this shape
    for (img, bx, by), out in zip(b, outs):
        assert np.array_equal(out, single(enc, img, bx, by))


def test_no_graph_and_small_chunks_identical():
    tex = textures(800)
    e1 = ab.ASTCEncoder(device=0)
    ref = e1.encode_batch(tex)
    e1.close()
    e2 = ab.ASTCEncoder(device=0, chunk_blocks=64, use_graphs=False)  # many chunks over 4 streams
    outs = e2.encode_batch(tex)
    e2.close()
    for r, o in zip(ref, outs):
        assert np.array_equal(r, o)


def test_device_batch_and_autotune(enc):
    import torch
    tex = textures(900)
    d_in, d_out, desc = [], [], []
    for img, bx, by in tex:
        h, w = img.shape[:2]
        n = ((w + bx - 1) // bx) * ((h + by - 1) // by)
        d_in.append(torch.from_numpy(img.reshape(-1)).cuda())
        d_out.append(torch.zeros(n * 16, dtype=torch.uint8, device="cuda"))
        desc.append((d_in[-1].data_ptr(), w, h, bx, by, d_out[-1].data_ptr(), n * 16))
    best, tried = enc.autotune_batch(desc)
    assert len(tried) >= 1 and best[2] > 0 and best[:2] in [t[:2] for t in tried]
    for o in d_out:
        o.zero_()
    stream = torch.cuda.current_stream()
    enc.encode_batch_device(desc, stream.cuda_stream)
    torch.cuda.synchronize()
    for (img, bx, by), o in zip(tex, d_out):
        assert np.array_equal(o.cpu().numpy(), single(enc, img, bx, by))


def box_down(img):
    h, w = img.shape[:2]
    dh, dw = max(1, h // 2), max(1, w // 2)
    ys, xs = np.arange(dh), np.arange(dw)
    y0, y1 = np.minimum(2 * ys, h - 1), np.minimum(2 * ys + 1, h - 1)
    x0, x1 = np.minimum(2 * xs, w - 1), np.minimum(2 * xs + 1, w - 1)
    s = (img[y0][:, x0].astype(np.int32) + img[y0][:, x1] + img[y1][:, x0] + img[y1][:, x1] + 2) >> 2
    return s.astype(np.uint8)


def test_mip_chain_downsample_and_batch(enc):
    import torch
    img = synth.make_texture(45, 22, 31)
    dims = ab.mip_dims(45, 22)
    assert dims[-1] == (1, 1) and dims[1] == (22, 11)
    level = torch.from_numpy(img.reshape(-1)).cuda()
    ref = img
    chain = [img]
    for (w, h), (dw, dh) in zip(dims[:-1], dims[1:]):
        nxt = torch.empty(dw * dh * 4, dtype=torch.uint8, device="cuda")
        ab.downsample_device(level.data_ptr(), w, h, nxt.data_ptr(), torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        ref = box_down(ref)
        got = nxt.cpu().numpy().reshape(dh, dw, 4)
        assert np.array_equal(got, ref), (dw, dh)
        chain.append(got)
        level = nxt
    outs = enc.encode_batch([(m, 6, 6) for m in chain] + [(m, 4, 4) for m in chain])
    for (m, bx, by), o in zip([(m, 6, 6) for m in chain] + [(m, 4, 4) for m in chain], outs):
        assert np.array_equal(o, single(enc, m, bx, by))


def test_astc_containers_from_device_equal_store_image(enc, tmp_path):
    """astcb200_astc_containers_device: header and blocks copied from device memory are the
    bytes store_image writes for the same blocks."""
    import torch
    tex = textures(700)
    d_img = [torch.from_numpy(img.reshape(-1)).cuda() for img, _, _ in tex]
    nb = [((img.shape[1] + bx - 1) // bx) * ((img.shape[0] + by - 1) // by) for img, bx, by in tex]
    d_out = [torch.empty(n * 16, dtype=torch.uint8, device="cuda") for n in nb]
    s = torch.cuda.current_stream().cuda_stream
    enc.encode_batch_device([(d_img[i].data_ptr(), img.shape[1], img.shape[0], bx, by, d_out[i].data_ptr(), nb[i] * 16)
                             for i, (img, bx, by) in enumerate(tex)], s)
    host = [torch.zeros(16 + n * 16, dtype=torch.uint8).pin_memory().numpy() for n in nb]
    ab.astc_containers_device([(d_out[i].data_ptr(), host[i], img.shape[1], img.shape[0], bx, by)
                               for i, (img, bx, by) in enumerate(tex)], s)
    torch.cuda.synchronize()
    for i, (img, bx, by) in enumerate(tex):
        path = tmp_path / ("t%d.astc" % i)
        ab.store_image(bx, by, img.shape[1], img.shape[0], single(enc, img, bx, by), str(path))
        assert bytes(host[i]) == path.read_bytes()
    with pytest.raises(ab.ASTCError):  # host_out too small
        ab.astc_containers_device([(d_out[0].data_ptr(), host[0][:-1].copy(), 37, 19, 4, 4)], s)


def test_mip_chain_astc_writer(enc, tmp_path):
    """The mip-chain writer (downsampled, encoded and containerised on the device) gives,
    per level, the file store_image writes for a single encode of that level."""
    from astc_implementation_b200 import mipchain
    img = synth.make_texture(45, 22, 33)
    dims = ab.mip_dims(45, 22)
    paths = [str(tmp_path / ("level%d.astc" % i)) for i in range(len(dims))]
    files = mipchain.encode_mip_chain_astc(enc, img, 6, 6, paths=paths)
    assert len(files) == len(dims)
    ref = img
    for i, ((w, h), data) in enumerate(zip(dims, files)):
        if i:
            ref = box_down(ref)
        path = tmp_path / "ref.astc"
        ab.store_image(6, 6, w, h, single(enc, ref, 6, 6), str(path))
        assert data == path.read_bytes()
        assert open(paths[i], "rb").read() == data
    assert len(mipchain.encode_mip_chain_astc(enc, img, 4, 4, levels=2)) == 2


def test_batch_argument_errors(enc):
    img = synth.make_texture(16, 16, 1)
    with pytest.raises(ab.ASTCError) as e:
        enc.encode_batch([(img, 7, 7)])
    assert e.value.status == ab.INVALID_FOOTPRINT
    with pytest.raises(ab.ASTCError) as e:
        enc.encode_batch([])
    assert e.value.status == ab.BAD_ARG
