"""CUDA encoder vs the CPU oracle (bit-exact), through the C-ABI."""
import ctypes

import numpy as np
import pytest

import _libs
import astc_implementation_b200 as ab
from astc_implementation_b200 import synth

pytestmark = pytest.mark.gpu


def oracle_encode(img, bx, by):
    h, w = img.shape[:2]
    n = ((w + bx - 1) // bx) * ((h + by - 1) // by)
    out = np.zeros((n, 16), np.uint8)
    sym = np.zeros((n, 108), np.uint32)
    assert _libs.oracle().orc_encode(_libs.ptr(np.ascontiguousarray(img)), w, h, bx, by, 0, _libs.ptr(out), _libs.ptr(sym)) == 0
    return out, sym


@pytest.fixture(scope="module")
def enc():
    e = ab.ASTCEncoder(device=0)
    e.init()
    yield e
    e.close()


def gpu_encode(enc, img, bx, by):
    h, w = img.shape[:2]
    enc.secondaryInit(w, h, bx, by)
    sym = enc.encode_symbolic(img)
    out = enc.encode(img).reshape(-1, 16)
    return out, sym


def test_config1_256_seed0_4x4_bit_exact(enc):
    img = synth.make_texture(256, 256, 0)
    out, sym = gpu_encode(enc, img, 4, 4)
    ref_out, ref_sym = oracle_encode(img, 4, 4)
    assert np.array_equal(sym, ref_sym)
    assert np.array_equal(out, ref_out)
    psnr = ab.psnr(ab.decode(4, 4, 256, 256, out), img)
    assert psnr == ab.psnr(ab.decode(4, 4, 256, 256, ref_out), img) and psnr > 40.0


@pytest.mark.parametrize("bx,by", _libs.FOOTPRINTS)
def test_every_footprint_bit_exact(enc, bx, by):
    w, h = 5 * bx + 3, 3 * by + 1  # ragged edges
    img = synth.make_texture(w, h, 100 + bx * 16 + by)
    out, sym = gpu_encode(enc, img, bx, by)
    ref_out, ref_sym = oracle_encode(img, bx, by)
    assert np.array_equal(sym, ref_sym)
    assert np.array_equal(out, ref_out)


def test_6x6_medium_bit_exact(enc):
    img = synth.make_texture(192, 132, 9)
    out, sym = gpu_encode(enc, img, 6, 6)
    ref_out, ref_sym = oracle_encode(img, 6, 6)
    assert np.array_equal(sym, ref_sym)


@pytest.mark.parametrize("w,h", [(1, 1), (3, 5), (17, 13)])
def test_tiny_images(enc, w, h):
    img = synth.make_texture(24, 24, 4)[:h, :w].copy()
    for bx, by in [(4, 4), (6, 6), (12, 12)]:
        out, sym = gpu_encode(enc, img, bx, by)
        ref_out, ref_sym = oracle_encode(img, bx, by)
        assert np.array_equal(sym, ref_sym)


@pytest.mark.parametrize("kind", ["black", "white", "gray", "opaque_gray", "alpha_only"])
def test_degenerate_blocks(enc, kind):
    rng = np.random.default_rng(1)
    img = np.zeros((20, 20, 4), np.uint8)
    if kind == "white":
        img[:] = 255
    elif kind == "gray":
        v = rng.integers(0, 256, (20, 20), dtype=np.uint8)
        img[..., 0] = img[..., 1] = img[..., 2] = v
        img[..., 3] = rng.integers(0, 256, (20, 20), dtype=np.uint8)
    elif kind == "opaque_gray":
        v = rng.integers(0, 256, (20, 20), dtype=np.uint8)
        img[..., 0] = img[..., 1] = img[..., 2] = v
        img[..., 3] = 255
    elif kind == "alpha_only":
        img[..., 3] = rng.integers(0, 256, (20, 20), dtype=np.uint8)
    out, sym = gpu_encode(enc, img, 4, 4)
    ref_out, ref_sym = oracle_encode(img, 4, 4)
    assert np.array_equal(sym, ref_sym) and np.array_equal(out, ref_out)


@pytest.mark.parametrize("bx,by", [(4, 4), (6, 6), (8, 5)])
@pytest.mark.parametrize("kind", ["noise", "opposed_gradients"])
def test_endpoint_search_hard_blocks_bit_exact(enc, kind, bx, by):
    """Blocks whose fitted endpoints come out inverted or far apart make the endpoint
    packer's nudge loop run for hundreds of steps (found by bisection on the GPU)."""
    rng = np.random.default_rng(7)
    h, w = 48, 60
    if kind == "noise":
        img = rng.integers(0, 256, (h, w, 4), dtype=np.uint8)
    else:
        x = np.linspace(0, 1, w, dtype=np.float32)[None, :].repeat(h, 0)
        y = np.linspace(0, 1, h, dtype=np.float32)[:, None].repeat(w, 1)
        img = np.stack([255 * x, 255 * (1 - x), 255 * y, 255 * (1 - y * x)], axis=2)
        img = (img + rng.normal(0, 12, img.shape)).clip(0, 255).astype(np.uint8)
    out, sym = gpu_encode(enc, img, bx, by)
    ref_out, ref_sym = oracle_encode(img, bx, by)
    assert np.array_equal(sym, ref_sym) and np.array_equal(out, ref_out)


def test_full_size_2048_properties():
    """BASELINE config 2 sizes: deterministic, chunking-invariant, decodes well, and a
    sampled set of blocks matches the oracle exactly."""
    img = synth.make_texture(2048, 2048, 1)
    tex4 = synth.texel_blocks(img, 4, 4)
    for bx, by in [(4, 4), (6, 6)]:
        e1 = ab.ASTCEncoder(0)
        e1.secondaryInit(2048, 2048, bx, by)
        a = e1.encode(img).reshape(-1, 16).copy()
        b = e1.encode(img).reshape(-1, 16)
        assert np.array_equal(a, b)
        e2 = ab.ASTCEncoder(0, chunk_blocks=12345)
        e2.secondaryInit(2048, 2048, bx, by)
        assert np.array_equal(a, e2.encode(img).reshape(-1, 16))
        psnr = ab.psnr(ab.decode(bx, by, 2048, 2048, a), img)
        assert psnr > (38.0 if bx == 4 else 30.0)
        tex = tex4 if bx == 4 else synth.texel_blocks(img, 6, 6)
        idx = np.random.default_rng(0).choice(tex.shape[0], 256, replace=False)
        sub = np.ascontiguousarray(tex[idx])
        ref = np.zeros((256, 16), np.uint8)
        assert _libs.oracle().orc_encode_blocks(_libs.ptr(sub), 256, bx, by, 0, None, _libs.ptr(ref)) == 0
        assert np.array_equal(a[idx], ref)
        e1.close(); e2.close()


def test_device_entry_matches_host_entry(enc):
    import torch
    img = synth.make_texture(64, 64, 3)
    enc.secondaryInit(64, 64, 4, 4)
    host = enc.encode(img)
    d_in = torch.from_numpy(img.reshape(-1)).cuda()
    d_out = torch.zeros(host.size, dtype=torch.uint8, device="cuda")
    enc.encode_device(d_in.data_ptr(), d_out.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert np.array_equal(d_out.cpu().numpy(), host)


def test_api_errors(enc):
    with pytest.raises(ab.ASTCError) as e:
        enc.secondaryInit(64, 64, 3, 3)
    assert e.value.status == ab.INVALID_FOOTPRINT
    fresh = ab.ASTCEncoder(0)
    lib = ab.load_library()
    img = np.zeros(64 * 64 * 4, np.uint8)
    out = np.zeros(256 * 16, np.uint8)
    assert lib.astcb200_encode(fresh._ctx, _libs.ptr(img), _libs.ptr(out), out.size, None) == ab.NO_IMAGE
    fresh.secondaryInit(64, 64, 4, 4)
    assert lib.astcb200_encode(fresh._ctx, _libs.ptr(img), _libs.ptr(out), 100, None) == ab.BAD_ARG
    fresh.close()


def test_bounded_wait_configuration():
    e = ab.ASTCEncoder(0, timeout_ms=60000)
    img = synth.make_texture(32, 32, 2)
    e.secondaryInit(32, 32, 4, 4)
    ref = oracle_encode(img, 4, 4)[0]
    assert np.array_equal(e.encode(img).reshape(-1, 16), ref)
    e.close()


def test_store_image_roundtrip_through_api(enc, tmp_path):
    img = synth.make_texture(40, 24, 8)
    enc.secondaryInit(40, 24, 8, 6)
    blocks = enc.encode(img)
    path = tmp_path / "t.astc"
    ab.store_image(8, 6, 40, 24, blocks, str(path))
    raw = np.frombuffer(path.read_bytes(), np.uint8)
    assert raw[:4].tolist() == [0x13, 0xAB, 0xA1, 0x5C] and raw[4] == 8 and raw[5] == 6
    assert np.array_equal(raw[16:], blocks)
