"""C-ABI surface that needs no GPU: symbols, status strings, argument checks."""
import ctypes
import os
import re

import numpy as np
import pytest

import _libs
import astc_implementation_b200 as ab

HEADER = os.path.join(_libs.REPO, "include", "astcb200.h")


def declared_functions():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"\b(astcb200_\w+)\s*\(", src)))


def test_library_exports_every_declared_function():
    lib = ab.load_library()
    names = declared_functions()
    assert len(names) >= 14
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_status_strings():
    lib = ab.load_library()
    for code in range(9):
        assert lib.astcb200_status_string(code)
    assert b"2048" in lib.astcb200_status_string(ab.TOO_LARGE)


def test_decode_rejects_bad_arguments():
    lib = ab.load_library()
    buf = np.zeros(16, np.uint8)
    out = np.zeros(64, np.uint8)
    assert lib.astcb200_decode(3, 3, 4, 4, buf.ctypes.data_as(ctypes.c_void_p), 16, out.ctypes.data_as(ctypes.c_void_p)) == ab.BAD_ARG
    assert lib.astcb200_decode(4, 4, 8, 8, buf.ctypes.data_as(ctypes.c_void_p), 16, out.ctypes.data_as(ctypes.c_void_p)) == ab.BAD_ARG


def test_store_image_io_error(tmp_path):
    with pytest.raises(ab.ASTCError) as e:
        ab.store_image(4, 4, 4, 4, np.zeros(16, np.uint8), str(tmp_path / "missing" / "x.astc"))
    assert e.value.status == ab.IO_ERROR


def test_noalloc_rejects_before_touching_the_device():
    lib = ab.load_library()
    # footprint and size checks come before any CUDA call
    assert lib.astcb200_encode_noalloc(0, ctypes.c_void_p(16), 64, 64, 3, 3, ctypes.c_void_p(16), None) == ab.INVALID_FOOTPRINT
    assert lib.astcb200_encode_noalloc(0, ctypes.c_void_p(16), 4096, 4096, 4, 4, ctypes.c_void_p(16), None) == ab.TOO_LARGE
    assert lib.astcb200_encode_noalloc(0, None, 64, 64, 4, 4, ctypes.c_void_p(16), None) == ab.BAD_ARG


def test_flop_model_per_block_totals():
    """The op-count model's totals per block: 4.29 MFLOP at 4x4, 9.61 MFLOP at 6x6."""
    from astc_implementation_b200 import flop_model
    lib = ab.load_library()
    assert abs(flop_model.per_block(lib, 4, 4)["total"] / 1e6 - 4.29) < 0.01
    assert abs(flop_model.per_block(lib, 6, 6)["total"] / 1e6 - 9.61) < 0.01


def test_work_counter_model_reproduces_the_per_block_model():
    """The op-count model applied to full-search work counters equals the per-block model."""
    from astc_implementation_b200 import flop_model
    lib = ab.load_library()
    for bx, by, ndm, nbm in [(4, 4, 6, 53), (6, 6, 22, 198)]:
        w = np.zeros(16)
        w[0], w[1:4] = 1, 4                # partitioned blocks by P
        w[4], w[5] = ndm * 13, nbm * 13    # decimation and block modes evaluated
        w[6], w[7:10] = 8, 32              # candidates refined by P
        w[10:13] = 1                       # partition searches
        f = flop_model.from_work(lib, bx, by, w)
        pb = flop_model.per_block(lib, bx, by)
        for k in ("search", "front", "refine"):
            assert abs(f[k] - pb[k]) <= 1e-9 * pb[k], (bx, k)


def test_astc_containers_argument_errors():
    """astcb200_astc_containers_device checks every image before queuing any copy."""
    lib = ab.load_library()
    img = lambda d, h, n, w, hh, bx, by: (ab.AstcImage * 1)(ab.AstcImage(d, h, n, w, hh, bx, by))
    assert lib.astcb200_astc_containers_device(img(16, 16, 100, 8, 8, 7, 7), 1, None) == ab.INVALID_FOOTPRINT
    assert lib.astcb200_astc_containers_device(img(16, 16, 16 + 4 * 16 - 1, 8, 8, 4, 4), 1, None) == ab.BAD_ARG
    assert lib.astcb200_astc_containers_device(img(0, 16, 100, 8, 8, 4, 4), 1, None) == ab.BAD_ARG
    assert lib.astcb200_astc_containers_device(img(16, 0, 100, 8, 8, 4, 4), 1, None) == ab.BAD_ARG
    assert lib.astcb200_astc_containers_device(img(16, 16, 100, 0, 8, 4, 4), 1, None) == ab.BAD_ARG
    assert lib.astcb200_astc_containers_device(None, 1, None) == ab.BAD_ARG
    assert lib.astcb200_astc_containers_device(None, 0, None) == ab.OK
