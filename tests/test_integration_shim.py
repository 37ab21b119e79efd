"""The C++ shim of INTEGRATION.md (the reference's ASTCEncoder / store_image shape over the
C-ABI, replacing code/astc.h:724-984 and code/astc_store.cpp:18): extracted from the document,
compiled with g++ against include/astcb200.h and libastcb200.so, and driven the way
code/main.cpp:327-340 drives the reference's encoder.  Compiling and linking needs no GPU; the
run is compared, block for block and byte for byte of the .astc file, with the Python
binding."""
import os
import re
import subprocess

import numpy as np
import pytest

import _libs
import astc_implementation_b200 as ab
from astc_implementation_b200 import synth

MAIN = r"""
#include <cstdio>
#include <cstdlib>
#include <vector>
#include "shim.h"

// argv: raw RGBA8 input, width, height, block x, block y, blocks out, .astc out
int main(int argc, char** argv) {
    if (argc != 8) return 2;
    const unsigned w = (unsigned)atoi(argv[2]), h = (unsigned)atoi(argv[3]);
    const uint8_t bx = (uint8_t)atoi(argv[4]), by = (uint8_t)atoi(argv[5]);
    std::vector<uint8_t> pixels((size_t)w * h * 4);
    FILE* f = fopen(argv[1], "rb");
    if (!f || fread(pixels.data(), 1, pixels.size(), f) != pixels.size()) return 3;
    fclose(f);
    try {
        ASTCEncoder* encoder = new ASTCEncoder(0);
        encoder->init();
        encoder->secondaryInit(w, h, bx, by);
        size_t dataLen = (size_t)encoder->blocksX * encoder->blocksY * 16;
        uint8_t* dataOut = new uint8_t[dataLen];
        encoder->encode(pixels.data(), dataOut, dataLen);
        FILE* o = fopen(argv[6], "wb");
        fwrite(dataOut, 1, dataLen, o);
        fclose(o);
        store_image(bx, by, w, h, dataOut, dataLen, argv[7]);
        delete[] dataOut;
        delete encoder;
    } catch (const std::exception& e) {
        fprintf(stderr, "%s\n", e.what());
        return 1;
    }
    return 0;
}
"""


def shim_source():
    text = open(os.path.join(_libs.REPO, "INTEGRATION.md")).read()
    section = text[text.index("## C++ binding a maintainer adds"):]
    return re.search(r"```cpp\n(.*?)```", section, re.S).group(1)


@pytest.fixture(scope="module")
def shim_binary(tmp_path_factory):
    d = tmp_path_factory.mktemp("shim")
    (d / "shim.h").write_text("#pragma once\n#include <cstdint>\n" + shim_source())
    (d / "main.cpp").write_text(MAIN)
    libdir = os.path.dirname(ab.load_library()._name)
    exe = d / "encode_with_shim"
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-I", str(d), "-I", os.path.join(_libs.REPO, "include"),
           str(d / "main.cpp"), "-L", libdir, "-lastcb200", "-Wl,-rpath," + libdir, "-o", str(exe)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_shim_compiles_and_links(shim_binary):
    assert os.access(shim_binary, os.X_OK)


@pytest.mark.gpu
@pytest.mark.parametrize("bx,by", [(4, 4), (6, 6)])
def test_shim_encodes_like_the_python_binding(shim_binary, tmp_path, bx, by):
    w, h = 64, 48
    img = synth.make_texture(w, h, 77)
    raw = tmp_path / "in.rgba"
    raw.write_bytes(np.ascontiguousarray(img).tobytes())
    blocks_path, astc_path = tmp_path / "blocks.bin", tmp_path / "out.astc"
    r = subprocess.run([str(shim_binary), str(raw), str(w), str(h), str(bx), str(by), str(blocks_path), str(astc_path)],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    enc = ab.ASTCEncoder(device=0)
    enc.init()
    enc.secondaryInit(w, h, bx, by)
    ref = enc.encode(img)
    enc.close()
    assert np.array_equal(np.frombuffer(blocks_path.read_bytes(), np.uint8), ref.reshape(-1))
    ref_astc = tmp_path / "ref.astc"
    ab.store_image(bx, by, w, h, ref, str(ref_astc))
    assert astc_path.read_bytes() == ref_astc.read_bytes()
