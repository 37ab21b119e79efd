"""Physical block packing and the .astc container against the reference's own
symbolic_to_physical / store_image outputs (tests/golden/physical_vectors.npz)."""
import os

import numpy as np

import _libs
import astc_implementation_b200 as ab


def test_oracle_symbolic_to_physical_matches_reference_vectors():
    pv = np.load(os.path.join(_libs.GOLDEN, "physical_vectors.npz"))
    lib = _libs.oracle()
    bad = 0
    for s, p, fp in zip(pv["symbolic"], pv["physical"], pv["footprint"]):
        out = np.zeros(16, np.uint8)
        assert lib.orc_symbolic_to_physical(int(fp[0]), int(fp[1]), _libs.ptr(np.ascontiguousarray(s)), _libs.ptr(out)) == 0
        bad += not np.array_equal(out, p)
    assert bad == 0 and len(pv["physical"]) == 360


def test_reference_build_reproduces_vectors():
    ref = _libs.ref_lib()
    if ref is None:
        import pytest
        pytest.skip("oracle/_ref not built")
    pv = np.load(os.path.join(_libs.GOLDEN, "physical_vectors.npz"))
    for s, p, fp in list(zip(pv["symbolic"], pv["physical"], pv["footprint"]))[:50]:
        out = np.zeros(16, np.uint8)
        ref.astcref_symbolic_to_physical(int(fp[0]), int(fp[1]), _libs.ptr(np.ascontiguousarray(s)), _libs.ptr(out))
        assert np.array_equal(out, p)


def test_store_image_matches_reference_file(tmp_path):
    pv = np.load(os.path.join(_libs.GOLDEN, "physical_vectors.npz"))
    data = np.arange(4 * 16, dtype=np.uint8)
    path = tmp_path / "x.astc"
    ab.store_image(6, 6, 23, 17, data, str(path))
    assert np.array_equal(np.frombuffer(path.read_bytes(), np.uint8), pv["store_image_6x6_23x17"])


def test_decoder_inverts_oracle_blocks():
    """Decoding the oracle's blocks of a small texture reproduces it closely, and
    every block decodes (no error colour)."""
    from astc_implementation_b200 import synth
    img = synth.make_texture(48, 40, 7)
    for bx, by in [(4, 4), (6, 6), (5, 4)]:
        n = ((48 + bx - 1) // bx) * ((40 + by - 1) // by)
        out = np.zeros(n * 16, np.uint8)
        assert _libs.oracle().orc_encode(_libs.ptr(img), 48, 40, bx, by, 0, _libs.ptr(out), None) == 0
        dec = ab.decode(bx, by, 48, 40, out)
        magenta = np.all(dec == np.array([255, 0, 255, 255], np.uint8), axis=2)
        assert not magenta.any()
        assert ab.psnr(dec, img) > 18.0
