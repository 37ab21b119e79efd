"""Generates the golden fixtures under tests/golden/ from the reference.

Run after `oracle/build_ref.sh <reference_root>` has built oracle/_ref/libastcref.so,
giving the same reference checkout (the directory holding code/ and shaders/):

    python tests/golden/gen_reference_fixtures.py <reference_root>

Outputs (committed; the tests never read the reference itself):
  reference_tables.npz
    * constant tables transcribed from the reference's WGSL source text:
        quant_to_unquant        shaders/pass07_weights_and_error_for_bm.wgsl:12-37
        quant_mode_table        shaders/pass11_best_color_combination_for_mode_1part.wgsl:12-64
        color_unquant_to_uquant shaders/pass14_pack_color_endpoints.wgsl:29-319
        prev_next_values        shaders/pass16_realign_weights.wgsl:13-74
        baseline_quant_error    shaders/pass09_compute_color_error.wgsl:10-28 (f32 const-eval)
    * tables transcribed from code/physical_compression.cpp:
        integer_of_trits (:44), integer_of_quints (:207), weight_scramble (:249),
        color_scramble (:284)
    * per footprint, sha256 digests of every table the reference builds on the host
      (block modes, decimation info, texel<->weight maps, partition tables, coverage
      bitmaps, k-means texels) and of the sin/cos angular tables.
  physical_vectors.npz
    * symbolic -> physical block vectors produced by the reference's own
      symbolic_to_physical (code/physical_compression.cpp:843) on seeded random but
      encodable SymbolicBlocks, and an .astc header produced by store_image.
"""
import ctypes
import hashlib
import os
import re
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
FOOTPRINTS = [(4, 4), (5, 4), (5, 5), (6, 5), (6, 6), (8, 5), (8, 6), (10, 5),
              (10, 6), (8, 8), (10, 8), (10, 10), (12, 10), (12, 12)]


def _numbers(text):
    text = re.sub(r"//[^\n]*", "", text)
    return [int(t, 0) for t in re.findall(r"0x[0-9a-fA-F]+|-?\d+", text)]


def wgsl_array(path, name):
    src = open(path).read()
    m = re.search(r"const\s+%s\s*=\s*array<[^>]*>\s*\((.*?)\);" % name, src, re.S)
    if not m:
        raise RuntimeError("table %s not found in %s" % (name, path))
    return _numbers(m.group(1))


def cpp_block(path, start_pat):
    src = open(path).read()
    i = src.index(start_pat)
    j = src.index("{", i)
    depth, k = 0, j
    while True:
        if src[k] == "{":
            depth += 1
        elif src[k] == "}":
            depth -= 1
            if depth == 0:
                break
        k += 1
    return src[j:k + 1]


def baseline_quant_error(path):
    src = open(path).read()
    m = re.search(r"const\s+BASELINE_QUANT_ERROR\s*=\s*array<f32,\s*17>\s*\((.*?)\);", src, re.S)
    divs = [int(a) * int(b) for a, b in re.findall(r"/\s*\((\d+)\s*\*\s*(\d+)\)", m.group(1))]
    f = np.float32
    base = f(f(65536.0) * f(65536.0)) / f(18.0)
    return np.array([f(base) / f(d) for d in divs], dtype=np.float32)


def transfer_scramble(path):
    body = cpp_block(path, "static transfer_table transfet_tables")
    rows = re.findall(r"\{\{([^}]*)\}\}", body)
    out = np.zeros((12, 32), np.uint8)
    for q, r in enumerate(rows):
        vals = _numbers(r)
        out[q, :len(vals)] = vals
    return out


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: gen_reference_fixtures.py <reference_root>")
    ref = sys.argv[1]
    sh = os.path.join(ref, "shaders")
    code = os.path.join(ref, "code")
    lib = ctypes.CDLL(os.path.join(REPO, "oracle", "_ref", "libastcref.so"))
    P = ctypes.c_void_p

    fx = {}
    fx["quant_to_unquant"] = np.array(wgsl_array(os.path.join(sh, "pass07_weights_and_error_for_bm.wgsl"), "QUANT_TO_UNQUANT"), np.int32)
    fx["quant_mode_table"] = np.array(wgsl_array(os.path.join(sh, "pass11_best_color_combination_for_mode_1part.wgsl"), "QUANT_MODE_TABLE"), np.int32).reshape(10, 128)
    for k in (2, 3, 4):
        other = np.array(wgsl_array(os.path.join(sh, "pass11_best_color_combination_for_mode_%dpart.wgsl" % k), "QUANT_MODE_TABLE"), np.int32).reshape(10, 128)
        assert (other == fx["quant_mode_table"]).all()
    fx["color_unquant_to_uquant"] = np.array(wgsl_array(os.path.join(sh, "pass14_pack_color_endpoints.wgsl"), "COLOR_UNQUANT_TO_QUANT_TABLE"), np.int32).reshape(17, 512)
    fx["prev_next_values"] = np.array(wgsl_array(os.path.join(sh, "pass16_realign_weights.wgsl"), "ALL_PREV_NEXT_VALUES"), np.int32).reshape(12, 65)
    fx["baseline_quant_error"] = baseline_quant_error(os.path.join(sh, "pass09_compute_color_error.wgsl"))
    pc = os.path.join(code, "physical_compression.cpp")
    fx["integer_of_trits"] = np.array(_numbers(cpp_block(pc, "static const uint8_t integer_of_trits")), np.uint8).reshape(3, 3, 3, 3, 3)
    fx["integer_of_quints"] = np.array(_numbers(cpp_block(pc, "static const uint8_t integer_of_quints")), np.uint8).reshape(5, 5, 5)
    fx["weight_scramble"] = transfer_scramble(pc)
    fx["color_scramble"] = np.array(_numbers(cpp_block(pc, "const uint8_t color_uquant_to_scrambled_pquant_tables")), np.uint8).reshape(17, 256)

    # per-footprint digests of the host-built tables
    digests = []
    names = []
    for (bx, by) in FOOTPRINTS:
        c = np.zeros(13, np.uint32)
        lib.astcref_counts(bx, by, c.ctypes.data_as(P))
        nbm, ndm, n_t2w, n_w2t = int(c[1]), int(c[2]), int(c[3]), int(c[4])
        bmi = np.zeros(2048, np.uint32)
        bms = np.zeros((max(nbm, 1), 5), np.uint32)
        lib.astcref_block_modes(bx, by, bmi.ctypes.data_as(P), bms.ctypes.data_as(P))
        dmodes = np.zeros((ndm, 4), np.uint32)
        dinfo = np.zeros((ndm, 424), np.uint32)
        lib.astcref_decimation(bx, by, dmodes.ctypes.data_as(P), dinfo.ctypes.data_as(P))
        # decimation modes that no single-plane block mode can use have
        # maxprec_1plane == -1, and the reference then reads steps_for_quant_level[-1]
        # (metadata_structures.cpp:328-335, undefined); those three fields are masked to 0.
        dinfo[dmodes[:, 0] == 0xFFFFFFFF, 4:7] = 0
        t2wi = np.zeros(n_t2w, np.uint32); t2wc = np.zeros(n_t2w, np.float32)
        w2ti = np.zeros(n_w2t, np.uint32); w2tc = np.zeros(n_w2t, np.float32)
        lib.astcref_maps(bx, by, t2wi.ctypes.data_as(P), t2wc.ctypes.data_as(P), w2ti.ctypes.data_as(P), w2tc.ctypes.data_as(P))
        pinfo = np.zeros((3073, 150), np.uint32)
        cov2 = np.zeros((1024, 2), np.uint64); cov3 = np.zeros((1024, 3), np.uint64); cov4 = np.zeros((1024, 4), np.uint64)
        km = np.zeros(64, np.uint32); pidx = np.zeros((3, 1024), np.uint16)
        lib.astcref_partitions(bx, by, pinfo.ctypes.data_as(P), cov2.ctypes.data_as(P), cov3.ctypes.data_as(P),
                               cov4.ctypes.data_as(P), km.ctypes.data_as(P), pidx.ctypes.data_as(P))
        parts = dict(counts=c, bm_index=bmi, block_modes=bms[:nbm], dmodes=dmodes, dinfo=dinfo,
                     t2w_idx=t2wi, t2w_c=t2wc, w2t_idx=w2ti, w2t_c=w2tc, pinfo=pinfo,
                     cov2=cov2, cov3=cov3, cov4=cov4, kmeans=km, packed_index=pidx)
        for k, v in parts.items():
            names.append("%dx%d:%s" % (bx, by, k))
            digests.append(hashlib.sha256(np.ascontiguousarray(v).tobytes()).hexdigest())
    s = np.zeros(16384, np.float32); co = np.zeros(16384, np.float32)
    lib.astcref_angular(s.ctypes.data_as(P), co.ctypes.data_as(P))
    names += ["angular:sin", "angular:cos"]
    digests += [hashlib.sha256(s.tobytes()).hexdigest(), hashlib.sha256(co.tobytes()).hexdigest()]
    fx["digest_names"] = np.array(names)
    fx["digests"] = np.array(digests)
    np.savez_compressed(os.path.join(HERE, "reference_tables.npz"), **fx)

    # symbolic -> physical vectors
    lib.astcref_ise_bitcount.restype = ctypes.c_uint
    rng = np.random.default_rng(20251203)
    qmt = fx["quant_mode_table"]
    syms, outs, fps = [], [], []
    ldr_formats = [0, 1, 4, 5, 6, 8, 9, 10, 12, 13]
    for (bx, by) in [(4, 4), (6, 6), (8, 8), (5, 4), (12, 12), (10, 6)]:
        c = np.zeros(13, np.uint32)
        lib.astcref_counts(bx, by, c.ctypes.data_as(P))
        nbm = int(c[1])
        bmi = np.zeros(2048, np.uint32); bms = np.zeros((nbm, 5), np.uint32)
        lib.astcref_block_modes(bx, by, bmi.ctypes.data_as(P), bms.ctypes.data_as(P))
        ndm = int(c[2])
        dmodes = np.zeros((ndm, 4), np.uint32); dinfo = np.zeros((ndm, 424), np.uint32)
        lib.astcref_decimation(bx, by, dmodes.ctypes.data_as(P), dinfo.ctypes.data_as(P))
        single = [i for i in range(nbm) if bms[i, 4] == 0]
        made = 0
        while made < 60:
            b = single[rng.integers(len(single))]
            mode_index, dm, wq, wbits, _ = bms[b]
            pc_ = int(rng.integers(1, 5))
            free = [111, 97, 94, 91][pc_ - 1] - int(wbits)
            if free <= 0:
                continue
            fmts = [ldr_formats[rng.integers(len(ldr_formats))] for _ in range(pc_)]
            if pc_ > 1 and rng.random() < 0.5:
                fmts = [fmts[0]] * pc_
            # formats of one block may differ by at most one class
            cls = [f >> 2 for f in fmts]
            if max(cls) - min(cls) > 1:
                continue
            matched = int(len(set(fmts)) == 1)
            nvals = sum(2 * (f >> 2) + 2 for f in fmts)
            bits = free if (pc_ == 1 or matched) else free - (3 * pc_ - 4)
            if nvals // 2 >= 10 or bits <= 0:
                continue
            q = int(qmt[nvals // 2, bits])
            if q < 4:
                continue
            sym = np.zeros(108, np.uint32)
            sym.view(np.float32)[0] = 1.0
            sym[1] = mode_index
            sym[2] = pc_
            sym[3] = int(rng.integers(0, 1024)) if pc_ > 1 else 0
            sym[4] = matched
            sym[5] = q
            sym[8:8 + pc_] = fmts
            sym[12:44] = rng.integers(0, 256, 32)
            w = int(dinfo[dm, 1])
            sym[44:44 + w] = rng.integers(0, 65, w)
            out = np.zeros(16, np.uint8)
            lib.astcref_symbolic_to_physical(bx, by, sym.ctypes.data_as(P), out.ctypes.data_as(P))
            syms.append(sym); outs.append(out); fps.append((bx, by))
            made += 1
    tmp = tempfile.NamedTemporaryFile(suffix=".astc", delete=False)
    tmp.close()
    data = np.arange(4 * 16, dtype=np.uint8)
    lib.astcref_store_image(6, 6, 23, 17, data.ctypes.data_as(P), ctypes.c_size_t(data.size), tmp.name.encode())
    astc_file = np.frombuffer(open(tmp.name, "rb").read(), np.uint8)
    os.unlink(tmp.name)
    np.savez_compressed(os.path.join(HERE, "physical_vectors.npz"), symbolic=np.array(syms),
                        physical=np.array(outs), footprint=np.array(fps, np.int32),
                        store_image_6x6_23x17=astc_file)
    print("wrote", len(names), "digests and", len(syms), "physical vectors")


if __name__ == "__main__":
    main()
