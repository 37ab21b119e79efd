"""ctypes loaders shared by the tests: the CPU oracle, the reference's own
compiled CPU code (oracle/_ref) and table-digest helpers."""
import ctypes
import hashlib
import os

import numpy as np

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(REPO, "tests", "golden")
P = ctypes.c_void_p
FOOTPRINTS = [(4, 4), (5, 4), (5, 5), (6, 5), (6, 6), (8, 5), (8, 6), (10, 5),
              (10, 6), (8, 8), (10, 8), (10, 10), (12, 10), (12, 12)]


def ptr(a):
    return a.ctypes.data_as(P)


_oracle = None


def oracle():
    global _oracle
    if _oracle is None:
        path = os.path.join(REPO, "oracle", "liboracle.so")
        if not os.path.exists(path):
            import subprocess
            subprocess.check_call([os.path.join(REPO, "oracle", "build_oracle.sh")])
        _oracle = ctypes.CDLL(path)
    return _oracle


def ref_lib():
    path = os.path.join(REPO, "oracle", "_ref", "libastcref.so")
    return ctypes.CDLL(path) if os.path.exists(path) else None


def golden_tables():
    return np.load(os.path.join(GOLDEN, "reference_tables.npz"))


def footprint_digests(lib, prefix, bx, by):
    """sha256 of every host table, in the layout of oracle/ref_shim.cpp."""
    f = lambda name: getattr(lib, prefix + name)
    c = np.zeros(13, np.uint32)
    f("counts")(bx, by, ptr(c))
    nbm, ndm, n_t2w, n_w2t = int(c[1]), int(c[2]), int(c[3]), int(c[4])
    bmi = np.zeros(2048, np.uint32)
    bms = np.zeros((max(nbm, 1), 5), np.uint32)
    f("block_modes")(bx, by, ptr(bmi), ptr(bms))
    dmodes = np.zeros((ndm, 4), np.uint32)
    dinfo = np.zeros((ndm, 424), np.uint32)
    f("decimation")(bx, by, ptr(dmodes), ptr(dinfo))
    dinfo[dmodes[:, 0] == 0xFFFFFFFF, 4:7] = 0
    t2wi = np.zeros(n_t2w, np.uint32); t2wc = np.zeros(n_t2w, np.float32)
    w2ti = np.zeros(n_w2t, np.uint32); w2tc = np.zeros(n_w2t, np.float32)
    f("maps")(bx, by, ptr(t2wi), ptr(t2wc), ptr(w2ti), ptr(w2tc))
    pinfo = np.zeros((3073, 150), np.uint32)
    cov2 = np.zeros((1024, 2), np.uint64); cov3 = np.zeros((1024, 3), np.uint64); cov4 = np.zeros((1024, 4), np.uint64)
    km = np.zeros(64, np.uint32); pidx = np.zeros((3, 1024), np.uint16)
    f("partitions")(bx, by, ptr(pinfo), ptr(cov2), ptr(cov3), ptr(cov4), ptr(km), ptr(pidx))
    parts = dict(counts=c, bm_index=bmi, block_modes=bms[:nbm], dmodes=dmodes, dinfo=dinfo,
                 t2w_idx=t2wi, t2w_c=t2wc, w2t_idx=w2ti, w2t_c=w2tc, pinfo=pinfo,
                 cov2=cov2, cov3=cov3, cov4=cov4, kmeans=km, packed_index=pidx)
    return {"%dx%d:%s" % (bx, by, k): hashlib.sha256(np.ascontiguousarray(v).tobytes()).hexdigest()
            for k, v in parts.items()}
