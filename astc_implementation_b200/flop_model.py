"""Algorithmic FP32-operation model of the full search, per ASTC block.

Counts the floating-point operations the reference's WGSL passes perform per
block (one multiply or add = 1 op), from the footprint's tables:

  T   texels per block;  P  partition count
  per valid decimation mode: W weights, E texel->weight entries, S angular steps
  W_, E_ means over the valid decimation modes;  Nbm valid block modes
  sel_P selected partitionings for P partitions

  front(P)  = 40T (pass01) + 60T (pass08) + 680P (pass09) + 2 Nbm (pass12)
            + sum_dm [ (13E + 4W if W < T) + (35W + 320) + (10SW + 10S) + 200 ]   passes 02-05
            + Nbm (12 W_ + 2 E_ + 4T + 30)                                        passes 07, 11
  refine(P) = 8 [ p17 + 6 (p13 + p14 + p15 + p16 + p17) ]                         passes 13-17
            p13 = W_ + 2E_ + 45T + 60P,  p14 = 900P,  p15 = 40P,
            p16 = mean_dm(35T if W = T else E (2E/T + 38)),  p17 = 2E_ + 20T
  search(P) = 48TP + 6 sel_P P^2 + 3 (1024 * 55 / 2) + 128 * 60 T                passes 001-007

  per block = front(1) + refine(1) + sum_{P=2..4} [ search(P) + 4 (front(P) + refine(P)) ]

The split by kernel is search -> k_partition_search, front -> k_front,
refine -> k_refine.  Algorithmic bytes per block: 4 B per texel read + 16 B
written.
"""
import numpy as np


def _tables(lib, bx, by):
    import ctypes
    P = ctypes.c_void_p
    c = np.zeros(13, np.uint32)
    lib.astcb200_tables_counts(bx, by, c.ctypes.data_as(P))
    ndm, nbm = int(c[2]), int(c[1])
    bmi = np.zeros(2048, np.uint32)
    bms = np.zeros((nbm, 5), np.uint32)
    lib.astcb200_tables_block_modes(bx, by, bmi.ctypes.data_as(P), bms.ctypes.data_as(P))
    dmodes = np.zeros((ndm, 4), np.uint32)
    dinfo = np.zeros((ndm, 424), np.uint32)
    lib.astcb200_tables_decimation(bx, by, dmodes.ctypes.data_as(P), dinfo.ctypes.data_as(P))
    return c, bms, dmodes, dinfo


def _parts(lib, bx, by):
    c, bms, dmodes, dinfo = _tables(lib, bx, by)
    T = bx * by
    valid_dm = [i for i in range(len(dmodes)) if dmodes[i, 2] & 0xFF]
    Ws = np.array([int(dinfo[i, 1]) for i in valid_dm], float)
    Es = np.array([int(dinfo[i, 8:8 + T].sum()) for i in valid_dm], float)
    Ss = np.array([int(dinfo[i, 5]) for i in valid_dm], float)
    valid_set = set(valid_dm)
    nbm = sum(1 for b in bms if b[4] == 0 and int(b[1]) in valid_set)
    Wm, Em = Ws.mean(), Es.mean()
    dm_costs = [((13 * E + 4 * W) if W < T else 0.0) + (35 * W + 320) + (10 * S * W + 10 * S) + 200 for W, E, S in zip(Ws, Es, Ss)]
    p16 = float(np.mean([35 * T if W == T else E * (2 * E / T + 38) for W, E in zip(Ws, Es)]))
    return c, T, nbm, Wm, Em, dm_costs, p16


def from_work(lib, bx, by, work, mlp_blocks=0):
    """FP32 operations of each kernel for the work counters of astcb200_work_counters
    (the per-partitioned-block, per-decimation-mode, per-block-mode, per-candidate and
    per-partition-search terms of the model above, counted as the kernels ran them), and
    the tensor-core operations of the proposal network for mlp_blocks blocks."""
    c, T, nbm, Wm, Em, dm_costs, p16 = _parts(lib, bx, by)
    w = np.asarray(work, np.float64)
    front = sum(w[P - 1] * (40 * T + 60 * T + 680 * P + 2 * nbm) for P in (1, 2, 3, 4))
    front += w[4] * float(np.mean(dm_costs)) + w[5] * (12 * Wm + 2 * Em + 4 * T + 30)

    def refine_cand(P):
        p13 = Wm + 2 * Em + 45 * T + 60 * P
        p17 = 2 * Em + 20 * T
        return p17 + 6 * (p13 + 900 * P + 40 * P + p16 + p17)

    refine = sum(w[6 + P - 1] * refine_cand(P) for P in (1, 2, 3, 4))
    search = sum(w[10 + P - 2] * (48 * T * P + 6 * int(c[5 + P - 1]) * P * P + 3 * (1024 * 55 / 2) + 128 * 60 * T)
                 for P in (2, 3, 4))
    return {"search": search, "front": front, "refine": refine, "mlp": mlp_blocks * mlp_flops(lib, bx, by)}


def mlp_flops(lib, bx, by):
    """Multiply-add operations (2 per MAC) of the proposal network for one block."""
    import ctypes
    u = [ctypes.c_uint32() for _ in range(6)]
    sel = (ctypes.c_uint32 * 3)()
    lib.astcb200_proposal_layout(bx, by, *[ctypes.byref(x) for x in u], sel)
    k0p, nout = u[1].value, u[2].value
    return 2.0 * (k0p * 256 + 256 * 256 + 256 * nout)


def per_block(lib, bx, by):
    """Returns {'search':, 'front':, 'refine':, 'total':, 'bytes':} per block."""
    c, bms, dmodes, dinfo = _tables(lib, bx, by)
    T = bx * by
    valid_dm = [i for i in range(len(dmodes)) if dmodes[i, 2] & 0xFF]
    Ws = np.array([int(dinfo[i, 1]) for i in valid_dm], float)
    Es = np.array([int(dinfo[i, 8:8 + T].sum()) for i in valid_dm], float)
    Ss = np.array([int(dinfo[i, 5]) for i in valid_dm], float)
    valid_set = set(valid_dm)
    nbm = sum(1 for b in bms if b[4] == 0 and int(b[1]) in valid_set)
    Wm, Em = Ws.mean(), Es.mean()
    dm_sum = float(sum(((13 * E + 4 * W) if W < T else 0.0) + (35 * W + 320) + (10 * S * W + 10 * S) + 200
                       for W, E, S in zip(Ws, Es, Ss)))

    def front(P):
        return 40 * T + 60 * T + 680 * P + 2 * nbm + dm_sum + nbm * (12 * Wm + 2 * Em + 4 * T + 30)

    p16 = float(np.mean([35 * T if W == T else E * (2 * E / T + 38) for W, E in zip(Ws, Es)]))

    def refine(P):
        p13 = Wm + 2 * Em + 45 * T + 60 * P
        p17 = 2 * Em + 20 * T
        return 8 * (p17 + 6 * (p13 + 900 * P + 40 * P + p16 + p17))

    def search(P):
        sel = int(c[5 + P - 1])
        return 48 * T * P + 6 * sel * P * P + 3 * (1024 * 55 / 2) + 128 * 60 * T

    s = sum(search(P) for P in (2, 3, 4))
    f = front(1) + sum(4 * front(P) for P in (2, 3, 4))
    r = refine(1) + sum(4 * refine(P) for P in (2, 3, 4))
    return {"search": s, "front": f, "refine": r, "total": s + f + r, "bytes": 4 * T + 16}
