"""CPU restatement of the proposal network -- TEST INFRASTRUCTURE ONLY.

The learned proposal has no counterpart in the reference (Jure-Z/ASTC_implementation
searches every candidate); this module is the checker for the CUDA kernels that
implement it (astc_implementation_b200/csrc/mlp.cu, mlp_train.cu), written from the
mathematics of the network:

  x  = bf16(rgba8 / 255), the block's texels in raster order, channels interleaved,
       zero-padded to a multiple of 16 inputs
  h1 = relu(x W1^T + b1), h2 = relu(h1 W2^T + b2), z = h2 W3^T + b3
  inference: W1..W3, x, h1 and h2 rounded to bf16, sums in (at least) FP32
  training:  everything FP32/FP64, loss = CE(partition head) + CE(block-mode head of the
             label's partition count), gradients by backpropagation

Output classes (sel3 = the footprint's selected table entries of P = 2, 3, 4): the
partitionings of P = 2, 3, 4 one count after another (entry e of P at part_base[P-2] + e),
then the single-partition block p1 = sum(sel3), then from head_base (p1 + 1 rounded up to a
multiple of 32) one head of `nbm` block modes per partition count P = 1..4, `head_stride`
apart.

Only tests/ may import this module; the product never does.
"""
import numpy as np

HIDDEN = 256


class Classes:
    """The class plan of a footprint with selected table entries sel3 (P = 2, 3, 4)."""

    def __init__(self, sel3):
        s = [int(v) for v in sel3]
        self.part_base = (0, s[0], s[0] + s[1])
        self.p1 = s[0] + s[1] + s[2]
        self.head_base = (self.p1 + 1 + 31) & ~31

    def head_of(self, part):
        """Block-mode head (0..3 for P = 1..4) of partition classes."""
        part = np.asarray(part)
        return np.where(part == self.p1, 0, 1 + (part >= self.part_base[1]).astype(np.int64) + (part >= self.part_base[2]))


def bf16_round(x):
    """Round float32 values to the nearest bf16 (ties to even), returned as float32."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    u = x.view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return u.astype(np.uint32).view(np.float32)


def block_rgba8(img, bx, by):
    """(nblocks, bx*by, 4) uint8 texels per block, raster block order, edges clamped."""
    h, w, _ = img.shape
    nbx, nby = (w + bx - 1) // bx, (h + by - 1) // by
    ys = np.minimum(np.arange(nby * by), h - 1).reshape(nby, by)
    xs = np.minimum(np.arange(nbx * bx), w - 1).reshape(nbx, bx)
    blk = img[ys[:, None, :, None], xs[None, :, None, :]]
    return blk.reshape(nby * nbx, by * bx, 4)


def inputs(texels_u8, k0p):
    """Network inputs of blocks given as (n, T, 4) uint8."""
    n = texels_u8.shape[0]
    x = np.zeros((n, k0p), np.float32)
    v = texels_u8.reshape(n, -1).astype(np.float32) / np.float32(255.0)
    x[:, : v.shape[1]] = v
    return bf16_round(x)


def infer(x, w):
    """bf16 inference logits (float32) for inputs x (n, k0p); w holds FP32 w1 (256 x k0),
    b1, w2, b2, w3 (nout x 256), b3."""
    k0 = w["w1"].shape[1]
    w1 = np.zeros((HIDDEN, x.shape[1]), np.float32)
    w1[:, :k0] = w["w1"]
    w1 = bf16_round(w1).astype(np.float64)
    w2 = bf16_round(w["w2"]).astype(np.float64)
    w3 = bf16_round(w["w3"]).astype(np.float64)
    h1 = bf16_round(np.maximum(x.astype(np.float64) @ w1.T + w["b1"], 0.0).astype(np.float32)).astype(np.float64)
    h2 = bf16_round(np.maximum(h1 @ w2.T + w["b2"], 0.0).astype(np.float32)).astype(np.float64)
    return (h2 @ w3.T + w["b3"]).astype(np.float32)


def loss_and_grads(x, w, part_label, bm_label, nbm, head_stride, sel3):
    """FP64 forward and backward pass of the training loss (mean over the batch).
    Returns (loss_part, loss_bm, grads, dz) with grads keyed like w."""
    x = x.astype(np.float64)
    k0 = w["w1"].shape[1]
    xx = x[:, :k0]
    W = {k: np.asarray(v, np.float64) for k, v in w.items()}
    a1 = xx @ W["w1"].T + W["b1"]
    h1 = np.maximum(a1, 0.0)
    a2 = h1 @ W["w2"].T + W["b2"]
    h2 = np.maximum(a2, 0.0)
    z = h2 @ W["w3"].T + W["b3"]
    B = x.shape[0]
    dz = np.zeros_like(z)
    cl = Classes(sel3)
    zp = z[:, : cl.p1 + 1]
    mx = zp.max(axis=1, keepdims=True)
    e = np.exp(zp - mx)
    se = e.sum(axis=1, keepdims=True)
    lp = np.log(se[:, 0]) + mx[:, 0] - z[np.arange(B), part_label]
    sp = e / se
    sp[np.arange(B), part_label] -= 1.0
    dz[:, : cl.p1 + 1] = sp / B
    heads = cl.head_of(part_label)
    lb = np.zeros(B)
    for i in range(B):
        h0 = cl.head_base + heads[i] * head_stride
        zh = z[i, h0: h0 + nbm]
        m = zh.max()
        eh = np.exp(zh - m)
        s = eh.sum()
        lb[i] = np.log(s) + m - zh[bm_label[i]]
        g = eh / s
        g[bm_label[i]] -= 1.0
        dz[i, h0: h0 + nbm] = g / B
    grads = {"w3": dz.T @ h2, "b3": dz.sum(axis=0)}
    dh2 = (dz @ W["w3"]) * (a2 > 0)
    grads["w2"] = dh2.T @ h1
    grads["b2"] = dh2.sum(axis=0)
    dh1 = (dh2 @ W["w2"]) * (a1 > 0)
    grads["w1"] = dh1.T @ xx
    grads["b1"] = dh1.sum(axis=0)
    return float(lp.mean()), float(lb.mean()), grads, dz


def select(z, sel3, kmax, coverage, threshold, kbm, nbm, head_stride):
    """Selection rule of the proposal search for one block's logits z: returns
    (confident, proposed partition classes best first, block-mode sets per head)."""
    z = np.asarray(z, np.float64)
    cl = Classes(sel3)
    zp = z[: cl.p1 + 1]
    mx = zp.max()
    p = np.exp(zp - mx)
    p /= p.sum()
    order = sorted(range(cl.p1), key=lambda c: (-z[c], c))[:kmax]
    mass = p[cl.p1] + np.cumsum([p[c] for c in order]) if order else np.array([])
    confident = (p[cl.p1] + sum(p[c] for c in order)) >= threshold
    used = len(order)
    for k, m in enumerate(mass):
        if m >= coverage:
            used = k + 1
            break
    if p[cl.p1] >= coverage:
        used = 0
    modes = []
    for h in range(4):
        zh = z[cl.head_base + h * head_stride: cl.head_base + h * head_stride + nbm]
        modes.append(set(sorted(range(nbm), key=lambda c: (-zh[c], c))[: min(kbm, nbm)]))
    return bool(confident), order[:used], modes
