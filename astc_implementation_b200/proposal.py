"""Learned proposal search: the network's class layout, training labels taken from the
full search, training on the GPU with the library's own kernels (astcb200_train_*),
and trained weights for an encoder.

    from astc_implementation_b200 import proposal
    net = proposal.load_weights(4, 4)                 # shipped network (weights/)
    enc.set_proposal_net(net); enc.set_pruning(True, max_partitionings=4, ...)

Training (needs a GPU):

    python -m astc_implementation_b200.proposal --footprint 4x4 --out weights/proposal_4x4.npz

labels 2M blocks of synthetic textures (generator seeds 100-199) with the full search
(FIXED semantics by default: the reference's search with its shader bugs repaired) and trains
the network on them (inputs: texels / 255 in bf16; classes: the winning
partitioning or the single-partition class, and the winning block mode of that
partition count).  PyTorch only holds the device memory and the stream.
"""
import argparse
import ctypes
import os
import time

import numpy as np

from . import ASTCEncoder, _check, load_library

HIDDEN = 256
WEIGHTS_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "weights")


class Layout:
    def __init__(self, bx, by):
        lib = load_library()
        u = [ctypes.c_uint32() for _ in range(6)]
        sel = (ctypes.c_uint32 * 3)()
        _check(lib.astcb200_proposal_layout(bx, by, *[ctypes.byref(x) for x in u], sel))
        self.bx, self.by = bx, by
        self.inputs, self.inputs_padded, self.outputs, self.nbm, self.head_base, self.head_stride = (x.value for x in u)
        self.sel3 = tuple(int(v) for v in sel)
        # classes: the selected partitionings of P = 2, 3, 4 one count after another, then the
        # single-partition class p1, then the block-mode heads from head_base
        self.part_base = (0, self.sel3[0], self.sel3[0] + self.sel3[1])
        self.p1 = sum(self.sel3)

    def part_class(self, P, entry):
        """Class of table entry `entry` of partition count P = 2..4."""
        return np.asarray(self.part_base)[np.asarray(P) - 2] + entry

    def pick_of(self, c):
        """(P - 2) << 10 | entry of partition class c < p1 (the encoder's name of a partitioning)."""
        c = np.asarray(c)
        q = (c >= self.part_base[1]).astype(np.int64) + (c >= self.part_base[2])
        return (q << 10) | (c - np.asarray(self.part_base)[q])

    def head_of(self, part):
        """Block-mode head (0..3 for P = 1..4) of partition classes."""
        part = np.asarray(part)
        return np.where(part == self.p1, 0, 1 + (part >= self.part_base[1]).astype(np.int64) + (part >= self.part_base[2]))


def bf16_round(x):
    x = np.ascontiguousarray(x, dtype=np.float32)
    u = x.view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return u.astype(np.uint32).view(np.float32)


def block_rgba8(img, bx, by):
    """(nblocks, bx*by, 4) uint8: raster block order, texels in raster order, edges clamped."""
    h, w, _ = img.shape
    nbx, nby = (w + bx - 1) // bx, (h + by - 1) // by
    ys = np.minimum(np.arange(nby * by), h - 1).reshape(nby, by)
    xs = np.minimum(np.arange(nbx * bx), w - 1).reshape(nbx, bx)
    return img[ys[:, None, :, None], xs[None, :, None, :]].reshape(nby * nbx, by * bx, 4)


def network_inputs(texels_u8, k0p):
    n = texels_u8.shape[0]
    x = np.zeros((n, k0p), np.float32)
    x[:, : texels_u8.shape[1] * 4] = texels_u8.reshape(n, -1).astype(np.float32) / np.float32(255.0)
    return bf16_round(x)


def _trial_modes(bx, by):
    lib = load_library()
    f = lib.astcb200_tables_trial_modes
    f.restype = ctypes.c_int
    n = ctypes.c_uint32()
    f(bx, by, ctypes.byref(n), None)
    modes = np.zeros(n.value, np.uint16)
    f(bx, by, ctypes.byref(n), modes.ctypes.data_as(ctypes.c_void_p))
    return modes


def _seed_to_entry(bx, by):
    lib = load_library()
    f = lib.astcb200_tables_partitions
    f.restype = ctypes.c_int
    pinfo = np.zeros(3073 * 150, np.uint32)
    cov = [np.zeros(1024 * p, np.uint64) for p in (2, 3, 4)]
    km = np.zeros(64, np.uint32)
    pidx = np.zeros((3, 1024), np.uint16)
    p = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    f(bx, by, p(pinfo), p(cov[0]), p(cov[1]), p(cov[2]), p(km), p(pidx))
    return pidx


def labels_from_symbolic(sym, bx, by):
    """(partition class, block-mode class, usable) per block from SymbolicBlock records
    (108 u32: [1] block mode, [2] partition count, [3] partition seed)."""
    lay = Layout(bx, by)
    modes = _trial_modes(bx, by)
    trial_of_mode = np.full(2048, -1, np.int64)
    trial_of_mode[modes.astype(np.int64)] = np.arange(len(modes))
    pidx = _seed_to_entry(bx, by).astype(np.int64)
    pc = sym[:, 2].astype(np.int64)
    seed = sym[:, 3].astype(np.int64) & 1023
    q = np.clip(pc, 2, 4) - 2
    part = np.where(pc <= 1, lay.p1, np.asarray(lay.part_base)[q] + pidx[q, seed])
    bm = trial_of_mode[sym[:, 1].astype(np.int64) & 2047]
    usable = (sym[:, 0].view(np.float32) < 1e29) & (bm >= 0) & (pc >= 1) & (pc <= 4)
    return part.astype(np.int32), np.maximum(bm, 0).astype(np.int32), usable


def mip_down(img):
    """Next mip level: max(1, w/2) x max(1, h/2), each texel the rounded mean (sum + 2) / 4 of
    the 2x2 source texels, source coordinates clamped (astcb200_downsample_device's rule)."""
    h, w = img.shape[:2]
    dh, dw = max(1, h // 2), max(1, w // 2)
    y0, y1 = np.minimum(2 * np.arange(dh), h - 1), np.minimum(2 * np.arange(dh) + 1, h - 1)
    x0, x1 = np.minimum(2 * np.arange(dw), w - 1), np.minimum(2 * np.arange(dw) + 1, w - 1)
    s = img[y0][:, x0].astype(np.int32) + img[y0][:, x1] + img[y1][:, x0] + img[y1][:, x1] + 2
    return (s >> 2).astype(np.uint8)


def make_dataset(bx, by, seeds, side, device=0, log=print, mips=0, fixed=False):
    """Inputs (n, k0p) float32 and labels of every block of side x side textures of the
    given generator seeds and of their first `mips` mip levels, labelled by the full search
    on the GPU (with the reference's semantics, or FIXED ones: fixed=True)."""
    from . import synth
    lay = Layout(bx, by)
    enc = ASTCEncoder(device=device, fixed=fixed)
    enc.init()
    xs, ps, bs = [], [], []
    t0 = time.time()
    for s in seeds:
        img = synth.make_texture(side, side, s)
        for level in range(mips + 1):
            if level:
                img = mip_down(img)
            h, w = img.shape[:2]
            enc.secondaryInit(w, h, bx, by)
            sym = enc.encode_symbolic(img)
            part, bm, ok = labels_from_symbolic(sym, bx, by)
            xs.append(network_inputs(block_rgba8(img, bx, by)[ok], lay.inputs_padded))
            ps.append(part[ok])
            bs.append(bm[ok])
    enc.close()
    log("labelled %d blocks in %.1f s" % (sum(len(p) for p in ps), time.time() - t0))
    return np.concatenate(xs), np.concatenate(ps), np.concatenate(bs)


def init_weights(lay, seed=0):
    rng = np.random.default_rng(seed)

    def lin(n_out, n_in):
        bound = np.sqrt(6.0 / n_in)
        return rng.uniform(-bound, bound, (n_out, n_in)).astype(np.float32), np.zeros(n_out, np.float32)

    w1, b1 = lin(HIDDEN, lay.inputs)
    w2, b2 = lin(HIDDEN, HIDDEN)
    w3, b3 = lin(lay.outputs, HIDDEN)
    w3 *= 0.1
    return {"w1": w1, "b1": b1, "w2": w2, "b2": b2, "w3": w3, "b3": b3}


class Trainer:
    """Adam on the training loss with the library's kernels; parameters FP32 on the GPU."""

    def __init__(self, lay, weights, batch=2048, lr=1e-3, device=0):
        import torch
        self.torch = torch
        self.lay, self.batch, self.lr = lay, batch, lr
        self.dev = torch.device("cuda", device)
        self.stream = torch.cuda.Stream(device=self.dev)
        self.lib = load_library()
        k0p = lay.inputs_padded
        w1 = np.zeros((HIDDEN, k0p), np.float32)
        w1[:, : lay.inputs] = weights["w1"]
        host = dict(weights, w1=w1)
        self.p = {k: torch.from_numpy(np.ascontiguousarray(v)).to(self.dev) for k, v in host.items()}
        self.g = {k: torch.zeros_like(v) for k, v in self.p.items()}
        self.m = {k: torch.zeros_like(v) for k, v in self.p.items()}
        self.v = {k: torch.zeros_like(v) for k, v in self.p.items()}
        B, O = batch, lay.outputs
        z = lambda *s: torch.zeros(*s, dtype=torch.float32, device=self.dev)
        self.h1, self.h2, self.z, self.dz = z(B, HIDDEN), z(B, HIDDEN), z(B, O), z(B, O)
        self.dh1, self.dh2, self.loss = z(B, HIDDEN), z(B, HIDDEN), z(B, 2)
        self.sel3 = (ctypes.c_uint32 * 3)(*lay.sel3)
        self.step_no = 0

    def _ptr(self, t):
        return ctypes.c_void_p(t.data_ptr())

    def _gemm(self, A, B, C, M, N, K, sa_i, sa_l, sb_l, sb_j, bias=None, relu=0):
        _check(self.lib.astcb200_train_gemm(self._ptr(A), self._ptr(B), self._ptr(C), M, N, K, sa_i, sa_l, sb_l, sb_j,
                                            self._ptr(bias) if bias is not None else None, relu, 0,
                                            ctypes.c_void_p(self.stream.cuda_stream)))

    def forward(self, x, n):
        """Hidden activations and logits of n rows of x (device, n <= batch)."""
        k0p, O, p = self.lay.inputs_padded, self.lay.outputs, self.p
        self._gemm(x, p["w1"], self.h1, n, HIDDEN, k0p, k0p, 1, 1, k0p, p["b1"], 1)
        self._gemm(self.h1, p["w2"], self.h2, n, HIDDEN, HIDDEN, HIDDEN, 1, 1, HIDDEN, p["b2"], 1)
        self._gemm(self.h2, p["w3"], self.z, n, O, HIDDEN, HIDDEN, 1, 1, HIDDEN, p["b3"], 0)

    def backward(self, x, part, bm, n):
        """Gradients of the mean loss over n rows into self.g; returns the per-row losses."""
        lay, p, g, s = self.lay, self.p, self.g, ctypes.c_void_p(self.stream.cuda_stream)
        k0p, O, lib = lay.inputs_padded, lay.outputs, self.lib
        _check(lib.astcb200_train_xent(self._ptr(self.z), O, self._ptr(part), self._ptr(bm), n, lay.nbm, lay.head_stride,
                                       self.sel3, self._ptr(self.dz), self._ptr(self.loss), s))
        self._gemm(self.dz, self.h2, g["w3"], O, HIDDEN, n, 1, O, HIDDEN, 1)
        _check(lib.astcb200_train_colsum(self._ptr(self.dz), self._ptr(g["b3"]), n, O, s))
        self._gemm(self.dz, p["w3"], self.dh2, n, HIDDEN, O, O, 1, HIDDEN, 1)
        _check(lib.astcb200_train_relu_backward(self._ptr(self.dh2), self._ptr(self.h2), n * HIDDEN, s))
        self._gemm(self.dh2, self.h1, g["w2"], HIDDEN, HIDDEN, n, 1, HIDDEN, HIDDEN, 1)
        _check(lib.astcb200_train_colsum(self._ptr(self.dh2), self._ptr(g["b2"]), n, HIDDEN, s))
        self._gemm(self.dh2, p["w2"], self.dh1, n, HIDDEN, HIDDEN, HIDDEN, 1, HIDDEN, 1)
        _check(lib.astcb200_train_relu_backward(self._ptr(self.dh1), self._ptr(self.h1), n * HIDDEN, s))
        self._gemm(self.dh1, x, g["w1"], HIDDEN, k0p, n, 1, HIDDEN, k0p, 1)
        _check(lib.astcb200_train_colsum(self._ptr(self.dh1), self._ptr(g["b1"]), n, HIDDEN, s))
        return self.loss[:n]

    def adam(self):
        self.step_no += 1
        for k in self.p:
            _check(self.lib.astcb200_train_adam(self._ptr(self.p[k]), self._ptr(self.g[k]), self._ptr(self.m[k]),
                                                self._ptr(self.v[k]), self.p[k].numel(), self.lr, 0.9, 0.999, 1e-8,
                                                self.step_no, ctypes.c_void_p(self.stream.cuda_stream)))

    def fit(self, X, part, bm, epochs, seed=0, log=print, lr_end=None):
        torch = self.torch
        with torch.cuda.stream(self.stream):
            Xd = torch.from_numpy(X).to(self.dev)
            Pd = torch.from_numpy(part.astype(np.int32)).to(self.dev)
            Bd = torch.from_numpy(bm.astype(np.int32)).to(self.dev)
            n = X.shape[0]
            rng = np.random.default_rng(seed)
            steps = epochs * (n // self.batch)
            lr0 = self.lr
            for ep in range(epochs):
                perm = torch.from_numpy(rng.permutation(n)).to(self.dev)
                tot = torch.zeros(2, dtype=torch.float64, device=self.dev)
                for i in range(n // self.batch):
                    if lr_end is not None:  # cosine decay
                        f = (self.step_no) / max(steps - 1, 1)
                        self.lr = lr_end + 0.5 * (lr0 - lr_end) * (1.0 + np.cos(np.pi * f))
                    idx = perm[i * self.batch:(i + 1) * self.batch]
                    xb, pb, bb = Xd[idx].contiguous(), Pd[idx].contiguous(), Bd[idx].contiguous()
                    self.forward(xb, self.batch)
                    tot += self.backward(xb, pb, bb, self.batch).sum(dim=0, dtype=torch.float64)
                    self.adam()
                self.stream.synchronize()
                t = (tot / ((n // self.batch) * self.batch)).cpu().numpy()
                log("epoch %d: loss partition %.4f block mode %.4f" % (ep, t[0], t[1]))

    def weights(self):
        out = {k: v.detach().cpu().numpy().copy() for k, v in self.p.items()}
        out["w1"] = np.ascontiguousarray(out["w1"][:, : self.lay.inputs])
        return out

    def accuracy(self, X, part, bm, topk=4):
        """Top-1 partition accuracy, top-k partition recall and top-1 block-mode accuracy."""
        torch = self.torch
        from_np = lambda a: torch.from_numpy(a).to(self.dev)
        hits = np.zeros(3)
        n = (X.shape[0] // self.batch) * self.batch
        with torch.cuda.stream(self.stream):
            for i in range(0, n, self.batch):
                self.forward(from_np(X[i:i + self.batch]), self.batch)
                self.stream.synchronize()
                z = self.z.cpu().numpy()
                hits += _accuracy_counts(z, part[i:i + self.batch], bm[i:i + self.batch], self.lay, topk)
        return hits / max(n, 1)


def _accuracy_counts(z, part, bm, lay, topk):
    zp = z[:, : lay.p1 + 1]
    top1 = zp.argmax(axis=1) == part
    topk_idx = np.argsort(-zp[:, : lay.p1], axis=1)[:, :topk]
    recall = (topk_idx == part[:, None]).any(axis=1) | (part == lay.p1)
    heads = lay.head_of(part)
    hz = np.stack([z[np.arange(len(z)), lay.head_base + heads * lay.head_stride + c] for c in range(lay.nbm)], axis=1)
    bm1 = hz.argmax(axis=1) == bm
    return np.array([top1.sum(), recall.sum(), bm1.sum()], np.float64)


# ------------------------------------------------------------ weights on disk
def save_weights(path, w, lay):
    """bf16 weights (the precision the tensor cores use) and FP32 biases."""
    to16 = lambda a: (bf16_round(a).view(np.uint32) >> 16).astype(np.uint16)
    np.savez_compressed(path, w1=to16(w["w1"]), w2=to16(w["w2"]), w3=to16(w["w3"]), b1=w["b1"], b2=w["b2"], b3=w["b3"],
                        footprint=np.array([lay.bx, lay.by]), outputs=np.array(lay.outputs))


def load_weights(bx, by, path=None, labels="fixed"):
    """A shipped network: trained on the FIXED full search's labels (the default) or, with
    labels="ref", on the labels of the full search with the reference's semantics."""
    path = path or os.path.join(WEIGHTS_DIR, "proposal_%dx%d%s.npz" % (bx, by, "" if labels == "fixed" else "_ref"))
    d = np.load(path)
    to32 = lambda a: (a.astype(np.uint32) << 16).view(np.float32)
    return {"w1": to32(d["w1"]), "w2": to32(d["w2"]), "w3": to32(d["w3"]), "b1": d["b1"].astype(np.float32),
            "b2": d["b2"].astype(np.float32), "b3": d["b3"].astype(np.float32), "footprint": tuple(int(v) for v in d["footprint"])}


def available(bx, by):
    return os.path.exists(os.path.join(WEIGHTS_DIR, "proposal_%dx%d.npz" % (bx, by)))


def main():
    ap = argparse.ArgumentParser(description="train the proposal network of one footprint on the GPU")
    ap.add_argument("--footprint", default="4x4")
    ap.add_argument("--blocks", type=int, default=2_000_000, help="training blocks (seeds 100-199)")
    ap.add_argument("--epochs", type=int, default=10)
    ap.add_argument("--batch", type=int, default=2048)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--mips", type=int, default=2, help="also train on this many mip levels of each texture")
    ap.add_argument("--semantics", default="fixed", choices=["ref", "fixed"],
                    help="labels from the full search with the reference's semantics or with its shader bugs repaired")
    ap.add_argument("--out", required=True)
    args = ap.parse_args()
    bx, by = (int(v) for v in args.footprint.split("x"))
    lay = Layout(bx, by)
    seeds = list(range(100, 200))
    per = args.blocks / len(seeds)
    side = int(np.ceil(np.sqrt(per))) * max(bx, by)  # about blocks/100 blocks per texture
    X, part, bm = make_dataset(bx, by, seeds, side, mips=args.mips, fixed=args.semantics == "fixed")
    nval = min(65536, len(X) // 20)
    tr = Trainer(lay, init_weights(lay, seed=1), batch=args.batch, lr=args.lr)
    t0 = time.time()
    tr.fit(X[nval:], part[nval:], bm[nval:], args.epochs, lr_end=args.lr * 0.05)
    print("trained in %.1f s" % (time.time() - t0))
    print("held-out accuracy (partition top-1, partition top-4 recall, block mode top-1):", tr.accuracy(X[:nval], part[:nval], bm[:nval]))
    save_weights(args.out, tr.weights(), lay)


if __name__ == "__main__":
    main()
