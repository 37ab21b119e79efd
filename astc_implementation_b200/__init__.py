"""ASTC LDR block-compression search on one NVIDIA B200.

Host-side mirror of Jure-Z/ASTC_implementation's encoder facade over the C-ABI
library ``libastcb200.so`` (include/astcb200.h):

    enc = ASTCEncoder(device=0)            # ASTCEncoder(const wgpu::Device&)   astc.h:726
    enc.init()                             # ASTCEncoder::init()                 compression_pipeline.cpp:219
    enc.secondaryInit(w, h, bx, by)        # ASTCEncoder::secondaryInit(...)     compression_pipeline.cpp:263
    blocks = enc.encode(rgba8)             # ASTCEncoder::encode(data, out, len) compression_pipeline.cpp:323
    store_image(bx, by, w, h, blocks, path)  # store_image(...)                 astc_store.cpp:18

Errors are raised as ASTCError carrying the library's status code (the
reference throws std::runtime_error).  The CUDA library is required: nothing
here falls back to a CPU path.
"""
import ctypes
import os

import numpy as np

__all__ = ["ASTCEncoder", "ASTCError", "store_image", "decode", "load_library", "VALID_FOOTPRINTS", "Texture",
           "downsample_device", "mip_dims", "astc_containers_device"]

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libastcb200.so")
_lib = None

VALID_FOOTPRINTS = [(4, 4), (5, 4), (5, 5), (6, 5), (6, 6), (8, 5), (8, 6), (10, 5), (10, 6),
                    (8, 8), (10, 8), (10, 10), (12, 10), (12, 12)]

OK, INVALID_FOOTPRINT, BAD_ARG, OOM, CUDA_ERROR, TIMEOUT, NO_IMAGE, IO_ERROR, TOO_LARGE = range(9)


class ASTCError(RuntimeError):
    def __init__(self, status, message):
        super().__init__("%s (status %d)" % (message, status))
        self.status = status


class _Config(ctypes.Structure):
    _fields_ = [("struct_size", ctypes.c_uint32), ("chunk_blocks", ctypes.c_uint32),
                ("timeout_ms", ctypes.c_uint32), ("flags", ctypes.c_uint32)]


class Stats(ctypes.Structure):
    _fields_ = [("ms_wall", ctypes.c_double), ("ms_device", ctypes.c_double), ("blocks", ctypes.c_uint64),
                ("h2d_bytes", ctypes.c_uint64), ("d2h_bytes", ctypes.c_uint64),
                ("launches", ctypes.c_uint32), ("reserved", ctypes.c_uint32)]


class Texture(ctypes.Structure):
    """astcb200_texture: one texture of a batch."""
    _fields_ = [("rgba8", ctypes.c_void_p), ("out_blocks", ctypes.c_void_p), ("out_len", ctypes.c_size_t),
                ("width", ctypes.c_uint32), ("height", ctypes.c_uint32), ("block_x", ctypes.c_uint8),
                ("block_y", ctypes.c_uint8), ("reserved", ctypes.c_uint8 * 6)]


class AstcImage(ctypes.Structure):
    """astcb200_astc_image: one image of astcb200_astc_containers_device."""
    _fields_ = [("d_blocks", ctypes.c_void_p), ("host_out", ctypes.c_void_p), ("out_len", ctypes.c_size_t),
                ("width", ctypes.c_uint32), ("height", ctypes.c_uint32), ("block_x", ctypes.c_uint8),
                ("block_y", ctypes.c_uint8), ("reserved", ctypes.c_uint8 * 6)]


class Tuning(ctypes.Structure):
    _fields_ = [("chunk_blocks", ctypes.c_uint32), ("streams", ctypes.c_uint32), ("ms", ctypes.c_double)]


FLAG_STAGE_TIMING, FLAG_NO_GRAPH, FLAG_FIXED_SEMANTICS, FLAG_VOID_EXTENT, FLAG_DUAL_PLANE = 1, 2, 4, 8, 16


class ProposalNet(ctypes.Structure):
    _fields_ = [("struct_size", ctypes.c_uint32), ("block_x", ctypes.c_uint8), ("block_y", ctypes.c_uint8),
                ("reserved", ctypes.c_uint8 * 2), ("inputs", ctypes.c_uint32), ("hidden", ctypes.c_uint32),
                ("outputs", ctypes.c_uint32), ("w1", ctypes.c_void_p), ("b1", ctypes.c_void_p), ("w2", ctypes.c_void_p),
                ("b2", ctypes.c_void_p), ("w3", ctypes.c_void_p), ("b3", ctypes.c_void_p)]


class Pruning(ctypes.Structure):
    _fields_ = [("struct_size", ctypes.c_uint32), ("enable", ctypes.c_uint32), ("max_partitionings", ctypes.c_uint32),
                ("block_modes", ctypes.c_uint32), ("refine_candidates", ctypes.c_uint32), ("coverage", ctypes.c_float),
                ("threshold", ctypes.c_float), ("reroute_error", ctypes.c_float), ("front_threads", ctypes.c_uint32),
                ("refine_iterations", ctypes.c_uint32), ("single_partition_floor", ctypes.c_float),
                ("fallback_iterations", ctypes.c_uint32)]


def load_library():
    """Loads libastcb200.so, building it first when it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH):
        from . import build as _build
        _build.build()
    lib = ctypes.CDLL(_LIB_PATH)
    P, U32, I32, SZ = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_int, ctypes.c_size_t
    sig = {
        "astcb200_create": (I32, [ctypes.POINTER(P), I32, ctypes.POINTER(_Config)]),
        "astcb200_destroy": (I32, [P]),
        "astcb200_set_image": (I32, [P, U32, U32, ctypes.c_uint8, ctypes.c_uint8]),
        "astcb200_blocks": (I32, [P, ctypes.POINTER(U32), ctypes.POINTER(U32)]),
        "astcb200_set_timeout": (I32, [P, U32]),
        "astcb200_set_inference_wait_limit": (I32, [P, U32]),
        "astcb200_encode": (I32, [P, P, P, SZ, ctypes.POINTER(Stats)]),
        "astcb200_encode_device": (I32, [P, P, P, P]),
        "astcb200_encode_symbolic": (I32, [P, P, P, SZ]),
        "astcb200_search_stages": (I32, [P, P, P, SZ, P, SZ, P, SZ]),
        "astcb200_store_image": (I32, [U32, U32, U32, U32, P, SZ, ctypes.c_char_p]),
        "astcb200_astc_containers_device": (I32, [ctypes.POINTER(AstcImage), U32, P]),
        "astcb200_decode": (I32, [U32, U32, U32, U32, P, SZ, P]),
        "astcb200_stage_times": (I32, [P, P, P]),
        "astcb200_stage_times_detail": (I32, [P, P, P]),
        "astcb200_work_counters": (I32, [P, P]),
        "astcb200_encode_noalloc": (I32, [I32, P, U32, U32, ctypes.c_uint8, ctypes.c_uint8, P, P]),
        "astcb200_encode_batch": (I32, [P, ctypes.POINTER(Texture), U32, ctypes.POINTER(Stats)]),
        "astcb200_encode_batch_device": (I32, [P, ctypes.POINTER(Texture), U32, P]),
        "astcb200_autotune_batch": (I32, [P, ctypes.POINTER(Texture), U32, ctypes.POINTER(Tuning), ctypes.POINTER(Tuning),
                                          U32, ctypes.POINTER(U32)]),
        "astcb200_downsample_device": (I32, [P, U32, U32, P, P]),
        "astcb200_proposal_layout": (I32, [ctypes.c_uint8, ctypes.c_uint8] + [ctypes.POINTER(U32)] * 6 + [P]),
        "astcb200_set_proposal_net": (I32, [P, ctypes.POINTER(ProposalNet)]),
        "astcb200_set_pruning": (I32, [P, ctypes.POINTER(Pruning)]),
        "astcb200_pruning_stats": (I32, [P, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64)]),
        "astcb200_decode_device": (I32, [U32, U32, U32, U32, P, P, P]),
        "astcb200_decode_error_device": (I32, [U32, U32, U32, U32, P, P, P, P]),
        "astcb200_proposal_logits": (I32, [P, P, P, SZ]),
        "astcb200_proposal_selection": (I32, [P, P, P, P, P, SZ]),
        "astcb200_train_gemm": (I32, [P, P, P, I32, I32, I32, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64,
                                      P, I32, I32, P]),
        "astcb200_train_xent": (I32, [P, U32, P, P, U32, U32, U32, P, P, P, P]),
        "astcb200_train_relu_backward": (I32, [P, P, SZ, P]),
        "astcb200_train_colsum": (I32, [P, P, U32, U32, P]),
        "astcb200_train_adam": (I32, [P, P, P, P, SZ, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float, U32, P]),
        "astcb200_status_string": (ctypes.c_char_p, [I32]),
        "astcb200_last_error": (ctypes.c_char_p, [P]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype, f.argtypes = res, args
    _lib = lib
    return lib


def _check(rc, ctx=None):
    if rc != OK:
        lib = load_library()
        msg = lib.astcb200_status_string(rc).decode()
        if ctx:
            detail = lib.astcb200_last_error(ctx).decode()
            if detail:
                msg += ": " + detail
        raise ASTCError(rc, msg)


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data)


class ASTCEncoder:
    """One encoder context bound to one GPU and one CUDA stream."""

    def __init__(self, device=0, chunk_blocks=0, timeout_ms=0, stage_timing=False, use_graphs=True, fixed=False,
                 void_extent=False, dual_plane=False):
        """fixed=True selects the search with the reference's deterministic shader bugs repaired
        (ASTCB200_FLAG_FIXED_SEMANTICS); the default reproduces the reference bit for bit.
        void_extent / dual_plane enable the encodings the reference never emits
        (ASTCB200_FLAG_VOID_EXTENT, ASTCB200_FLAG_DUAL_PLANE)."""
        lib = load_library()
        flags = ((FLAG_STAGE_TIMING if stage_timing else 0) | (0 if use_graphs else FLAG_NO_GRAPH)
                 | (FLAG_FIXED_SEMANTICS if fixed else 0) | (FLAG_VOID_EXTENT if void_extent else 0)
                 | (FLAG_DUAL_PLANE if dual_plane else 0))
        cfg = _Config(ctypes.sizeof(_Config), chunk_blocks, timeout_ms, flags)
        ctx = ctypes.c_void_p()
        _check(lib.astcb200_create(ctypes.byref(ctx), device, ctypes.byref(cfg)))
        self._ctx = ctx
        self.device = device
        self.fixed = bool(fixed)
        self.blocksX = self.blocksY = self.numBlocks = 0
        self.textureWidth = self.textureHeight = 0
        self.blockXDim = self.blockYDim = 4
        self.is_initialized = False
        self.last_stats = None

    def init(self):
        """Kernels are compiled ahead of time; kept for the reference's call sequence."""
        self.is_initialized = True

    def secondaryInit(self, textureWidth, textureHeight, blockXDim, blockYDim):
        lib = load_library()
        _check(lib.astcb200_set_image(self._ctx, textureWidth, textureHeight, blockXDim, blockYDim), self._ctx)
        bx, by = ctypes.c_uint32(), ctypes.c_uint32()
        _check(lib.astcb200_blocks(self._ctx, ctypes.byref(bx), ctypes.byref(by)), self._ctx)
        self.textureWidth, self.textureHeight = textureWidth, textureHeight
        self.blockXDim, self.blockYDim = blockXDim, blockYDim
        self.blocksX, self.blocksY = bx.value, by.value
        self.numBlocks = bx.value * by.value

    def _image(self, imageData):
        img = np.ascontiguousarray(imageData, dtype=np.uint8)
        if img.size != self.textureWidth * self.textureHeight * 4:
            raise ASTCError(BAD_ARG, "image must hold width*height*4 bytes")
        return img

    def encode(self, imageData, dataOut=None):
        """Encodes an RGBA8 image; returns (and fills dataOut with) numBlocks*16 bytes."""
        lib = load_library()
        img = self._image(imageData)
        out = dataOut if dataOut is not None else np.empty(self.numBlocks * 16, np.uint8)
        if not (isinstance(out, np.ndarray) and out.dtype == np.uint8 and out.flags.c_contiguous):
            raise ASTCError(BAD_ARG, "dataOut must be a contiguous uint8 array")
        st = Stats()
        _check(lib.astcb200_encode(self._ctx, _ptr(img), _ptr(out), out.size, ctypes.byref(st)), self._ctx)
        self.last_stats = st
        return out

    def encode_symbolic(self, imageData):
        """Returns the chosen SymbolicBlock per block (astc.h:639-655) as (numBlocks, 108) u32."""
        lib = load_library()
        img = self._image(imageData)
        sym = np.empty((self.numBlocks, 108), np.uint32)
        _check(lib.astcb200_encode_symbolic(self._ctx, _ptr(img), _ptr(sym), sym.size), self._ctx)
        return sym

    # One partitioned-block record of the front (astcb200_search_stages): pass01's averages and
    # endpoints, then pass12's candidates.
    CANDIDATE = np.dtype([("bm", "<u2"), ("ql", "u1"), ("qlm", "u1"), ("fmt", "u1", (4,)), ("qw", "u1", (64,))])
    RECORD = np.dtype([("avg", "<f4", (4, 4)), ("ep0", "<f4", (4, 4)), ("ep1", "<f4", (4, 4)), ("P", "<u4"),
                       ("entry", "<u4"), ("ncand", "<u4"), ("seed", "<u4"), ("cand", CANDIDATE, (8,))])

    SNAPSHOT = np.dtype([("err", "<f4"), ("bm", "<u2"), ("final_q", "u1"), ("matched", "u1"), ("ffmt", "u1", (4,)),
                         ("pad", "u1", (4,)), ("packed", "u1", (32,)), ("qw", "u1", (64,))])

    def search_stages(self, imageData):
        """Test hook: the full search's partition picks (numBlocks, 16) u16, the front's records
        (numBlocks, 13) of RECORD and, after 6 refinement iterations, every candidate's best
        state (numBlocks, 13, 8) of SNAPSHOT, for an image of at most one chunk."""
        lib = load_library()
        img = self._image(imageData)
        picks = np.empty((self.numBlocks, 16), np.uint16)
        recs = np.empty((self.numBlocks, 13), self.RECORD)
        snaps = np.empty((self.numBlocks, 13, 8), self.SNAPSHOT)
        assert self.RECORD.itemsize == 784 and self.SNAPSHOT.itemsize == 112
        _check(lib.astcb200_search_stages(self._ctx, _ptr(img), _ptr(picks), picks.nbytes, _ptr(recs), recs.nbytes,
                                          _ptr(snaps), snaps.nbytes), self._ctx)
        return picks, recs, snaps

    def encode_device(self, d_rgba8, d_out_blocks, stream=0):
        """Queues the search on device buffers (integer device addresses); does not wait."""
        lib = load_library()
        _check(lib.astcb200_encode_device(self._ctx, ctypes.c_void_p(d_rgba8), ctypes.c_void_p(d_out_blocks),
                                          ctypes.c_void_p(stream or None)), self._ctx)

    def encode_batch(self, textures):
        """Encodes [(rgba8 (h, w, 4) uint8, block_x, block_y), ...] as one batch; returns the
        blocks of each texture (uint8 arrays of blocks*16 bytes) in the same order."""
        lib = load_library()
        imgs, outs = [], []
        arr = (Texture * len(textures))()
        for i, (img, bx, by) in enumerate(textures):
            img = np.ascontiguousarray(img, dtype=np.uint8)
            h, w = img.shape[0], img.shape[1]
            out = np.empty(((w + bx - 1) // bx) * ((h + by - 1) // by) * 16, np.uint8)
            imgs.append(img)
            outs.append(out)
            arr[i] = Texture(img.ctypes.data, out.ctypes.data, out.size, w, h, bx, by)
        st = Stats()
        _check(lib.astcb200_encode_batch(self._ctx, arr, len(textures), ctypes.byref(st)), self._ctx)
        self.last_stats = st
        return outs

    @staticmethod
    def _device_textures(textures):
        arr = (Texture * len(textures))()
        for i, (d_img, w, h, bx, by, d_out, out_len) in enumerate(textures):
            arr[i] = Texture(d_img, d_out, out_len, w, h, bx, by)
        return arr

    def encode_batch_device(self, textures, stream=0):
        """Queues a batch of device textures [(d_rgba8, w, h, bx, by, d_out, out_len), ...]
        (integer device addresses) on `stream`; does not wait."""
        arr = self._device_textures(textures)
        _check(load_library().astcb200_encode_batch_device(self._ctx, arr, len(textures), ctypes.c_void_p(stream or None)),
               self._ctx)

    def autotune_batch(self, textures):
        """Times the launch configurations on a device batch (as for encode_batch_device) and
        keeps the fastest for batches of this shape.  Returns (best, tried) as
        (chunk_blocks, streams, ms) tuples."""
        arr = self._device_textures(textures)
        best, tried, n = Tuning(), (Tuning * 32)(), ctypes.c_uint32()
        _check(load_library().astcb200_autotune_batch(self._ctx, arr, len(textures), ctypes.byref(best), tried, 32,
                                                      ctypes.byref(n)), self._ctx)
        return ((best.chunk_blocks, best.streams, best.ms),
                [(tried[i].chunk_blocks, tried[i].streams, tried[i].ms) for i in range(n.value)])

    def set_proposal_net(self, w, block_x=None, block_y=None):
        """Loads a trained proposal network (dict of FP32 w1, b1, w2, b2, w3, b3) for a footprint."""
        bx, by = (block_x, block_y) if block_x else w["footprint"]
        arrs = {k: np.ascontiguousarray(w[k], dtype=np.float32) for k in ("w1", "b1", "w2", "b2", "w3", "b3")}
        net = ProposalNet(ctypes.sizeof(ProposalNet), bx, by, (ctypes.c_uint8 * 2)(), arrs["w1"].shape[1], arrs["w1"].shape[0],
                          arrs["w3"].shape[0], *[arrs[k].ctypes.data for k in ("w1", "b1", "w2", "b2", "w3", "b3")])
        _check(load_library().astcb200_set_proposal_net(self._ctx, ctypes.byref(net)), self._ctx)

    def set_pruning(self, enable=True, max_partitionings=0, block_modes=0, refine_candidates=0, coverage=0.8,
                    threshold=0.5, reroute_error=8.0, front_threads=0, refine_iterations=0,
                    single_partition_floor=0.0, fallback_iterations=0):
        """Proposal-search settings for later encodes of footprints with a network; 0 in the
        integer settings selects the footprint's tuned value (see astcb200_pruning)."""
        cfg = Pruning(ctypes.sizeof(Pruning), 1 if enable else 0, max_partitionings, block_modes, refine_candidates,
                      coverage, threshold, reroute_error, front_threads, refine_iterations, single_partition_floor,
                      fallback_iterations)
        _check(load_library().astcb200_set_pruning(self._ctx, ctypes.byref(cfg)), self._ctx)

    def pruning_stats(self):
        """(proposal-search blocks, full-search blocks) of the last encode."""
        a, b = ctypes.c_uint64(), ctypes.c_uint64()
        _check(load_library().astcb200_pruning_stats(self._ctx, ctypes.byref(a), ctypes.byref(b)), self._ctx)
        return a.value, b.value

    def proposal_logits(self, imageData, outputs):
        """The proposal network's logits (numBlocks, outputs) for an image (test hook)."""
        img = self._image(imageData)
        z = np.empty((self.numBlocks, outputs), np.float32)
        _check(load_library().astcb200_proposal_logits(self._ctx, _ptr(img), _ptr(z), z.size), self._ctx)
        return z

    def proposal_selection(self, imageData):
        """The proposal search's selection for an image (test hook): route (numBlocks,) with
        0 = proposal search, 1 = full search; picks (numBlocks, 18) = count, flags, then the
        partitionings (P - 2) << 10 | entry; masks (numBlocks, 16) = block-mode bits per P."""
        img = self._image(imageData)
        n = self.numBlocks
        route = np.empty(n, np.uint8)
        picks = np.empty((n, 18), np.uint16)
        masks = np.empty((n, 16), np.uint64)
        _check(load_library().astcb200_proposal_selection(self._ctx, _ptr(img), _ptr(route), _ptr(picks), _ptr(masks), n),
               self._ctx)
        return route, picks, masks

    def stage_times(self):
        """(ms[4], launches[4]) per kernel for the last encode (needs stage_timing=True)."""
        ms = np.zeros(4, np.float32)
        n = np.zeros(4, np.uint32)
        _check(load_library().astcb200_stage_times(self._ctx, _ptr(ms), _ptr(n)), self._ctx)
        return ms, n

    def stage_times_detail(self):
        """Per-launch milliseconds of the last encode by position in the chunk sequence (9 entries)."""
        ms = np.zeros(9, np.float32)
        k = np.zeros(9, np.int32)
        _check(load_library().astcb200_stage_times_detail(self._ctx, _ptr(ms), _ptr(k)), self._ctx)
        return ms, k

    def work_counters(self):
        """Work counters of the last encode (needs stage_timing=True); see astcb200_work_counters."""
        c = np.zeros(16, np.uint64)
        _check(load_library().astcb200_work_counters(self._ctx, _ptr(c)), self._ctx)
        return c

    def set_inference_wait_limit(self, polls):
        """Polls per mbarrier wait of the inference kernel before a CTA gives up (0 = default)."""
        _check(load_library().astcb200_set_inference_wait_limit(self._ctx, int(polls)), self._ctx)

    def set_timeout(self, timeout_ms):
        """Bound (ms) on each later host wait; 0 = none (astcb200_set_timeout)."""
        _check(load_library().astcb200_set_timeout(self._ctx, int(timeout_ms)), self._ctx)

    def close(self):
        if getattr(self, "_ctx", None):
            load_library().astcb200_destroy(self._ctx)
            self._ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def store_image(block_x, block_y, dim_x, dim_y, data, filename):
    """Writes the .astc container (astc_store.cpp:18-62)."""
    lib = load_library()
    buf = np.ascontiguousarray(data, dtype=np.uint8)
    _check(lib.astcb200_store_image(block_x, block_y, dim_x, dim_y, _ptr(buf), buf.size, os.fsencode(filename)))


def astc_containers_device(images, stream=0):
    """Queues the .astc containers of images whose blocks are in device memory:
    [(d_blocks, host_out, width, height, block_x, block_y), ...] with integer device
    addresses and host_out a writable uint8 array (pinned for an asynchronous copy) of at
    least 16 + 16 * blocks bytes.  Synchronise `stream` before reading host_out."""
    arr = (AstcImage * len(images))()
    for i, (d_blocks, host_out, w, h, bx, by) in enumerate(images):
        if not (isinstance(host_out, np.ndarray) and host_out.dtype == np.uint8 and host_out.flags.c_contiguous
                and host_out.flags.writeable):
            raise ASTCError(BAD_ARG, "host_out must be a writable contiguous uint8 array")
        arr[i] = AstcImage(d_blocks, host_out.ctypes.data, host_out.size, w, h, bx, by)
    _check(load_library().astcb200_astc_containers_device(arr, len(images), ctypes.c_void_p(stream or None)))


def decode(block_x, block_y, dim_x, dim_y, blocks):
    """Decodes physical ASTC blocks to an (dim_y, dim_x, 4) uint8 image."""
    lib = load_library()
    buf = np.ascontiguousarray(blocks, dtype=np.uint8)
    out = np.empty((dim_y, dim_x, 4), np.uint8)
    _check(lib.astcb200_decode(block_x, block_y, dim_x, dim_y, _ptr(buf), buf.size, _ptr(out)))
    return out


def decode_device(block_x, block_y, dim_x, dim_y, d_blocks, d_rgba8, stream=0):
    """GPU decode between device buffers (pointers as integers), queued on `stream`;
    the same texels as decode()."""
    _check(load_library().astcb200_decode_device(block_x, block_y, dim_x, dim_y, d_blocks, d_rgba8, stream))


def decode_error_device(block_x, block_y, dim_x, dim_y, d_blocks, d_ref_rgba8, d_sse, stream=0):
    """GPU decode compared with a reference image: writes the per-channel sums of squared
    differences (4 x uint64) to device memory d_sse, queued on `stream`."""
    _check(load_library().astcb200_decode_error_device(block_x, block_y, dim_x, dim_y, d_blocks, d_ref_rgba8, d_sse, stream))


def psnr_from_sse(sse, dim_x, dim_y):
    """PSNR over all RGBA channels from decode_error_device's four sums (same as psnr())."""
    tot = float(sum(int(v) for v in sse))
    return float("inf") if tot == 0 else 10.0 * np.log10(255.0 * 255.0 * 4.0 * dim_x * dim_y / tot)


def encode_noalloc(device, d_rgba8, width, height, block_x, block_y, d_out_blocks, stream=0):
    """Allocation-free encode of at most 2048 blocks between device buffers (queued on
    `stream`, not waited for); see astcb200_encode_noalloc in include/astcb200.h."""
    _check(load_library().astcb200_encode_noalloc(device, ctypes.c_void_p(d_rgba8), width, height, block_x, block_y,
                                                 ctypes.c_void_p(d_out_blocks), ctypes.c_void_p(stream or None)))


def downsample_device(d_src, width, height, d_dst, stream=0):
    """Queues one 2x2 box-filter mip step between device RGBA8 buffers (integer addresses);
    the result is max(1, width//2) x max(1, height//2)."""
    _check(load_library().astcb200_downsample_device(ctypes.c_void_p(d_src), width, height, ctypes.c_void_p(d_dst),
                                                     ctypes.c_void_p(stream or None)))


def mip_dims(width, height):
    """Sizes of the full mip chain of a width x height image, level 0 first, down to 1x1."""
    dims = [(width, height)]
    while dims[-1] != (1, 1):
        w, h = dims[-1]
        dims.append((max(1, w // 2), max(1, h // 2)))
    return dims


def psnr(a, b):
    """PSNR in dB over all RGBA channels of two uint8 images."""
    d = a.astype(np.float64) - b.astype(np.float64)
    mse = float(np.mean(d * d))
    return float("inf") if mse == 0 else 10.0 * np.log10(255.0 * 255.0 / mse)
