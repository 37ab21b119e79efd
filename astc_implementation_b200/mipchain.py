"""Mip-chain encoding to .astc containers, on the device from upload to container.

The reference encodes the one image it is given and writes it with store_image
(astc_store.cpp:18-62).  Here a texture's whole box-filtered mip chain is built on the
GPU (astcb200_downsample_device), every level is encoded in one batch
(astcb200_encode_batch_device) and each level's .astc container is assembled by
astcb200_astc_containers_device: the 16-byte header written on the host, the blocks
copied straight from device memory into pinned host memory, so the only host-side work
is the final copy out of the pinned buffers.  PyTorch provides the device and pinned
buffers and the stream.
"""
import numpy as np

from . import ASTCError, BAD_ARG, astc_containers_device, downsample_device, mip_dims


def blocks_of(width, height, block_x, block_y):
    return ((width + block_x - 1) // block_x) * ((height + block_y - 1) // block_y)


def encode_mip_chain_astc(encoder, rgba8, block_x, block_y, levels=None, paths=None):
    """Encodes the mip chain of rgba8 ((h, w, 4) uint8, host) with `encoder` (an
    ASTCEncoder, whose search settings and networks apply) and returns one .astc
    container (bytes) per level, level 0 first; `levels` limits the chain's length.
    With `paths` (one file name per level), the containers are also written there."""
    import torch

    img = np.ascontiguousarray(rgba8, dtype=np.uint8)
    if img.ndim != 3 or img.shape[2] != 4:
        raise ASTCError(BAD_ARG, "rgba8 must be an (h, w, 4) uint8 array")
    h, w = img.shape[0], img.shape[1]
    dims = mip_dims(w, h)
    if levels is not None:
        dims = dims[:max(1, int(levels))]
    if paths is not None and len(paths) != len(dims):
        raise ASTCError(BAD_ARG, "one path per mip level is needed")
    dev = torch.device("cuda", encoder.device)
    stream = torch.cuda.Stream(device=dev)
    with torch.cuda.device(dev), torch.cuda.stream(stream):
        src = torch.from_numpy(img.reshape(-1)).pin_memory()
        lv = [torch.empty(lw * lh * 4, dtype=torch.uint8, device=dev) for lw, lh in dims]
        lv[0].copy_(src, non_blocking=True)
        for i in range(1, len(dims)):
            downsample_device(lv[i - 1].data_ptr(), dims[i - 1][0], dims[i - 1][1], lv[i].data_ptr(), stream.cuda_stream)
        nb = [blocks_of(lw, lh, block_x, block_y) for lw, lh in dims]
        outs = [torch.empty(n * 16, dtype=torch.uint8, device=dev) for n in nb]
        encoder.encode_batch_device([(lv[i].data_ptr(), lw, lh, block_x, block_y, outs[i].data_ptr(), nb[i] * 16)
                                     for i, (lw, lh) in enumerate(dims)], stream.cuda_stream)
        host = [torch.empty(16 + n * 16, dtype=torch.uint8).pin_memory() for n in nb]
        astc_containers_device([(outs[i].data_ptr(), host[i].numpy(), lw, lh, block_x, block_y)
                                for i, (lw, lh) in enumerate(dims)], stream.cuda_stream)
    stream.synchronize()
    files = [bytes(hb.numpy()) for hb in host]
    if paths is not None:
        for data, path in zip(files, paths):
            with open(path, "wb") as f:
                f.write(data)
    return files
