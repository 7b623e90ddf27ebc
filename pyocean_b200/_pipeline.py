"""Host-array paths with the copies overlapped: blocks of the arrays move host -> device on one stream, the kernels of
a block run on a second, results move device -> host on a third, so the copies of one block overlap the kernels of
another and the two copy directions overlap each other.

Used for pinned, contiguous host (CPU) torch tensors only (pageable memory cannot be copied asynchronously); the
arithmetic is the same launches on smaller independent pieces (row blocks of columns for the remap, single tracers
of the stack for the FCT step), so results equal the one-shot path bit for bit.  PyTorch provides the device memory,
streams and events; the strided block copies are ``pocean_memcpy2d_async``.
"""
from __future__ import annotations

import torch

from . import _lib

_STREAMS: dict = {}
MIN_BYTES = 32 << 20            # smaller calls run the one-shot path (their copies are short anyway)
REMAP_ROW_BLOCKS = 8            # row blocks of the remap's host path (swept at 512 x 512 x 50)
FCT_LAYER_BLOCKS = 6            # layer blocks of the FCT step's host path (swept likewise)


def streams(device: torch.device) -> tuple:
    """(in, compute, out) streams of a device, created once."""
    key = device.index
    if key not in _STREAMS:
        _STREAMS[key] = tuple(torch.cuda.Stream(device) for _ in range(3))
    return _STREAMS[key]


def pinned(*arrays) -> bool:
    """Every array given (None skipped) is a contiguous pinned CPU torch tensor."""
    got = False
    for a in arrays:
        if a is None:
            continue
        if not (isinstance(a, torch.Tensor) and not a.is_cuda and a.is_pinned() and a.is_contiguous()):
            return False
        got = True
    return got


def copy2d(dst: int, dpitch: int, src: int, spitch: int, width: int, height: int, stream: torch.cuda.Stream) -> None:
    """Strided block copy of ``height`` rows of ``width`` bytes (pointers as integers)."""
    _lib.check(_lib.lib().pocean_memcpy2d_async(dst, dpitch, src, spitch, width, height, stream.cuda_stream),
               "memcpy2d")


def row_blocks(ny: int, nblocks: int) -> list[tuple[int, int]]:
    """``nblocks`` (or fewer) consecutive row ranges covering 0 .. ny."""
    nblocks = max(1, min(nblocks, ny))
    step = -(-ny // nblocks)
    return [(j, min(j + step, ny)) for j in range(0, ny, step)]


def device_now() -> torch.device:
    if not torch.cuda.is_available():
        raise RuntimeError("pyocean_b200 needs a CUDA device (B200); none is visible")
    return torch.device("cuda", torch.cuda.current_device())
