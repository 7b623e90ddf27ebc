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
# Blocks of the host paths: (full blocks, relative sizes of the smaller last blocks).  The work that follows the
# last upload of a call — the last block's kernels and the downloads of what they finish — shrinks with the last
# blocks.  Swept at 512 x 512 x 50 with T and S (pinned host tensors, ms per step): the two drop-in calls 23.38 ms
# with 6 / 8 equal blocks, 22.82 ms with the tapered blocks below; the one-call step (``ale_tracer_step``, no
# download between the two parts) is fastest with 6 / 8 equal blocks (17.70 ms against 18.28 ms tapered).
FCT_BLOCKS = (10, (0.5, 0.25))          # layer blocks of advect_fct
REMAP_BLOCKS = (12, (0.5, 0.25))        # row blocks of remap_columns
FUSED_FCT_BLOCKS = (6, ())              # the same inside ale_tracer_step
FUSED_REMAP_BLOCKS = (8, ())


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


def row_blocks(ny: int, nblocks: int, tail: tuple = ()) -> list[tuple[int, int]]:
    """Consecutive row ranges covering 0 .. ny: ``nblocks`` full blocks (or fewer), then blocks of the relative
    sizes ``tail`` (fractions of a full block, e.g. (0.5, 0.25)); every block holds at least one row."""
    nblocks = max(1, min(nblocks, ny))
    if not tail:
        step = -(-ny // nblocks)
        return [(j, min(j + step, ny)) for j in range(0, ny, step)]
    weights = [1.0] * nblocks + [float(w) for w in tail]
    edges, acc, tot = [0], 0.0, sum(weights)
    for w in weights[:-1]:
        acc += w
        edges.append(min(max(round(ny * acc / tot), edges[-1] + 1), ny))
    edges.append(ny)
    return [(a, b) for a, b in zip(edges[:-1], edges[1:]) if b > a]


def device_now() -> torch.device:
    if not torch.cuda.is_available():
        raise RuntimeError("pyocean_b200 needs a CUDA device (B200); none is visible")
    return torch.device("cuda", torch.cuda.current_device())
