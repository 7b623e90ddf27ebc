"""Device buffers of the host mirror: inputs as contiguous CUDA tensors, outputs back in the caller's type.

Arrays may be NumPy (copied to the current CUDA device, results copied back to NumPy) or CUDA torch tensors
(used in place, results returned as torch tensors on the same device).  PyTorch is used here for device memory and
streams only; every computation happens in libpocean_b200.so.
"""
from __future__ import annotations

import numpy as np
import torch


class Converter:
    """Moves a call's arrays to one CUDA device and remembers whether the caller wants NumPy back."""

    def __init__(self, *arrays) -> None:
        dev = None
        host_torch = False
        for a in arrays:
            if isinstance(a, torch.Tensor):
                if not a.is_cuda:
                    host_torch = True
                    continue
                if dev is not None and a.device != dev:
                    raise ValueError(f"arrays on different devices: {dev} and {a.device}")
                dev = a.device
        # results come back as the inputs came: CUDA tensors stay on the device, host torch tensors (pinned
        # ones copy asynchronously) come back as pinned host tensors, NumPy arrays as NumPy arrays
        self.mode = "cuda" if dev is not None else ("host" if host_torch else "numpy")
        self.numpy_out = self.mode == "numpy"
        if dev is None:
            if not torch.cuda.is_available():
                raise RuntimeError("pyocean_b200 needs a CUDA device (B200); none is visible")
            dev = torch.device("cuda", torch.cuda.current_device())
        self.device = dev

    def f64(self, a, shape: tuple | None = None) -> torch.Tensor:
        """``a`` as a C-contiguous float64 tensor on the device (broadcast to ``shape`` if given)."""
        if isinstance(a, torch.Tensor):
            t = a.to(device=self.device, dtype=torch.float64, non_blocking=True)
        else:
            t = torch.from_numpy(np.ascontiguousarray(np.asarray(a, dtype=np.float64))).to(self.device)
        if shape is not None and tuple(t.shape) != tuple(shape):
            t = t.expand(shape)
        return t.contiguous()

    def u8(self, a, shape: tuple) -> torch.Tensor:
        """A boolean mask as a contiguous uint8 (0/1) tensor of ``shape`` on the device."""
        if isinstance(a, torch.Tensor):
            t = a.to(self.device, non_blocking=True)
            t = t if t.dtype == torch.uint8 else (t != 0).to(torch.uint8)
        else:
            t = torch.from_numpy(np.ascontiguousarray(np.asarray(a, dtype=bool)).view(np.uint8)).to(self.device)
        if tuple(t.shape) != tuple(shape):
            t = t.expand(shape)
        return t.contiguous()

    def empty(self, shape) -> torch.Tensor:
        return torch.empty(tuple(shape), dtype=torch.float64, device=self.device)

    def workspace(self, nbytes: int) -> torch.Tensor:
        return torch.empty(max(int(nbytes), 256), dtype=torch.uint8, device=self.device)

    def stream(self) -> int:
        return torch.cuda.current_stream(self.device).cuda_stream

    def out(self, t: torch.Tensor):
        """The result in the caller's type (host copies synchronise on the current stream)."""
        if self.mode == "cuda":
            return t
        if self.mode == "numpy":
            return t.cpu().numpy()
        h = torch.empty(t.shape, dtype=t.dtype, pin_memory=True)
        h.copy_(t, non_blocking=True)
        torch.cuda.current_stream(self.device).synchronize()
        return h


def shape_of(a) -> tuple:
    return tuple(a.shape) if isinstance(a, torch.Tensor) else np.shape(a)
