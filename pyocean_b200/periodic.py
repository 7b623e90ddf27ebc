"""Periodic horizontal axes of a domain, as the reference names them (core/model/periodic.py:47-70).

The reference reaches the wrap by padding its inputs with ``TRACER_HALO`` wrapped cells and cropping the result;
the CUDA kernels wrap every stencil index natively, which gives the same numbers (the FCT step's dependency radius
is 10 cells, below the 13-cell halo) without the copies.  Any object with boolean ``x`` / ``y`` attributes (the
reference's own ``Periodic`` included) is accepted where a ``Periodic`` is expected.
"""
from __future__ import annotations

TRACER_HALO = 13      # core/model/periodic.py:31 (kept for callers that pad themselves)
AXES = ("x", "y")


class Periodic:
    """Which horizontal axes wrap: a tuple with ``"x"``, ``"y"`` or both; falsy when none."""

    def __init__(self, axes=()) -> None:
        if isinstance(axes, str):
            axes = (axes,)
        axes = tuple(axes or ())
        bad = [a for a in axes if a not in AXES]
        if bad:
            raise ValueError(f"unknown periodic axes {bad}; use 'x', 'y' or both")
        self.x, self.y = "x" in axes, "y" in axes
        self.axes = tuple(a for a in AXES if a in axes)

    def __bool__(self) -> bool:
        return self.x or self.y

    def __repr__(self) -> str:
        return f"Periodic({self.axes})"


NONE = Periodic()
