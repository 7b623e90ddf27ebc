"""
pyocean_b200 — pyOCEAN's baroclinic tracer hot path on NVIDIA B200 (sm_100a).

* ``TracerAdvection`` (advect_fct: SSP-RK3 WENO5 with Zalesak FCT; advect: SSP-RK3 without limiter) and
  ``remap_columns`` / ``remap_column`` (PCM / PLM / PPM_H4 conservative remap) and ``reconstruct`` with the
  reference's signatures.
* The neighbours: ``ALECoordinate`` (z* / sigma / hybrid ``regrid_remap``, ``regrid``, ``remap_faces``),
  ``regrid_columns`` (the rules' interface heights, a hybrid target layer count other than the source's included),
  ``face_fractions``
  and ``diffuse_ale`` (the ALE horizontal diffusion kernel); ``producers`` (face transport thickness, transport
  velocity, PPM layer transport, outflow limiter, Lagrangian thickness).
* ``ale_tracer_step``: advect_fct then remap_columns in one call, the advected stack kept on the device.
* The compute path is libpocean_b200.so (hand-written CUDA, C ABI in include/pocean_b200.h), loaded with ctypes;
  PyTorch provides device memory and streams.  There is no CPU fallback.
"""
from __future__ import annotations

from .periodic import NONE, TRACER_HALO, Periodic
from .remap import MAX_LAYERS, PCM, PLM, PPM_H4, SCHEMES, reconstruct, remap_column, remap_columns
from .tracers import OpenEdges, TracerAdvection
from .vertical import ALECoordinate, face_fractions, regrid_columns, remap_faces
from .diffusion import diffuse_ale
from .step import ale_tracer_step
from . import producers

__all__ = ["TracerAdvection", "OpenEdges", "Periodic", "NONE", "TRACER_HALO", "remap_columns", "remap_column",
           "reconstruct", "PCM", "PLM", "PPM_H4", "SCHEMES", "MAX_LAYERS", "ALECoordinate", "face_fractions", "remap_faces",
           "diffuse_ale", "producers", "ale_tracer_step", "regrid_columns"]
