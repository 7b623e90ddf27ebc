"""ctypes binding of libpocean_b200.so (include/pocean_b200.h).

The CUDA library is the only compute path of this package: there is no CPU fallback.  ``lib()`` raises a
``RuntimeError`` naming the missing piece when the shared object has not been built or cannot be loaded.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpocean_b200.so")

# flags and codes of include/pocean_b200.h
OPEN_W, OPEN_E, OPEN_S, OPEN_N = 0x1, 0x2, 0x4, 0x8
PERIODIC_X, PERIODIC_Y = 0x10, 0x20
WENO_JS = 0x40
FCT_UNLIMITED = 0x80
FACES_UP3 = 0x100
FACES_UP1 = 0x200
TIME_PC = 0x400
HELPER_SCHEME, HELPER_CENTRED, HELPER_DONOR = 0, 1, 2
PCM, PLM, PPM_H4 = 0, 1, 2
REGRID_ZSTAR, REGRID_SIGMA = 0, 1
ERRORS = {1: "invalid argument", 2: "workspace", 3: "CUDA error", 4: "unsupported device", 5: "step cannot proceed"}

# Every symbol the header declares, with its ctypes signature.
_P, _I, _U, _D, _Z = ctypes.c_void_p, ctypes.c_int, ctypes.c_uint, ctypes.c_double, ctypes.c_size_t
_L = ctypes.c_longlong
SIGNATURES: dict[str, tuple] = {
    "pocean_advect_fct_layers": (_I, [_I, _P, _P, _P, _P, _P, _P, _P, _I, _I, _I, _I, _U, _D, _P, _P, _Z, _I, _I, _I,
                                      _P]),
    "pocean_memcpy2d_async": (_I, [_P, _Z, _P, _Z, _Z, _Z, _P]),
    "pocean_reconstruct_f64": (_I, [_P, _P, _I, _L, _I, _P, _P]),
    "pocean_advect_faces_f64": (_I, [_P, _P, _P, _P, _P, _I, _I, _I, _I, _U, _I, _P, _P, _P]),
    "pocean_advect_rhs_workspace_bytes": (_Z, [_I, _I, _I, _I]),
    "pocean_advect_rhs_f64": (_I, [_P, _P, _P, _P, _P, _P, _I, _I, _I, _I, _U, _I, _P, _P, _Z, _P]),
    "pocean_last_error": (ctypes.c_char_p, []),
    "pocean_version": (_I, []),
    "pocean_advect_fct_workspace_bytes": (_Z, [_I, _I, _I, _I]),
    "pocean_advect_fct_f64": (_I, [_P, _P, _P, _P, _P, _P, _P, _I, _I, _I, _I, _U, _D, _P, _I, _P, _P, _P, _Z,
                                   _P]),
    "pocean_advect_fct_mixed": (_I, [_P, _P, _P, _P, _P, _P, _P, _I, _I, _I, _I, _U, _D, _P, _I, _P, _P, _P, _Z,
                                     _P]),
    "pocean_advect_fct_f64_noalloc": (_I, [_P, _P, _P, _P, _P, _P, _P, _I, _I, _I, _I, _U, _D, _P, _I, _P, _P,
                                           _P]),
    "pocean_advect_rk3_workspace_bytes": (_Z, [_I, _I, _I, _I]),
    "pocean_advect_rk3_f64": (_I, [_P, _P, _P, _P, _P, _P, _P, _P, _I, _I, _I, _I, _U, _D, _P, _I, _P, _P, _Z,
                                   _P]),
    "pocean_remap_columns_f64": (_I, [_P, _P, _P, _P, _I, _I, _I, _I, _I, _I, _P, _P]),
    "pocean_regrid_remap_f64": (_I, [_I, _P, _P, _P, _P, _P, _D, _P, _I, _I, _I, _I, _I, _P, _P, _P, _P, _P]),
    "pocean_regrid_hybrid_remap_f64": (_I, [_P, _P, _P, _P, _P, _P, _P, _P, _P, _D, _D, _D, _I, _P, _I, _I, _I, _I,
                                            _I, _P, _P, _P, _P, _P]),
    "pocean_face_fractions_f64": (_I, [_P, _I, _I, _I, _P, _P]),
    "pocean_remap_faces_f64": (_I, [_P, _P, _P, _P, _I, _I, _I, _I, _I, _P, _P]),
    "pocean_diffuse_ale_f64": (_I, [_P, _P, _P, _P, _P, _P, _P, _P, _P, _I, _I, _I, _I, _U, _D, _D, _P, _P]),
    "pocean_face_transport_thickness_f64": (_I, [_P, _P, _P, _I, _I, _I, _I, _P, _P, _P]),
    "pocean_transport_velocity_f64": (_I, [_P, _P, _P, _P, _P, _P, _I, _I, _I, _D, _D, _P, _P, _P]),
    "pocean_ppm_edges_f64": (_I, [_P, _P, _I, _I, _I, _D, _P, _P, _P]),
    "pocean_ppm_transport_workspace_bytes": (_Z, [_I, _I, _I, _I]),
    "pocean_ppm_transport_f64": (_I, [_P, _P, _P, _P, _P, _P, _P, _P, _I, _I, _I, _D, _I, _P, _P, _Z, _P]),
    "pocean_limit_outflow_workspace_bytes": (_Z, [_I, _I, _I]),
    "pocean_limit_outflow_f64": (_I, [_P, _P, _P, _P, _P, _I, _I, _I, _D, _D, _I, _U, ctypes.POINTER(_I),
                                      ctypes.POINTER(_I), _P, _Z, _P]),
    "pocean_lagrangian_thickness_f64": (_I, [_P, _P, _P, _I, _I, _I, _D, _D, _P, _P, _P]),
    "pocean_upwind_transport_f64": (_I, [_P, _P, _P, _P, _P, _I, _I, _I, _P, _P]),
    "pocean_freshwater_volumes_f64": (_I, [_P, _P, _P, _D, _I, _I, _I, _P, _P, _P]),
    "pocean_flux_divergence_f64": (_I, [_P, _P, _I, _I, _I, _P, _P]),
    "pocean_layer_volumes_f64": (_I, [_P, _P, _P, _I, _I, _I, _P, _P, _P]),
    "pocean_regrid_columns_f64": (_I, [_I, _P, _P, _P, _P, _P, _P, _P, _P, _P, _D, _D, _D, _I, _I, _I, _I, _I, _P,
                                       _P]),
    "pocean_periodic_pad_f64": (_I, [_P, _I, _I, _I, _I, _I, _I, _I, _I, _P, _P]),
    "pocean_periodic_pad_u8": (_I, [_P, _I, _I, _I, _I, _I, _I, _I, _I, _P, _P]),
    "pocean_periodic_crop_f64": (_I, [_P, _I, _I, _I, _I, _I, _I, _I, _I, _P, _P]),
    "pocean_open_face_transport_f64": (_I, [_P, _L, _L, _P, _P, _L, _L, _P, _P, _P, _L, _I, _I, _D, _P, _L, _L,
                                            _P]),
    "pocean_batch_device_bytes": (_Z, [_I]),
    "pocean_batch_create": (_I, [_P, _I, _I, _P, _Z, ctypes.POINTER(_P), _P]),
    "pocean_batch_step": (_I, [_P, _I, _I, _I, _P]),
    "pocean_batch_destroy": (None, [_P]),
}

_LIB: ctypes.CDLL | None = None


class PoceanError(RuntimeError):
    """A libpocean_b200 call returned an error status."""


def lib() -> ctypes.CDLL:
    """The loaded library with typed entry points; raises if it is missing."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m pyocean_b200.build` "
                               "(or __graft_entry__.build()); this package has no CPU fallback")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = L
    return _LIB


def check(rc: int, what: str) -> None:
    """Raise PoceanError (ValueError for argument errors) when a call returned a non-zero status."""
    if rc == 0:
        return
    msg = lib().pocean_last_error().decode(errors="replace")
    if rc == 1:
        raise ValueError(f"{what}: {msg}")
    raise PoceanError(f"{what}: {ERRORS.get(rc, rc)}: {msg}")
