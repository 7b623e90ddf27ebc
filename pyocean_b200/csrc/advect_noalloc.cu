// advect_fct for callers that cannot allocate device memory.
//
// pocean_advect_fct_f64 takes its scratch from a caller-provided workspace.  Some callers have no way to provide
// one: a host model that reaches the GPU only through this C ABI from a language binding with no device
// allocator of its own (a Fortran or plain ctypes driver without PyTorch), or a caller whose device memory is
// owned by a pool or budget that forbids side allocations.  For them, pocean_advect_fct_f64_noalloc runs the same
// FCT step on a fixed scratch array that lives in this translation unit's module: it allocates nothing
// (no cudaMalloc, no cudaFree, no allocating library call).
//
// Limits and rules of the shared scratch:
//   * size: POCEAN_NOALLOC_SCRATCH_BYTES (64 MiB).  Every GPU that loads this module holds the array until the
//     process exits.  A shape whose workspace (pocean_advect_fct_workspace_bytes) exceeds it is rejected with
//     POCEAN_EINVAL and a message; nothing is launched.
//   * every call looks up the array's device address on the current device (cudaGetSymbolAddress, a host-side
//     table lookup once the module is loaded) and checks the result.  The address is not kept between calls: a
//     module loaded again (after cudaDeviceReset, or in another context of the same device) may sit at another
//     address, and a cached one would then point at unmapped memory.  The first call on a device loads the module
//     there; make it before any stream capture on that device.
//   * every call on a device uses the same array and it keeps the last call's contents.  The FCT passes write
//     every scratch element before they read it, so nothing needs clearing between calls; but calls that overlap
//     on the GPU (different streams, or different host threads, without ordering between them) race on the
//     array and give wrong results.  Order them on one stream.
#include "common.cuh"

static __device__ __align__(256) unsigned char g_fct_scratch[POCEAN_NOALLOC_SCRATCH_BYTES];

namespace {

// Device address of g_fct_scratch in the current context of the current device.
int scratch_for_current_device(void** out)
{
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_fct_scratch);
    if (e != cudaSuccess || p == nullptr)
        return pocean_fail(POCEAN_ECUDA, "pocean_advect_fct_f64_noalloc: cudaGetSymbolAddress: %s",
                           cudaGetErrorString(e));
    *out = p;
    return POCEAN_OK;
}

}  // namespace

extern "C" int pocean_advect_fct_f64_noalloc(const double* C, const double* V0, const double* V1, const double* Qx,
                                             const double* Qy, const uint8_t* ok, const double* inflow, int nt,
                                             int nz, int ny, int nx, unsigned flags, double dt, double* C_out,
                                             int face_i, double* fx_face, double* open_flux, void* stream)
{
    const size_t need = pocean_advect_fct_workspace_bytes(nt, nz, ny, nx);
    if (need == 0)
        return pocean_fail(POCEAN_EINVAL, "pocean_advect_fct_f64_noalloc: sizes must be >= 1 (nt=%d nz=%d ny=%d nx=%d)",
                           nt, nz, ny, nx);
    if (need > (size_t)POCEAN_NOALLOC_SCRATCH_BYTES)
        return pocean_fail(POCEAN_EINVAL,
                           "pocean_advect_fct_f64_noalloc: shape nt=%d nz=%d ny=%d nx=%d needs %zu bytes of scratch, "
                           "more than the fixed %zu-byte array; use pocean_advect_fct_f64 with a workspace",
                           nt, nz, ny, nx, need, (size_t)POCEAN_NOALLOC_SCRATCH_BYTES);
    void* scratch = nullptr;
    int rc = scratch_for_current_device(&scratch);
    if (rc) return rc;
    return pocean_advect_fct_f64(C, V0, V1, Qx, Qy, ok, inflow, nt, nz, ny, nx, flags, dt, C_out, face_i, fx_face,
                                 open_flux, scratch, (size_t)POCEAN_NOALLOC_SCRATCH_BYTES, stream);
}
