// C-ABI plumbing of libpocean_b200.so: per-thread error messages, launch checks, device check, version.
#include <cstdarg>
#include <cstdio>

#include "common.cuh"

static thread_local char g_last_error[512] = "";

int pocean_fail(int code, const char* fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
    va_end(ap);
    return code;
}

// Reports a launch failure of the kernels just enqueued (configuration errors surface here; faults during
// execution surface at the caller's next synchronisation).
int pocean_check_launch(const char* what)
{
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return pocean_fail(POCEAN_ECUDA, "%s: %s", what, cudaGetErrorString(e));
    g_last_error[0] = '\0';
    return POCEAN_OK;
}

// The kernels are built for sm_100a only; refuse other devices with a clear message instead of a launch error.
int pocean_check_device()
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return pocean_fail(POCEAN_ECUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
    static thread_local int checked_dev = -1;
    if (checked_dev == dev) return POCEAN_OK;
    int major = 0, minor = 0;
    cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
    cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, dev);
    if (major != 10 || minor != 0)
        return pocean_fail(POCEAN_EDEVICE, "libpocean_b200 is built for sm_100a (B200); device %d is sm_%d%d", dev,
                           major, minor);
    checked_dev = dev;
    return POCEAN_OK;
}

extern "C" const char* pocean_last_error(void) { return g_last_error; }

extern "C" int pocean_version(void) { return 100; }   // 0.1.0

// A strided 2-D copy in either direction (host pinned <-> device, or device <-> device), stream-ordered: the
// host-buffer paths of the Python layer use it to move row blocks of a (planes, rows, columns) array between a
// strided host array and a dense device block, so copies of one block overlap work on another.
extern "C" int pocean_memcpy2d_async(void* dst, size_t dpitch, const void* src, size_t spitch, size_t width,
                                     size_t height, void* stream)
{
    if (!dst || !src) return pocean_fail(POCEAN_EINVAL, "pocean_memcpy2d_async: null pointer");
    if (width > dpitch || width > spitch)
        return pocean_fail(POCEAN_EINVAL, "pocean_memcpy2d_async: width %zu exceeds a pitch (%zu, %zu)", width, dpitch,
                           spitch);
    if (width == 0 || height == 0) return POCEAN_OK;
    cudaError_t e = cudaMemcpy2DAsync(dst, dpitch, src, spitch, width, height, cudaMemcpyDefault,
                                      (cudaStream_t)stream);
    if (e != cudaSuccess) return pocean_fail(POCEAN_ECUDA, "pocean_memcpy2d_async: %s", cudaGetErrorString(e));
    return POCEAN_OK;
}
