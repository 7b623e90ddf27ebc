// Shared definitions of the pyOCEAN B200 kernels: indexing of the (t, k, j, i) stacks and C-grid faces, the
// periodic wrap, error reporting of the C ABI.
#pragma once

#include <cstdint>
#include <cstddef>
#include <cuda_runtime.h>

#include "../../include/pocean_b200.h"
#include "planediv.cuh"

typedef long long i64;

// Error reporting of the C ABI (defined in abi.cu).
int pocean_fail(int code, const char* fmt, ...);
int pocean_check_launch(const char* what);
int pocean_check_device();

namespace po {

// Shape of one domain and the indexing of its arrays (C order, k = 0 at the bed).
struct Shape {
    int nt, n, ny, nx;
    __host__ __device__ i64 plane() const { return (i64)ny * nx; }
    __host__ __device__ i64 xplane() const { return (i64)ny * (nx + 1); }
    __host__ __device__ i64 yplane() const { return (i64)(ny + 1) * nx; }
    // cell (t, k, j, i) of a stack; geometry (k, j, i); u-face (t, k, j, f); v-face (t, k, f, i)
    __host__ __device__ i64 cell(int t, int k, int j, int i) const { return (((i64)t * n + k) * ny + j) * nx + i; }
    __host__ __device__ i64 geo(int k, int j, int i) const { return ((i64)k * ny + j) * nx + i; }
    __host__ __device__ i64 ux(int t, int k, int j, int f) const { return (((i64)t * n + k) * ny + j) * (nx + 1) + f; }
    __host__ __device__ i64 vy(int t, int k, int f, int i) const { return (((i64)t * n + k) * (ny + 1) + f) * nx + i; }
    __host__ __device__ i64 qx(int k, int j, int f) const { return ((i64)k * ny + j) * (nx + 1) + f; }
    __host__ __device__ i64 qy(int k, int f, int i) const { return ((i64)k * (ny + 1) + f) * nx + i; }
};

// Offset of plane p of a stack whose planes hold `elems` elements, as one 32 x 32 -> 64-bit product (p >= 0 and
// elems < 2^31: the entry points bound every field by 2^31 entries).
__host__ __device__ __forceinline__ i64 plane_at(int p, int elems)
{
    return (i64)((unsigned long long)(unsigned)p * (unsigned)elems);
}

// Periodic wrap of a cell index (any integer) onto 0..n-1.
__host__ __device__ __forceinline__ int wrap(int i, int n) {
    int r = i % n;
    return r < 0 ? r + n : r;
}

// Python's builtin max/min on floats: the first argument unless the second is strictly larger / smaller.
__host__ __device__ __forceinline__ double pmax(double a, double b) { return (b > a) ? b : a; }
__host__ __device__ __forceinline__ double pmin(double a, double b) { return (b < a) ? b : a; }

__host__ __device__ __forceinline__ int ceil_div(int a, int b) { return (a + b - 1) / b; }

}  // namespace po
