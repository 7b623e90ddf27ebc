// The per-column remap driver shared by every kernel that remaps columns (remap.cu, neighbours.cu): how a column's
// thicknesses and fields are reached is the IO object's business (plain arrays, a regrid computed in registers,
// fractions formed on the fly), the remap arithmetic is remap_core.cuh's.
#pragma once

#include "common.cuh"
#include "remap_core.cuh"

namespace po {
namespace remap {

// Bit pattern left in out[field, 0, column] for a column that the general algorithm must finish (a NaN payload
// that no arithmetic here produces; a coincidental match only costs a recomputation with the exact algorithm).
constexpr long long kRedo = 0x7FF40000C0DE0001ll;

// Column c of (k, plane) arrays: thicknesses h (source) and t (target), NF fields u in, o out.
template <int NF>
struct ColumnIO {
    const double* __restrict__ h;
    const double* __restrict__ t;
    const double* __restrict__ u[NF];
    double* __restrict__ o[NF];
    i64 plane;
    __device__ __forceinline__ double hs(int k) const { return __ldg(h + k * plane); }
    __device__ __forceinline__ double ht(int k) const { return __ldg(t + k * plane); }
    __device__ __forceinline__ double f(int m, int k) const { return __ldg(u[m] + k * plane); }
    __device__ __forceinline__ void put(int m, int k, double v) { o[m][k * plane] = v; }
};

// The same for fields of fewer than 2^31 entries: the arrays' bases are the same for every thread of a block (kept
// in uniform registers), the column and layer enter as one 32-bit offset per access.
template <int NF>
struct ColumnIO32 {
    const double* __restrict__ h;
    const double* __restrict__ t;
    const double* __restrict__ u[NF];
    double* __restrict__ o[NF];
    int c, plane;
    __device__ __forceinline__ double hs(int k) const { return __ldg(h + (c + k * plane)); }
    __device__ __forceinline__ double ht(int k) const { return __ldg(t + (c + k * plane)); }
    __device__ __forceinline__ double f(int m, int k) const { return __ldg(u[m] + (c + k * plane)); }
    __device__ __forceinline__ void put(int m, int k, double v) { o[m][c + k * plane] = v; }
};

// remap.py:400-415 for one column and NF fields: a column that is not wet is copied (n0 == n1) or NaN; a column
// with a negative or NaN target thickness gets the sentinel (the general algorithm finishes it in a later launch);
// otherwise the one-pass sweep, or the no-active-source rule.
template <int NF, class IO>
__device__ __forceinline__ void remap_column_io(IO& io, bool wet, int n0, int n1, int scheme)
{
    if (!wet) {                                      // remap.py:405-408
#pragma unroll
        for (int m = 0; m < NF; ++m)
            for (int k = 0; k < n1; ++k) io.put(m, k, n0 == n1 ? io.f(m, k) : nan(""));
        return;
    }
    int n_active = 0, last = -1;
    for (int k = 0; k < n0; ++k)
        if (io.hs(k) > 0.0) { ++n_active; last = k; }
    bool regular = true;
    for (int k = 0; k < n1; ++k) regular = regular && io.ht(k) >= 0.0;
    if (!regular) {
#pragma unroll
        for (int m = 0; m < NF; ++m) io.put(m, 0, __longlong_as_double(kRedo));
        return;
    }
    if (n_active == 0) rc::remap_column_dry<NF>(io, n0, n1);
    else rc::remap_column_stream<NF>(io, n0, n1, scheme, n_active, last);
}

}  // namespace remap

// The general-algorithm fixup of every sentinel column of out (nfields, n1, plane) (remap.cu).
void remap_general_launch(const double* h_src, const double* f_src, const double* h_tgt, int n0, int n1, i64 plane,
                          int nfields, int scheme, double* out, cudaStream_t st);

}  // namespace po
