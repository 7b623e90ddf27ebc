// FP64 conservative vertical remap (PCM / PLM / PPM_H4) of water columns on B200.
//
// Reference: core/vertical/remap.py — remap_column :306-397, reconstruct :234-294, _average :297-303,
// _remap_columns :400-415 (one call per field there; here every field of the stack in one launch).
//
// Mapping.  One thread owns one column and NF fields of it; consecutive threads take consecutive i, so each
// per-layer load or store of a warp is one contiguous 256-byte segment of the (k, j, i) arrays (a warp per column
// would touch 8 bytes of every 32-byte sector instead).  The column is processed in one pass (remap_core.cuh,
// remap_column_stream): a 6-cell register window builds each source cell's polynomial from its neighbours and the
// cell is integrated at once over the targets it overlaps; no column array is stored, thickness-only factors are
// computed once for all NF fields.  Columns whose target thicknesses are not all >= 0 (outside the sweep's
// domain) are marked with a sentinel in their first output layer and finished by a second launch with the
// reference's array formulation (remap_column_general); the second launch reads one value per column otherwise.
// Both paths give the reference's numbers bit for bit (-fmad=false, reference expression order).
#include <cmath>

#include "common.cuh"
#include "fct_args.cuh"
#include "remap_core.cuh"
#include "remap_io.cuh"

// Launch bounds of the streaming remap; POCEAN_REMAP_CTAS (resident CTAs per SM) sets its register budget.  Fitted to 5 CTAs (20 warps) per SM: 10 % faster than ptxas's choice (128
// registers with spills, 4 CTAs), 6 % faster than 6 CTAs, measured at 512 x 512 x 50 with two fields.
#ifndef POCEAN_REMAP_CTAS
#define POCEAN_REMAP_CTAS 5
#endif
// One field per thread (NF = 1: a lone or odd field, one-tracer domains of a batch) has fewer registers to keep:
// fitted to 7 CTAs per SM, 15 % faster than 5 (1.30 against 1.53 ms for two single-field remaps at 512 x 512 x 50)
// and than 6 or 8.
#ifndef POCEAN_REMAP1_CTAS
#define POCEAN_REMAP1_CTAS 7
#endif
#define REMAP_BOUNDS __launch_bounds__(128, NF == 1 ? POCEAN_REMAP1_CTAS : POCEAN_REMAP_CTAS)

namespace po {
namespace remap {

// One column c of NF fields m0 .. m0+NF-1: f_src (nfields, n0, plane) -> out (nfields, n1, plane).
template <int NF, typename IX>
__device__ __forceinline__ void remap_stream_body(const double* __restrict__ h_src, const double* __restrict__ f_src,
                                                  const double* __restrict__ h_tgt, const uint8_t* __restrict__ wet,
                                                  int n0, int n1, i64 plane, int m0, int scheme,
                                                  double* __restrict__ out, i64 c)
{
    if (sizeof(IX) == 4) {
        ColumnIO32<NF> io;
        io.h = h_src;
        io.t = h_tgt;
        io.c = (int)c;
        io.plane = (int)plane;
#pragma unroll
        for (int m = 0; m < NF; ++m) {
            io.u[m] = f_src + (i64)(m0 + m) * n0 * plane;
            io.o[m] = out + (i64)(m0 + m) * n1 * plane;
        }
        remap_column_io<NF>(io, wet[c] != 0, n0, n1, scheme);
    } else {
        ColumnIO<NF> io;
        io.h = h_src + c;
        io.t = h_tgt + c;
        io.plane = plane;
#pragma unroll
        for (int m = 0; m < NF; ++m) {
            io.u[m] = f_src + (i64)(m0 + m) * n0 * plane + c;
            io.o[m] = out + (i64)(m0 + m) * n1 * plane + c;
        }
        remap_column_io<NF>(io, wet[c] != 0, n0, n1, scheme);
    }
}

template <int NMAX>
__device__ __forceinline__ void remap_general_body(const double* __restrict__ h_src, const double* __restrict__ f_src,
                                                   const double* __restrict__ h_tgt, int n0, int n1, i64 plane,
                                                   int m, int scheme, double* __restrict__ out, i64 c)
{
    double* o = out + (i64)m * n1 * plane + c;
    if (__double_as_longlong(o[0]) != kRedo) return;
    ColumnIO<1> io;
    io.h = h_src + c;
    io.t = h_tgt + c;
    io.plane = plane;
    io.u[0] = f_src + (i64)m * n0 * plane + c;
    io.o[0] = o;
    rc::remap_column_general<NMAX>(io, 0, n0, n1, scheme);
}

template <int NF, typename IX>
__global__ void REMAP_BOUNDS remap_stream_kernel(const double* __restrict__ h_src,
                                                           const double* __restrict__ f_src,
                                                           const double* __restrict__ h_tgt,
                                                           const uint8_t* __restrict__ wet, int n0, int n1, i64 plane,
                                                           int field0, int scheme, double* __restrict__ out)
{
    const i64 c = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= plane) return;
    remap_stream_body<NF, IX>(h_src, f_src, h_tgt, wet, n0, n1, plane, field0 + (int)blockIdx.y * NF, scheme, out, c);
}

template <int NMAX>
__global__ void __launch_bounds__(128) remap_general_kernel(const double* __restrict__ h_src,
                                                            const double* __restrict__ f_src,
                                                            const double* __restrict__ h_tgt, int n0, int n1,
                                                            i64 plane, int scheme, double* __restrict__ out)
{
    const i64 c = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= plane) return;
    remap_general_body<NMAX>(h_src, f_src, h_tgt, n0, n1, plane, blockIdx.y, scheme, out, c);
}

// Batched remap of every domain's advected stack (D.a.out -> D.rout).  Mode: NF = 2 over field pairs (group g =
// fields 2g, 2g+1), or NF = 1 over single fields starting at `first` (the odd field left by the pairs, or all).
template <int NF>
__global__ void REMAP_BOUNDS remap_stream_batched(const BatchDomain* __restrict__ doms,
                                                            const int* __restrict__ off, int ndom, int odd_only)
{
    const int d = find_domain(off, ndom, blockIdx.x);
    const BatchDomain& D = doms[d];
    const Shape s = D.a.s;
    const i64 plane = (i64)s.ny * s.nx;
    const int cblocks = (int)((plane + 127) / 128);
    const int local = blockIdx.x - __ldg(off + d);
    const int g = local / cblocks;
    const i64 c = (i64)(local - g * cblocks) * 128 + threadIdx.x;
    if (c >= plane) return;
    const int m0 = NF == 2 ? 2 * g : (odd_only ? s.nt - 1 : g);
    // the batch bounds every field by 2^31 entries
    remap_stream_body<NF, int>(D.h_src, D.a.out, D.h_tgt, D.wet, s.n, s.n, plane, m0, D.remap_scheme, D.rout, c);
}

template <int NMAX>
__global__ void __launch_bounds__(128) remap_general_batched(const BatchDomain* __restrict__ doms,
                                                             const int* __restrict__ off, int ndom)
{
    const int d = find_domain(off, ndom, blockIdx.x);
    const BatchDomain& D = doms[d];
    const Shape s = D.a.s;
    const i64 plane = (i64)s.ny * s.nx;
    const int cblocks = (int)((plane + 127) / 128);
    const int local = blockIdx.x - __ldg(off + d);
    const int m = local / cblocks;
    const i64 c = (i64)(local - m * cblocks) * 128 + threadIdx.x;
    if (c >= plane) return;
    remap_general_body<NMAX>(D.h_src, D.a.out, D.h_tgt, s.n, s.n, plane, m, D.remap_scheme, D.rout, c);
}

// reconstruct (remap.py:234-294) of ncols columns of n cells: h, u (n, ncols), coef (n, ncols, 3); the scheme as
// given (PCM below 3 cells, PLM below 4 for PPM_H4, as there).
template <int NMAX>
__global__ void __launch_bounds__(128) reconstruct_kernel(const double* __restrict__ h, const double* __restrict__ u,
                                                          int n, i64 ncols, int scheme, double* __restrict__ coef)
{
    const i64 c = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncols) return;
    double hh[NMAX], uu[NMAX], c0[NMAX], c1[NMAX], c2[NMAX], e0[NMAX], e1[NMAX];
    for (int k = 0; k < n; ++k) {
        hh[k] = __ldg(h + (k * ncols + c));
        uu[k] = __ldg(u + (k * ncols + c));
    }
    rc::reconstruct_column(hh, uu, n, scheme, c0, c1, c2, e0, e1);
    for (int k = 0; k < n; ++k) {
        double* o = coef + 3 * (k * ncols + c);
        o[0] = c0[k];
        o[1] = c1[k];
        o[2] = c2[k];
    }
}

}  // namespace remap

// nf_mode 2: field pairs (+ the odd field); nf_mode 1: every field on its own.  nmax: the batch's deepest column.
void remap_batched_launch(const BatchDomain* doms, const int* off_dev, const int* off_host, int ndom, int nf_mode,
                          int nmax, cudaStream_t st)
{
    auto total = [&](int pass) { return (unsigned)off_host[pass * (ndom + 1) + ndom]; };
    auto offs = [&](int pass) { return off_dev + pass * (ndom + 1); };
    if (nf_mode == 2) {
        if (total(BP_RPAIR)) remap::remap_stream_batched<2><<<total(BP_RPAIR), 128, 0, st>>>(doms, offs(BP_RPAIR), ndom, 0);
        if (total(BP_RREM)) remap::remap_stream_batched<1><<<total(BP_RREM), 128, 0, st>>>(doms, offs(BP_RREM), ndom, 1);
    } else {
        remap::remap_stream_batched<1><<<total(BP_RALL), 128, 0, st>>>(doms, offs(BP_RALL), ndom, 0);
    }
    if (nmax <= 64) remap::remap_general_batched<64><<<total(BP_RGEN), 128, 0, st>>>(doms, offs(BP_RGEN), ndom);
    else if (nmax <= 128) remap::remap_general_batched<128><<<total(BP_RGEN), 128, 0, st>>>(doms, offs(BP_RGEN), ndom);
    else remap::remap_general_batched<256><<<total(BP_RGEN), 128, 0, st>>>(doms, offs(BP_RGEN), ndom);
}

void remap_general_launch(const double* h_src, const double* f_src, const double* h_tgt, int n0, int n1, i64 plane,
                          int nfields, int scheme, double* out, cudaStream_t st)
{
    const dim3 g2((unsigned)((plane + 127) / 128), (unsigned)nfields);
    const int nm = n0 > n1 ? n0 : n1;
    if (nm <= 64)
        remap::remap_general_kernel<64><<<g2, 128, 0, st>>>(h_src, f_src, h_tgt, n0, n1, plane, scheme, out);
    else if (nm <= 128)
        remap::remap_general_kernel<128><<<g2, 128, 0, st>>>(h_src, f_src, h_tgt, n0, n1, plane, scheme, out);
    else
        remap::remap_general_kernel<256><<<g2, 128, 0, st>>>(h_src, f_src, h_tgt, n0, n1, plane, scheme, out);
}

}  // namespace po

using namespace po;

extern "C" int pocean_remap_columns_f64(const double* h_src, const double* f_src, const double* h_tgt,
                                        const uint8_t* wet, int n0, int n1, int ny, int nx, int nfields, int scheme,
                                        double* out, void* stream)
{
    const char* fn = "pocean_remap_columns_f64";
    if (n0 < 1 || n1 < 1 || ny < 1 || nx < 1 || nfields < 1)
        return pocean_fail(POCEAN_EINVAL, "%s: sizes must be >= 1 (n0=%d n1=%d ny=%d nx=%d nfields=%d)", fn, n0, n1,
                           ny, nx, nfields);
    if (n0 > 256 || n1 > 256)
        return pocean_fail(POCEAN_EINVAL, "%s: at most 256 layers per column (n0=%d n1=%d)", fn, n0, n1);
    if (nfields > 65535) return pocean_fail(POCEAN_EINVAL, "%s: nfields=%d exceeds 65535", fn, nfields);
    if (scheme < POCEAN_PCM || scheme > POCEAN_PPM_H4)
        return pocean_fail(POCEAN_EINVAL, "%s: unknown scheme %d", fn, scheme);
    if (!h_src || !f_src || !h_tgt || !wet || !out) return pocean_fail(POCEAN_EINVAL, "%s: null pointer", fn);
    int rc = pocean_check_device();
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    const i64 plane = (i64)ny * nx;
    const unsigned gx = (unsigned)((plane + 127) / 128);
    const int pairs = nfields / 2;
    // 32-bit offsets within a field when every field (n0 or n1 layers of the plane) holds fewer than 2^31 entries
    const bool small = (i64)(n0 > n1 ? n0 : n1) * plane < (1ll << 31);
    if (pairs > 0) {
        if (small)
            remap::remap_stream_kernel<2, int><<<dim3(gx, pairs), 128, 0, st>>>(h_src, f_src, h_tgt, wet, n0, n1,
                                                                                plane, 0, scheme, out);
        else
            remap::remap_stream_kernel<2, i64><<<dim3(gx, pairs), 128, 0, st>>>(h_src, f_src, h_tgt, wet, n0, n1,
                                                                                plane, 0, scheme, out);
    }
    if (nfields & 1) {
        if (small)
            remap::remap_stream_kernel<1, int><<<dim3(gx, 1), 128, 0, st>>>(h_src, f_src, h_tgt, wet, n0, n1, plane,
                                                                            nfields - 1, scheme, out);
        else
            remap::remap_stream_kernel<1, i64><<<dim3(gx, 1), 128, 0, st>>>(h_src, f_src, h_tgt, wet, n0, n1, plane,
                                                                            nfields - 1, scheme, out);
    }
    remap_general_launch(h_src, f_src, h_tgt, n0, n1, plane, nfields, scheme, out, st);
    return pocean_check_launch(fn);
}

extern "C" int pocean_reconstruct_f64(const double* h, const double* u, int n, long long ncols, int scheme,
                                      double* coef, void* stream)
{
    const char* fn = "pocean_reconstruct_f64";
    if (n < 1 || ncols < 1)
        return pocean_fail(POCEAN_EINVAL, "%s: sizes must be >= 1 (n=%d ncols=%lld)", fn, n, ncols);
    if (n > 256) return pocean_fail(POCEAN_EINVAL, "%s: at most 256 cells per column (n=%d)", fn, n);
    if (ncols > (1ll << 40)) return pocean_fail(POCEAN_EINVAL, "%s: ncols=%lld too large", fn, ncols);
    if (scheme < POCEAN_PCM || scheme > POCEAN_PPM_H4)
        return pocean_fail(POCEAN_EINVAL, "%s: unknown scheme %d", fn, scheme);
    if (!h || !u || !coef) return pocean_fail(POCEAN_EINVAL, "%s: null pointer", fn);
    int rc = pocean_check_device();
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    const unsigned g = (unsigned)((ncols + 127) / 128);
    if (n <= 64) remap::reconstruct_kernel<64><<<g, 128, 0, st>>>(h, u, n, (i64)ncols, scheme, coef);
    else if (n <= 128) remap::reconstruct_kernel<128><<<g, 128, 0, st>>>(h, u, n, (i64)ncols, scheme, coef);
    else remap::reconstruct_kernel<256><<<g, 128, 0, st>>>(h, u, n, (i64)ncols, scheme, coef);
    return pocean_check_launch(fn);
}
