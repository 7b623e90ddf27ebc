// Plane index -> layer of the k-major (layer, tracer) planes of the advection launches, without an integer
// division (compiled for the host too by tests/hostcore).
#pragma once

#ifdef __CUDACC__
#define PO_PD __host__ __device__ __forceinline__
#else
#define PO_PD inline
#endif

namespace po {

// Division of a plane index p by the tracer count nt as a multiply-high (Granlund & Montgomery 1994, "Division by
// invariant integers using multiplication"): with m = ceil(2^32 / nt) and e = m nt - 2^32 < nt,
// floor(p m / 2^32) = floor(p / nt) whenever p e < 2^32, which holds for 0 <= p < 2^16 and 1 <= nt < 2^16 (the
// entry points bound nt * nz by 65535).  nt = 1 is encoded as m = 0 and divides by identity.
PO_PD unsigned plane_magic(int nt)
{
    return nt <= 1 ? 0u : (unsigned)((0x100000000ull + (unsigned long long)nt - 1) / (unsigned long long)nt);
}

PO_PD int plane_div(int p, unsigned m)
{
    return m == 0u ? p : (int)(((unsigned long long)(unsigned)p * m) >> 32);
}

}  // namespace po
