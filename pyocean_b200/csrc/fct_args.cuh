// Argument blocks of the advection kernels and of the batched (multi-domain) launches.
#pragma once

#include "common.cuh"

namespace po {

struct Flags {
    bool open_w, open_e, open_s, open_n, per_x, per_y, z;
    __host__ __device__ explicit Flags(unsigned f)
        : open_w(f & POCEAN_OPEN_W), open_e(f & POCEAN_OPEN_E), open_s(f & POCEAN_OPEN_S),
          open_n(f & POCEAN_OPEN_N), per_x(f & POCEAN_PERIODIC_X), per_y(f & POCEAN_PERIODIC_Y),
          z(!(f & POCEAN_WENO_JS)) {}
};

// Everything one FCT / RK3 step reads and writes.
struct StepArgs {
    Shape s;
    unsigned flags;
    double dt;
    const double* __restrict__ C;
    const double* __restrict__ V0;
    const double* __restrict__ V1;
    const double* __restrict__ Qx;
    const double* __restrict__ Qy;
    const double* __restrict__ Fz;      // RK3 only (nullable)
    const uint8_t* __restrict__ ok;
    const double* __restrict__ inflow;  // nullable
    // workspace
    double* q1;
    double* c1;
    double* q2;
    double* c2;
    double* Sx;                         // FCT: F0, then the antidiffusive flux A
    double* Sy;
    double* Tx;                         // FCT: F1
    double* Ty;
    double* tef0;                       // RK3 TEF column accumulators (nt, n, ny)
    double* tef1;
    // outputs
    double* out;
    int face_i;
    int k0;                             // first layer of a layer-range launch of the single-domain passes (else 0)
    unsigned tdiv;                      // plane_magic(s.nt): plane index -> layer without an integer division
    double* fx_face;
};

// One domain of a batch: its FCT arguments (a.C the stack, a.out the advected stack, a.q1.. its workspace) and
// the remap of the advected stack onto its target grid (into rout).  nstrips / nsegs: its strip decomposition for
// the batch's segment length.
struct BatchDomain {
    StepArgs a;
    const double* h_src;
    const double* h_tgt;
    const uint8_t* wet;
    double* rout;
    int remap_scheme;
};

// Layer k and tracer t of plane p = k nt + t (planes run k-major); tdiv = plane_magic(nt).  The multiply-high
// replaces a per-warp integer division (about twenty instructions): 1.6 % of advect_fct at 512 x 512 x 50.
__device__ __forceinline__ void split_plane(int p, int nt, unsigned tdiv, int& k, int& t)
{
    k = plane_div(p, tdiv);
    t = p - k * nt;
}

// CTA offsets of every batched pass: domain d owns CTAs off[d] .. off[d+1]-1 of the launch (ndom + 1 entries each).
enum BatchPass { BP_PTILE = 0, BP_TILE = 1, BP_RPAIR = 2, BP_RREM = 3, BP_RALL = 4, BP_RGEN = 5, BP_COUNT = 6 };

// The domain whose CTA range holds CTA b (binary search of off[0..ndom]).
__device__ __forceinline__ int find_domain(const int* __restrict__ off, int ndom, int b)
{
    int lo = 0, hi = ndom - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(off + mid) <= b) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// The argument block of the block's domain, copied once into shared memory (every thread of a batched CTA works on
// the same domain; reading the block from there is cheaper than a per-thread copy of ~200 bytes).  Call before any
// thread returns: it contains a block barrier.
__device__ __forceinline__ const StepArgs& block_args(const BatchDomain* __restrict__ doms, int d, StepArgs& sh)
{
    static_assert(sizeof(StepArgs) % sizeof(unsigned long long) == 0, "StepArgs is copied in 8-byte words");
    constexpr int W = sizeof(StepArgs) / sizeof(unsigned long long);
    const unsigned long long* src = reinterpret_cast<const unsigned long long*>(&doms[d].a);
    unsigned long long* dst = reinterpret_cast<unsigned long long*>(&sh);
    for (int w = threadIdx.x; w < W; w += blockDim.x) dst[w] = __ldg(src + w);
    __syncthreads();
    return sh;
}

// The FCT workspace cut into a's buffers (advect.cu).
void carve_fct_workspace(StepArgs& a, void* workspace);

// Host launchers of the batched passes (advect.cu, remap.cu).
void fct_batched_launch(const BatchDomain* doms, const int* off_dev, const int* off_host, int ndom, bool zv,
                        bool mixed, int tile_rows, cudaStream_t st);
void fct_batched_ctas(const Shape& s, int tile_rows, int& plane_ctas, int& tile_ctas);
void remap_batched_launch(const BatchDomain* doms, const int* off_dev, const int* off_host, int ndom, int nf_mode,
                          int nmax, cudaStream_t st);

}  // namespace po
