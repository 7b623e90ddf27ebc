// Batched ALE tracer steps of many independent domains: every pass of the FCT advection and the remap is one launch
// over all domains (domain d owns a contiguous range of the launch's CTAs, found by binary search of a CTA-offset
// table), so a batch of uneven domains costs 10-11 launches per step instead of 10-11 per domain, and the step
// sequence can be captured in one CUDA graph.  The batch plan (descriptors of both ping-pong parities and the
// offset tables) lives in a caller-provided device buffer; the library allocates no device memory.
#include <cstdlib>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "fct_args.cuh"

using namespace po;

struct pocean_batch {
    int ndom;
    int tile_rows;                     // rows of the 32-wide tiles of the stage passes
    int nmax;                          // deepest column of the batch
    bool zv;                           // WENO5-Z (else JS) for every domain
    BatchDomain* dev_doms;             // 2 * ndom descriptors: parity 0 then parity 1
    int* dev_off;                      // BP_COUNT * (ndom + 1) offsets
    std::vector<int> host_off;
};

extern "C" size_t pocean_batch_device_bytes(int ndom)
{
    if (ndom < 1) return 0;
    const size_t d = ((size_t)2 * ndom * sizeof(BatchDomain) + 255) & ~(size_t)255;
    return d + (size_t)BP_COUNT * (ndom + 1) * sizeof(int);
}

extern "C" int pocean_batch_create(const pocean_domain* domains, int ndom, int tile_rows, void* device_buf,
                                   size_t device_bytes, pocean_batch** out, void* stream)
{
    const char* fn = "pocean_batch_create";
    if (!out) return pocean_fail(POCEAN_EINVAL, "%s: null output handle", fn);
    *out = nullptr;
    if (ndom < 1 || !domains) return pocean_fail(POCEAN_EINVAL, "%s: no domains", fn);
    if (tile_rows != 4 && tile_rows != 8 && tile_rows != 16)
        return pocean_fail(POCEAN_EINVAL, "%s: tile rows %d (4, 8 or 16)", fn, tile_rows);
    if (!device_buf || device_bytes < pocean_batch_device_bytes(ndom) || ((uintptr_t)device_buf & 255))
        return pocean_fail(POCEAN_EWORKSPACE, "%s: device buffer of %zu bytes (256-byte aligned) needed", fn,
                           pocean_batch_device_bytes(ndom));
    int rc = pocean_check_device();
    if (rc) return rc;
    std::vector<BatchDomain> host(2 * (size_t)ndom);
    std::vector<int> off((size_t)BP_COUNT * (ndom + 1), 0);
    const bool zv = !(domains[0].flags & POCEAN_WENO_JS);
    int nmax = 1;
    long long tot[BP_COUNT] = {0, 0, 0, 0, 0, 0};
    for (int d = 0; d < ndom; ++d) {
        const pocean_domain& D = domains[d];
        if (D.nt < 1 || D.nz < 1 || D.ny < 1 || D.nx < 1 || (long long)D.nt * D.nz > 65535 || D.nz > 256)
            return pocean_fail(POCEAN_EINVAL, "%s: domain %d: bad shape nt=%d nz=%d ny=%d nx=%d", fn, d, D.nt, D.nz,
                               D.ny, D.nx);
        if ((long long)D.nz * (D.ny + 1) * (D.nx + 1) >= (1ll << 31))
            return pocean_fail(POCEAN_EINVAL, "%s: domain %d exceeds 2^31 entries per field", fn, d);
        if (!D.C || !D.V0 || !D.V1 || !D.Qx || !D.Qy || !D.ok || !D.C_adv || !D.h_src || !D.h_tgt || !D.wet ||
            !D.C_next)
            return pocean_fail(POCEAN_EINVAL, "%s: domain %d: null pointer", fn, d);
        if (D.flags & ~(unsigned)0x7F) return pocean_fail(POCEAN_EINVAL, "%s: domain %d: unknown flags", fn, d);
        if ((!(D.flags & POCEAN_WENO_JS)) != zv)
            return pocean_fail(POCEAN_EINVAL, "%s: every domain of a batch must use the same WENO variant", fn);
        if (D.remap_scheme < POCEAN_PCM || D.remap_scheme > POCEAN_PPM_H4)
            return pocean_fail(POCEAN_EINVAL, "%s: domain %d: unknown remap scheme", fn, d);
        const size_t need = pocean_advect_fct_workspace_bytes(D.nt, D.nz, D.ny, D.nx);
        if (!D.workspace || D.workspace_bytes < need || ((uintptr_t)D.workspace & 255))
            return pocean_fail(POCEAN_EWORKSPACE, "%s: domain %d: workspace of %zu bytes needed", fn, d, need);
        nmax = D.nz > nmax ? D.nz : nmax;
        for (int parity = 0; parity < 2; ++parity) {
            BatchDomain& B = host[(size_t)parity * ndom + d];
            std::memset(&B, 0, sizeof(B));
            B.a.s = Shape{D.nt, D.nz, D.ny, D.nx};
            B.a.tdiv = plane_magic(D.nt);
            B.a.flags = D.flags;
            B.a.dt = D.dt;
            B.a.C = parity == 0 ? D.C : D.C_next;
            B.a.V0 = D.V0; B.a.V1 = D.V1; B.a.Qx = D.Qx; B.a.Qy = D.Qy; B.a.ok = D.ok; B.a.inflow = D.inflow;
            B.a.Fz = nullptr;
            carve_fct_workspace(B.a, D.workspace);
            B.a.out = D.C_adv;
            B.h_src = D.h_src; B.h_tgt = D.h_tgt; B.wet = D.wet; B.remap_scheme = D.remap_scheme;
            B.rout = parity == 0 ? D.C_next : const_cast<double*>(D.C);
            int sc, tc;
            fct_batched_ctas(B.a.s, tile_rows, sc, tc);
            if (parity == 0) {
                const long long cb = ((long long)D.ny * D.nx + 127) / 128;
                const long long n_pass[BP_COUNT] = {sc, tc, cb * (D.nt / 2), cb * (D.nt % 2), cb * D.nt, cb * D.nt};
                for (int q = 0; q < BP_COUNT; ++q) {
                    off[(size_t)q * (ndom + 1) + d] = (int)tot[q];
                    tot[q] += n_pass[q];
                    if (tot[q] >= (1ll << 31))
                        return pocean_fail(POCEAN_EINVAL, "%s: batch too large for one launch", fn);
                }
            }
        }
    }
    for (int q = 0; q < BP_COUNT; ++q) off[(size_t)q * (ndom + 1) + ndom] = (int)tot[q];
    pocean_batch* b = new pocean_batch;
    b->ndom = ndom;
    b->tile_rows = tile_rows;
    b->nmax = nmax;
    b->zv = zv;
    b->dev_doms = (BatchDomain*)device_buf;
    b->dev_off = (int*)((char*)device_buf + (((size_t)2 * ndom * sizeof(BatchDomain) + 255) & ~(size_t)255));
    b->host_off = off;
    // Pageable sources: each copy is staged before the call returns, so the host vectors may go; on the device
    // the copies are ordered after the work already on `stream` (which may still read an older plan here).
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t e = cudaMemcpyAsync(b->dev_doms, host.data(), host.size() * sizeof(BatchDomain),
                                    cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(b->dev_off, off.data(), off.size() * sizeof(int), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) {
        delete b;
        return pocean_fail(POCEAN_ECUDA, "%s: %s", fn, cudaGetErrorString(e));
    }
    *out = b;
    return POCEAN_OK;
}

extern "C" int pocean_batch_step(const pocean_batch* b, int parity, int remap_nf, int mixed, void* stream)
{
    const char* fn = "pocean_batch_step";
    if (!b) return pocean_fail(POCEAN_EINVAL, "%s: null batch", fn);
    if (parity != 0 && parity != 1) return pocean_fail(POCEAN_EINVAL, "%s: parity must be 0 or 1", fn);
    if (remap_nf != 1 && remap_nf != 2) return pocean_fail(POCEAN_EINVAL, "%s: remap_nf must be 1 or 2", fn);
    cudaStream_t st = (cudaStream_t)stream;
    const BatchDomain* doms = b->dev_doms + (size_t)parity * b->ndom;
    fct_batched_launch(doms, b->dev_off, b->host_off.data(), b->ndom, b->zv, mixed != 0, b->tile_rows, st);
    remap_batched_launch(doms, b->dev_off, b->host_off.data(), b->ndom, remap_nf, b->nmax, st);
    return pocean_check_launch(fn);
}

extern "C" void pocean_batch_destroy(pocean_batch* b) { delete b; }
