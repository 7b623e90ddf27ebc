"""
Seeded synthetic workloads with the shapes and value distributions of the benchmark configurations.

No dataset is involved: every field is generated from ``numpy.random.default_rng(seed)``.

* ``zstar_box`` — 64 x 64 x 20 z* C-grid, dx = dy = 1 km, 5 m layers, periodic in x, walls in y; one temperature
  field (10 / 20 degC halves plus N(0, 0.01)); non-divergent flow from a random k^-3 streamfunction scaled to
  0.5 m/s; dt at CFL 0.4; PPM_H4 remap each step from thicknesses perturbed by +-20 % back to the z* grid.
* ``basin`` — 512 x 512 x 50 curvilinear basin (2 km spacing with a smooth +-5 % perturbation), Gaussian-bump
  bathymetry in [50, 4000] m with ~15 % land, T (25 -> 4 degC) and S (34 -> 35 psu) linear in depth plus 1 degC
  Gaussian eddies, geostrophic-like eddy flow up to 1 m/s, hybrid target grid, remap from thicknesses perturbed by
  +-30 %.

Transports come from a per-layer transport streamfunction on cell corners that vanishes on every corner touching
land or a wall, so the discrete divergence of (Qx, Qy) is zero up to round-off and V1 = V0 - dt div Q stays
positive wherever the column is wet.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass
class Workload:
    name: str
    C: np.ndarray          # (nt, N, ny, nx) tracer stack
    V0: np.ndarray         # (N, ny, nx) layer volumes at the start of the step [m3]
    V1: np.ndarray         # (N, ny, nx) layer volumes at the end of the step [m3]
    Qx: np.ndarray         # (N, ny, nx+1) [m3 s-1]
    Qy: np.ndarray         # (N, ny+1, nx)
    ok: np.ndarray         # (N, ny, nx) bool
    wet: np.ndarray        # (ny, nx) bool
    h_tgt: np.ndarray      # (N, ny, nx) target thicknesses of the remap [m]
    h_src: np.ndarray      # (N, ny, nx) source (Lagrangian) thicknesses of the remap [m]
    dt: float
    periodic: tuple = ()
    open: tuple = ()
    scheme: str = "weno5"
    remap_scheme: int = 2
    meta: dict = field(default_factory=dict)

    @property
    def shape(self) -> tuple:
        return self.C.shape

    @property
    def tracer_cells(self) -> int:
        return int(np.prod(self.C.shape))


def _streamfunction_transports(psi_c: np.ndarray, h: np.ndarray, water: np.ndarray, periodic_x: bool):
    """
    Layer transports from a corner streamfunction psi_c (ny+1, nx+1) [m2 s-1] scaled by the corner thickness:
    Qx = -(Psi[j+1, i] - Psi[j, i]), Qy = Psi[j, i+1] - Psi[j, i], Psi_k = psi * h_corner * mask.
    A corner carries transport only if every cell around it is water (walls and land are closed).
    """
    n, ny, nx = h.shape
    wp = np.pad(water, 1, constant_values=False)
    hp = np.pad(h, ((0, 0), (1, 1), (1, 1)))
    if periodic_x:
        wp[1:-1, 0], wp[1:-1, -1] = water[:, -1], water[:, 0]
        hp[:, 1:-1, 0], hp[:, 1:-1, -1] = h[:, :, -1], h[:, :, 0]
    # cells around corner (j, i): (j-1, i-1), (j-1, i), (j, i-1), (j, i) -> padded (j, i), (j, i+1), (j+1, i), (j+1, i+1)
    m = wp[:-1, :-1] & wp[:-1, 1:] & wp[1:, :-1] & wp[1:, 1:]
    hc = 0.25 * (hp[:, :-1, :-1] + hp[:, :-1, 1:] + hp[:, 1:, :-1] + hp[:, 1:, 1:])
    if periodic_x:
        m[:, -1] = m[:, 0]
        hc[:, :, -1] = hc[:, :, 0]
    Psi = psi_c[None] * hc * m[None]
    Qx = -(Psi[:, 1:, :] - Psi[:, :-1, :])          # (n, ny, nx+1)
    Qy = Psi[:, :, 1:] - Psi[:, :, :-1]             # (n, ny+1, nx)
    return Qx, Qy


def _smooth_noise(rng, shape, scale: float) -> np.ndarray:
    """Zero-mean field of unit max amplitude, smooth on ``scale`` cells (sum of random cosine modes)."""
    ny, nx = shape
    y, x = np.mgrid[0:ny, 0:nx]
    out = np.zeros(shape)
    for _ in range(12):
        kx, ky = rng.normal(0, 1.0 / scale, 2)
        out += np.cos(2 * np.pi * (kx * x + ky * y) + rng.uniform(0, 2 * np.pi))
    return out / np.abs(out).max()


def zstar_box(seed: int = 0, nx: int = 64, ny: int = 64, n: int = 20, nt: int = 1) -> Workload:
    """The z* box; ``nt`` tracers, each 10 / 20 degC halves in x plus its own N(0, 0.01) noise."""
    rng = np.random.default_rng(seed)
    dx = dy = 1000.0
    h0 = 5.0
    h = np.full((n, ny, nx), h0)
    area = dx * dy
    # k^-3 streamfunction on corners: walls at j = 0 and j = ny (psi = 0), periodic in x.  Mode (m, kk) is
    # k^-3 sin(pi m y) cos(2 pi kk x + phase), k = hypot(m / 2, kk); summed as an outer product over m.
    m = np.arange(1, 9)[:, None]
    kk = np.arange(-8, 9)[None, :]
    phase = rng.uniform(0, 2 * np.pi, (8, 17))
    amp = np.hypot(m / 2.0, kk) ** -3
    ic = np.arange(nx + 1) / nx
    jc = np.arange(ny + 1) / ny
    gx = np.einsum("mk,mki->mi", amp, np.cos(2 * np.pi * kk[..., None] * ic[None, None] + phase[..., None]))
    psi = np.sin(np.pi * m * jc[None]).T @ gx
    psi[:, -1] = psi[:, 0]
    water = np.ones((ny, nx), bool)
    # uniform layers: every layer carries the same transport, computed once and repeated
    Qx, Qy = _streamfunction_transports(psi, h[:1], water, periodic_x=True)
    umax = max(np.abs(Qx).max() / (dy * h0), np.abs(Qy).max() / (dx * h0))
    scale = 0.5 / umax
    Qx *= scale
    Qy *= scale
    Qx[..., -1] = Qx[..., 0]
    dt = 0.4 * dx / 0.5
    V0 = area * h
    div = Qx[..., 1:] - Qx[..., :-1] + Qy[:, 1:] - Qy[:, :-1]
    V1 = V0 - dt * div
    ok = V1 > 0
    Qx, Qy = np.repeat(Qx, n, axis=0), np.repeat(Qy, n, axis=0)
    halves = np.where(np.arange(nx)[None, None, :] < nx // 2, 10.0, 20.0)
    C = np.stack([halves + rng.normal(0, 0.01, (n, ny, nx)) for _ in range(nt)])
    h_src = h * (1 + rng.uniform(-0.2, 0.2, h.shape))
    h_src *= h.sum(0) / h_src.sum(0)
    return Workload(f"zstar_box_{nx}x{ny}x{n}" + (f"_nt{nt}" if nt != 1 else ""), C, V0, V1, Qx, Qy, ok, water,
                    h.copy(), h_src, dt, periodic=("x",), meta=dict(dx=dx, dy=dy, cfl=0.4, umax=0.5))


def uneven_domain_sizes(seed: int = 0, ndom: int = 64, lo: int = 96, hi: int = 384, nzs=(30, 50, 75),
                        nt: int = 1) -> list:
    """(seed, nx, ny, nz, nt) of ``ndom`` independent z* boxes: nx, ny log-uniform in [lo, hi], nz drawn from
    ``nzs``, domain d seeded with seed * 1000 + d (the batched uneven-domains configuration: 64 domains, 96..384,
    nz in {30, 50, 75})."""
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(lo), np.log(hi), (ndom, 2))).round().astype(int)
    nz = rng.choice(np.asarray(nzs), ndom)
    return [(seed * 1000 + d, int(sizes[d, 0]), int(sizes[d, 1]), int(nz[d]), nt) for d in range(ndom)]


def uneven_domains(seed: int = 0, ndom: int = 64, lo: int = 96, hi: int = 384, nzs=(30, 50, 75), nt: int = 1,
                   threads: int = 8):
    """Iterator over the ``ndom`` z* boxes of ``uneven_domain_sizes`` (generated ``threads`` at a time), so
    that a caller moving each to the GPU holds only a few on the host at once."""
    from concurrent.futures import ThreadPoolExecutor
    specs = uneven_domain_sizes(seed, ndom, lo, hi, nzs, nt)
    with ThreadPoolExecutor(max(1, threads)) as ex:
        for i in range(0, len(specs), max(1, threads)):
            futs = [ex.submit(lambda a: zstar_box(seed=a[0], nx=a[1], ny=a[2], n=a[3], nt=a[4]), sp)
                    for sp in specs[i:i + max(1, threads)]]
            for f in futs:
                yield f.result()


def hybrid_target(H: np.ndarray, n: int) -> np.ndarray:
    """Hybrid target thicknesses (n, ny, nx), bed first: z-like 10 m layers near the surface where the depth allows,
    stretched layers below, sigma in shallow water; zero thickness on land (H = 0)."""
    ny, nx = H.shape
    ntop = n // 2
    top = np.minimum(10.0, H / n)                    # shallow water: sigma
    rest = np.maximum(H - ntop * top, 0.0)
    w = np.linspace(2.0, 1.0, n - ntop)              # thicker layers toward the bed
    w /= w.sum()
    h = np.empty((n, ny, nx))
    h[: n - ntop] = w[:, None, None] * rest[None]
    h[n - ntop:] = top[None]
    return h


def basin(seed: int = 0, nx: int = 512, ny: int = 512, n: int = 50, nt: int = 2, passive: str = "uniform") -> Workload:
    """The curvilinear basin.  Tracers: T, S, then nt - 2 passive ones — uniform noise in [0, 1] (``passive=
    "uniform"``) or sharp top-hat patches of 1 in a field of 0 (``passive="tophat"``, the limiter stress test of
    the 1024 x 1024 x 75 mixed-precision configuration)."""
    rng = np.random.default_rng(seed)
    dx = 2000.0 * (1 + 0.05 * _smooth_noise(rng, (ny, nx), 64.0))
    dy = 2000.0 * (1 + 0.05 * _smooth_noise(rng, (ny, nx), 64.0))
    area = dx * dy
    # Gaussian-bump bathymetry in [50, 4000] m, land where it is shallowest (~15 %)
    y, x = np.mgrid[0:ny, 0:nx]
    bump = np.zeros((ny, nx))
    for _ in range(40):
        cx, cy = rng.uniform(0, nx), rng.uniform(0, ny)
        r = rng.uniform(0.03, 0.15) * nx
        bump += rng.uniform(-1, 1) * np.exp(-((x - cx) ** 2 + (y - cy) ** 2) / (2 * r * r))
    bump = (bump - bump.min()) / (bump.max() - bump.min())
    H = 50.0 + 3950.0 * bump
    water = H > np.quantile(H, 0.15)
    water[0, :] = water[-1, :] = water[:, 0] = water[:, -1] = False       # closed basin
    H = np.where(water, H, 0.0)
    h = hybrid_target(H, n)
    # geostrophic-like eddies: streamfunction of Gaussian eddies on corners
    yc, xc = np.mgrid[0:ny + 1, 0:nx + 1]
    psi = np.zeros((ny + 1, nx + 1))
    for _ in range(60):
        cx, cy = rng.uniform(0, nx), rng.uniform(0, ny)
        r = rng.uniform(8, 40)
        psi += rng.uniform(-1, 1) * r * np.exp(-((xc - cx) ** 2 + (yc - cy) ** 2) / (2 * r * r))
    dyf = np.concatenate([dy[:, :1], 0.5 * (dy[:, 1:] + dy[:, :-1]), dy[:, -1:]], axis=1)
    dxf = np.concatenate([dx[:1], 0.5 * (dx[1:] + dx[:-1]), dx[-1:]], axis=0)
    Qx, Qy = _streamfunction_transports(psi, h, water, periodic_x=False)
    hx = np.concatenate([h[..., :1], 0.5 * (h[..., 1:] + h[..., :-1]), h[..., -1:]], axis=-1)
    hy = np.concatenate([h[:, :1], 0.5 * (h[:, 1:] + h[:, :-1]), h[:, -1:]], axis=1)
    with np.errstate(divide="ignore", invalid="ignore"):
        ux = np.where(hx > 0, np.abs(Qx) / (dyf[None] * hx), 0.0)
        vy = np.where(hy > 0, np.abs(Qy) / (dxf[None] * hy), 0.0)
    scale = 1.0 / max(ux.max(), vy.max())
    Qx *= scale
    Qy *= scale
    dt = 0.4 * 2000.0 * 0.95 / 1.0
    V0 = area[None] * h
    div = Qx[..., 1:] - Qx[..., :-1] + Qy[:, 1:] - Qy[:, :-1]
    V1 = V0 - dt * div
    ok = water[None] & (V1 > 0)
    # T 25 -> 4 degC and S 34 -> 35 psu linear in depth (bed first), plus 1 degC Gaussian eddies on T
    zc = np.cumsum(h, axis=0) - 0.5 * h                  # height of the cell centre above the bed
    depth = H[None] - zc
    frac = np.where(H[None] > 0, np.clip(depth / 4000.0, 0, 1), 0.0)
    eddy = np.zeros((ny, nx))
    for _ in range(30):
        cx, cy = rng.uniform(0, nx), rng.uniform(0, ny)
        r = rng.uniform(5, 30)
        eddy += rng.choice([-1.0, 1.0]) * np.exp(-((x - cx) ** 2 + (y - cy) ** 2) / (2 * r * r))
    T = 25.0 - 21.0 * frac + np.clip(eddy, -1, 1)[None]
    S = 34.0 + 1.0 * frac
    extra = []
    for _ in range(max(0, nt - 2)):
        if passive == "tophat":
            f = np.zeros((ny, nx))
            for _ in range(6):
                cx, cy = rng.uniform(0.1, 0.9) * nx, rng.uniform(0.1, 0.9) * ny
                r = rng.uniform(0.03, 0.1) * nx
                f[(x - cx) ** 2 + (y - cy) ** 2 < r * r] = 1.0
            k0, k1 = sorted(rng.integers(0, n, 2))
            g = np.zeros((n, ny, nx))
            g[k0:k1 + 1] = f
            extra.append(g)
        else:
            extra.append(rng.uniform(0, 1, T.shape))
    stack = [T, S] + extra
    C = np.stack(stack[:nt])
    h_src = h * (1 + rng.uniform(-0.3, 0.3, h.shape))
    col = h_src.sum(0)
    h_src *= np.where(col > 0, h.sum(0) / np.where(col > 0, col, 1.0), 0.0)[None]
    return Workload(f"basin_{nx}x{ny}x{n}_nt{nt}", C, V0, V1, Qx, Qy, ok, water, h, h_src, dt,
                    meta=dict(land_frac=float(1 - water.mean()), umax=1.0))


def algorithmic_bytes(w: Workload) -> dict:
    """Compulsory HBM bytes of one step (each input read once, each output written once): advect_fct reads C, V0,
    V1, Qx, Qy, ok and writes C_out; the remap reads h_src, h_tgt, wet, the stack and writes it."""
    nt, n, ny, nx = w.C.shape
    cells = n * ny * nx
    adv = cells * (16 * nt + 8 + 8 + 1) + 8 * n * ny * (nx + 1) + 8 * n * (ny + 1) * nx
    rem = cells * (16 + 16 * nt) + ny * nx
    return dict(advect=adv, remap=rem, step=adv + rem)


def zstar_box_device(seed: int, nx: int, ny: int, n: int, nt: int, device) -> dict:
    """The z* box of ``zstar_box`` generated on the GPU with torch's CUDA generator (same construction, another
    random stream): the inputs of a served job, built where they are used.  Returns device tensors C, V0, V1, Qx,
    Qy, ok (uint8), h_src, h_tgt, wet (uint8) and the scalars dt, flags (periodic in x), remap_scheme."""
    import torch
    f64 = dict(dtype=torch.float64, device=device)
    gen = torch.Generator(device=device)
    gen.manual_seed(int(seed))
    dx = dy = 1000.0
    h0 = 5.0
    m = torch.arange(1, 9, **f64)[:, None]
    kk = torch.arange(-8, 9, **f64)[None, :]
    phase = torch.rand((8, 17), generator=gen, **f64) * (2 * np.pi)
    amp = torch.hypot(m / 2.0, kk) ** -3
    ic = torch.arange(nx + 1, **f64) / nx
    jc = torch.arange(ny + 1, **f64) / ny
    gx = torch.einsum("mk,mki->mi", amp, torch.cos(2 * np.pi * kk[..., None] * ic[None, None] + phase[..., None]))
    psi = torch.sin(np.pi * m * jc[None]).T @ gx
    psi[:, -1] = psi[:, 0]
    # all water, walls at j = 0 and j = ny: corners on the walls carry no transport; uniform h0 layers
    Psi = psi * h0
    Psi[0] = 0.0
    Psi[-1] = 0.0
    Qx = -(Psi[1:] - Psi[:-1])                         # (ny, nx+1)
    Qy = Psi[:, 1:] - Psi[:, :-1]                      # (ny+1, nx)
    umax = max(float(Qx.abs().max()) / (dy * h0), float(Qy.abs().max()) / (dx * h0))
    Qx *= 0.5 / umax
    Qy *= 0.5 / umax
    Qx[:, -1] = Qx[:, 0]
    dt = 0.4 * dx / 0.5
    V0 = torch.full((n, ny, nx), dx * dy * h0, **f64)
    div = Qx[:, 1:] - Qx[:, :-1] + Qy[1:] - Qy[:-1]
    V1 = V0 - dt * div[None]
    ok = (V1 > 0).to(torch.uint8)
    halves = torch.where(torch.arange(nx, device=device) < nx // 2, 10.0, 20.0).to(torch.float64)
    C = halves + 0.01 * torch.randn((nt, n, ny, nx), generator=gen, **f64)
    h = torch.full((n, ny, nx), h0, **f64)
    h_src = h * (1 + 0.4 * (torch.rand((n, ny, nx), generator=gen, **f64) - 0.5))
    h_src *= h.sum(0) / h_src.sum(0)
    return dict(C=C, V0=V0, V1=V1, Qx=Qx[None].expand(n, -1, -1).contiguous(),
                Qy=Qy[None].expand(n, -1, -1).contiguous(), ok=ok, h_src=h_src, h_tgt=h,
                wet=torch.ones((ny, nx), dtype=torch.uint8, device=device), dt=dt, flags=0x10, remap_scheme=2)
