"""Seeded synthetic inputs for the relaxation: label volumes, their brick-sparse
smooth fields, sizing fields and lattice seeds.

The reference builds these with build_grid_cpu (src/v2m_grid.cpp) and seed_cpu
(src/v2m_particles.cpp:624-700) of fangq/trussnet. Here they are only the
relaxation's *inputs*: the layout is the reference's (8^3 bricks listing the
labels within R voxels, ascending, 0xFFFF padded, V2M_BL+1 on overflow; one
slot of 512 smoothed-indicator values per (mixed brick, label), in brick then
label order: src/v2m_grid.cpp:109-146), the values come from numpy/scipy
(Gaussian-smoothed label indicators, sigma 1, radius ceil(3 sigma), the outside
of the grid counting as label 0: src/v2m_grid_body.cl:80-106). Both the CUDA
path and the CPU checkers read the same arrays.

Workloads (sizes as named):
  sphere64     64^3 sphere r=24 (label 1), h = 2, 2-voxel lattice + jitter
  shells256    256^3 six nested noisy ellipsoidal shells, h in [1.5, 6] graded by
               the distance to the nearest interface (gradient 0.3), ~1M nodes
  tpm182       182x218x182, argmax of 6 Gaussian-smoothed (sigma 4) noise fields,
               channel 0 = outside, ~3M nodes
  ellipsoids128  128^3, 4 labels (nested ellipsoids), ~150k nodes
  batch64      64 volumes 32^3..160^3 with 2..18 nested shells, ~4M nodes in all
"""
from __future__ import annotations

import math

import numpy as np
from scipy import ndimage

from .types import V2M_BL, V2M_BS, V2M_INTERIOR, V2M_NOLAB, V2M_SLOT, Grid, Nodes, RelaxParams


# ---------------------------------------------------------------------------
# fields
def value_noise(shape, cells, octaves, rng, persistence=0.5):
    """Seeded multi-octave value noise in about [-1, 1] on a grid of `shape`
    (z, y, x): random lattice values, `cells` cells per axis at the first octave,
    doubled each octave, trilinearly interpolated (scipy zoom, order 1)."""
    out = np.zeros(shape, np.float32)
    amp, tot = 1.0, 0.0
    for o in range(octaves):
        c = cells * (2 ** o)
        lat = rng.uniform(-1.0, 1.0, size=(c + 1, c + 1, c + 1)).astype(np.float32)
        zoom = [(s - 1) / c + 1e-9 for s in shape]
        f = ndimage.zoom(lat, [shape[i] / (c + 1) for i in range(3)], order=1, mode="nearest", grid_mode=True)
        f = f[: shape[0], : shape[1], : shape[2]]
        pad = [(0, shape[i] - f.shape[i]) for i in range(3)]
        f = np.pad(f, pad, mode="edge")
        out += amp * f
        tot += amp
        amp *= persistence
        del zoom
    return out / tot


def _gauss_weights(sigma, R):
    d = np.arange(-R, R + 1, dtype=np.float32)
    w = np.exp(-0.5 * d * d / (sigma * sigma)).astype(np.float32)
    return w / w.sum()


def build_grid(L: np.ndarray, h: np.ndarray, hmin: float, hmax: float, vs=(1.0, 1.0, 1.0), sigma: float = 1.0,
               R: int = 6) -> Grid:
    """Brick-sparse smooth fields of label volume L (uint16, [nz, ny, nx]).

    Bricks list the labels within R voxels (src/v2m_grid_body.cl:28-69); mixed
    bricks get one slot per label holding the Gaussian-smoothed indicator."""
    L = np.ascontiguousarray(L, dtype=np.uint16)
    nz, ny, nx = L.shape
    nbx, nby, nbz = [(n + V2M_BS - 1) // V2M_BS for n in (nx, ny, nz)]
    nb = nbx * nby * nbz
    labels = np.unique(L)
    # labels present in each brick's R-dilated box (outside the grid = 0)
    pad_lo = R
    pad_hi = nbx * V2M_BS - nx + R + 1, nby * V2M_BS - ny + R + 1, nbz * V2M_BS - nz + R + 1
    present = []
    lab_set = sorted(set(int(x) for x in labels) | {0})
    for l in lab_set:
        ind = np.pad((L == l).astype(np.int32), ((pad_lo, pad_hi[2]), (pad_lo, pad_hi[1]), (pad_lo, pad_hi[0])),
                     mode="constant", constant_values=1 if l == 0 else 0)
        win = V2M_BS + 2 * R + 1
        a = ind
        for ax, nbax in ((2, nbx), (1, nby), (0, nbz)):
            cs = np.cumsum(a, axis=ax, dtype=np.int32)
            cs = np.concatenate([np.zeros_like(np.take(cs, [0], axis=ax)), cs], axis=ax)
            starts = np.arange(nbax) * V2M_BS
            a = np.take(cs, starts + win, axis=ax) - np.take(cs, starts, axis=ax)
        present.append(a > 0)                       # [nbz, nby, nbx]
    present = np.stack(present, axis=-1).reshape(nb, len(lab_set))
    cnt = present.sum(axis=1).astype(np.int32)
    bl_lab = np.full((nb, V2M_BL), V2M_NOLAB, np.uint16)
    lab_arr = np.array(lab_set, np.uint16)
    for b in np.nonzero(cnt)[0]:
        ls = lab_arr[present[b]][:V2M_BL]
        bl_lab[b, : ls.size] = ls
    bl_cnt = np.where(cnt > V2M_BL, V2M_BL + 1, cnt).astype(np.int32)
    mixed = np.minimum(bl_cnt, V2M_BL) >= 2
    nper = np.where(mixed, np.minimum(bl_cnt, V2M_BL), 0)
    first = np.concatenate([[0], np.cumsum(nper)[:-1]]).astype(np.int64)
    bl_slot = np.where(mixed, first, -1).astype(np.int32)
    nslots = int(nper.sum())
    phi = np.zeros((nslots, V2M_SLOT), np.float32)
    # smoothed indicators, per label over the padded-to-brick volume
    Rs = min(6, max(1, int(math.ceil(3.0 * sigma))))
    w = _gauss_weights(sigma, Rs)
    mb = np.nonzero(mixed)[0]
    bz, by, bx = np.unravel_index(mb, (nbz, nby, nbx))
    for l in lab_set:
        sel = bl_lab[mb] == l
        rows, cols = np.nonzero(sel)
        if rows.size == 0:
            continue
        f = (L == l).astype(np.float32)
        cval = 1.0 if l == 0 else 0.0
        for ax in (2, 1, 0):
            f = ndimage.correlate1d(f, w, axis=ax, mode="constant", cval=cval, output=np.float32)
        fp = np.zeros((nbz * V2M_BS, nby * V2M_BS, nbx * V2M_BS), np.float32)
        fp[:nz, :ny, :nx] = f
        blocks = fp.reshape(nbz, V2M_BS, nby, V2M_BS, nbx, V2M_BS).transpose(0, 2, 4, 1, 3, 5)
        blk = blocks[bz[rows], by[rows], bx[rows]]          # [m, 8(z), 8(y), 8(x)]
        phi[first[mb[rows]] + cols] = blk.reshape(-1, V2M_SLOT)
    return Grid(nx=nx, ny=ny, nz=nz, vs=tuple(float(v) for v in vs), L=L, bl_cnt=bl_cnt,
                bl_lab=np.ascontiguousarray(bl_lab.reshape(-1)), bl_slot=bl_slot,
                phi=np.ascontiguousarray(phi.reshape(-1)), h=np.ascontiguousarray(h, dtype=np.float32),
                hmin=float(hmin), hmax=float(hmax), R=R)


def interface_distance(L: np.ndarray) -> np.ndarray:
    """Euclidean distance (voxels) to the nearest voxel face between two labels."""
    m = np.zeros(L.shape, bool)
    for ax in range(3):
        d = np.diff(L.astype(np.int32), axis=ax) != 0
        sl_lo = [slice(None)] * 3
        sl_hi = [slice(None)] * 3
        sl_lo[ax] = slice(0, -1)
        sl_hi[ax] = slice(1, None)
        m[tuple(sl_lo)] |= d
        m[tuple(sl_hi)] |= d
    if not m.any():
        return np.full(L.shape, 1e3, np.float32)
    return ndimage.distance_transform_edt(~m).astype(np.float32)


# ---------------------------------------------------------------------------
# seeds
def seed_lattice(L: np.ndarray, h: np.ndarray, rng, density: float = 1.0, levels: int = 6, jitter: float = 0.25,
                 hmin: float | None = None, hmax: float | None = None, vs=(1.0, 1.0, 1.0)) -> Nodes:
    """Jittered cubic lattices graded by h: level j has spacing s_j (geometric
    from hmin to hmax, divided by density); a level-j point is kept where the
    voxel under it is non-zero and its h falls in level j. Nodes are INTERIOR
    with the voxel's label, in voxel (raster) order like the reference's seeds."""
    nz, ny, nx = L.shape
    hmin = float(h.min()) if hmin is None else hmin
    hmax = float(h.max()) if hmax is None else hmax
    if hmax <= hmin * 1.0001:
        edges = np.array([-np.inf, np.inf])
        sp = np.array([hmin])
    else:
        sp = np.geomspace(hmin, hmax, levels)
        mids = np.sqrt(sp[:-1] * sp[1:])
        edges = np.concatenate([[-np.inf], mids, [np.inf]])
    lev = np.searchsorted(edges, h, side="right") - 1
    pts = []
    for j, s in enumerate(sp):
        s = s / density
        ax = [np.arange(0.5 * s, n * v - 0.5 * v, s) - 0.5 * v for n, v in zip((nx, ny, nz), vs)]
        if min(a.size for a in ax) == 0:
            continue
        zz, yy, xx = np.meshgrid(ax[2], ax[1], ax[0], indexing="ij")
        p = np.stack([xx.ravel(), yy.ravel(), zz.ravel()], axis=1).astype(np.float32)
        p += rng.uniform(-jitter * s, jitter * s, size=p.shape).astype(np.float32)
        ijk = np.floor(p / np.array(vs, np.float32) + 0.5).astype(np.int64)
        ok = np.all((ijk >= 0) & (ijk < np.array([nx, ny, nz])), axis=1)
        p, ijk = p[ok], ijk[ok]
        lab = L[ijk[:, 2], ijk[:, 1], ijk[:, 0]]
        keep = (lab != 0) & (lev[ijk[:, 2], ijk[:, 1], ijk[:, 0]] == j)
        pts.append((p[keep], lab[keep], ijk[keep]))
    P = np.concatenate([a for a, _, _ in pts]).astype(np.float32)
    lab = np.concatenate([b for _, b, _ in pts]).astype(np.uint16)
    ijk = np.concatenate([c for _, _, c in pts])
    vox = ijk[:, 0] + nx * (ijk[:, 1] + ny * ijk[:, 2])
    order = np.argsort(vox, kind="stable")
    n = order.size
    return Nodes(P=np.ascontiguousarray(P[order]), lab=np.ascontiguousarray(lab[order]),
                 typ=np.full(n, V2M_INTERIOR, np.uint8), part=np.full((n, 2), V2M_NOLAB, np.uint16))


# ---------------------------------------------------------------------------
# workloads
def sphere(dim=64, radius=24.0, h=2.0, spacing=2.0, seed=0):
    """Label-1 sphere of `radius` voxels centred in a dim^3 grid; h uniform;
    nodes on a `spacing`-voxel lattice inside the label with uniform jitter."""
    rng = np.random.default_rng(seed)
    c = (dim - 1) / 2.0
    z, y, x = np.mgrid[0:dim, 0:dim, 0:dim].astype(np.float32)
    L = (((x - c) ** 2 + (y - c) ** 2 + (z - c) ** 2) < radius * radius).astype(np.uint16)
    hf = np.full(L.shape, h, np.float32)
    g = build_grid(L, hf, h, h)
    nd = seed_lattice(L, hf, rng, density=h / spacing, hmin=h, hmax=h)
    return g, nd


def nested_shells(dim, nshell, rmin, rmax, amp, rng, axes=(1.0, 0.9, 0.8), octaves=4):
    """Label = number of nested ellipsoids (semi-axes r_k * axes, r_k from rmin
    to rmax) containing the voxel, each radius perturbed by the same seeded
    low-frequency value noise of amplitude `amp` voxels (so shells stay nested)."""
    dims = (dim, dim, dim) if np.isscalar(dim) else tuple(dim)
    nz, ny, nx = dims[2], dims[1], dims[0]
    noise = value_noise((nz, ny, nx), 2, octaves, rng)
    cz, cy, cx = (nz - 1) / 2.0, (ny - 1) / 2.0, (nx - 1) / 2.0
    z, y, x = np.ogrid[0:nz, 0:ny, 0:nx]
    rho = np.sqrt(((x - cx) / axes[0]) ** 2 + ((y - cy) / axes[1]) ** 2 + ((z - cz) / axes[2]) ** 2).astype(np.float32)
    rk = np.linspace(rmin, rmax, nshell) if nshell > 1 else np.array([rmax])
    L = np.zeros((nz, ny, nx), np.uint16)
    for r in rk:
        L += (rho < r + amp * noise).astype(np.uint16)
    return L


def shells(dim=256, nshell=6, rmin=60.0, rmax=120.0, amp=6.0, hlo=1.5, hhi=6.0, grad=0.3, density=1.18, seed=0):
    """Six nested noisy ellipsoidal shells; h = clamp(hlo + grad * distance to
    the nearest interface, hlo, hhi)."""
    rng = np.random.default_rng(seed)
    L = nested_shells(dim, nshell, rmin, rmax, amp, rng)
    dist = interface_distance(L)
    hf = np.clip(hlo + grad * dist, hlo, hhi).astype(np.float32)
    g = build_grid(L, hf, hlo, hhi)
    nd = seed_lattice(L, hf, rng, density=density, hmin=hlo, hmax=hhi)
    return g, nd


def size_grades(h: np.ndarray, hmin: float, hmax: float) -> np.ndarray:
    """Per-voxel size grades (tn::Grid::grade, the seeding's input): h mapped
    logarithmically onto 0..255 over [hmin, hmax]."""
    if not hmax > hmin:
        return np.zeros(h.shape, np.uint8)
    t = np.log(np.maximum(h, hmin) / hmin) / np.log(hmax / hmin)
    return np.clip(np.rint(255.0 * t), 0, 255).astype(np.uint8)


def tpm(shape=(182, 218, 182), nch=6, sigma=4.0, h=1.3, density=1.0, seed=0):
    """Argmax of `nch` Gaussian-smoothed (sigma voxels) seeded noise fields (the
    labels of a tissue-probability map whose softmax at any temperature has the
    same argmax); channel 0 is the outside."""
    rng = np.random.default_rng(seed)
    nx, ny, nz = shape
    best = None
    L = np.zeros((nz, ny, nx), np.uint16)
    for c in range(nch):
        f = rng.standard_normal((nz, ny, nx)).astype(np.float32)
        f = ndimage.gaussian_filter(f, sigma, mode="reflect", truncate=3.0, output=np.float32)
        if best is None:
            best = f
        else:
            m = f > best
            L[m] = c
            best = np.where(m, f, best)
    hf = np.full(L.shape, h, np.float32)
    g = build_grid(L, hf, h, h)
    nd = seed_lattice(L, hf, rng, density=density, hmin=h, hmax=h)
    return g, nd


def ellipsoids(dim=128, nlab=4, h=(1.5, 4.0), density=1.0, seed=0):
    """Nested ellipsoids with `nlab` labels (0 outside) and a smooth noise size
    field in [h0, h1]."""
    rng = np.random.default_rng(seed)
    L = nested_shells(dim, nlab - 1, 0.22 * dim, 0.44 * dim, 0.04 * dim, rng)
    noise = value_noise(L.shape, 2, 3, rng)
    hf = (h[0] + (h[1] - h[0]) * 0.5 * (noise / max(1e-6, float(np.abs(noise).max())) + 1.0)).astype(np.float32)
    g = build_grid(L, hf, h[0], h[1])
    nd = seed_lattice(L, hf, rng, density=density, hmin=h[0], hmax=h[1])
    return g, nd


def batch(nvol=64, seed=0, dmin=32, dmax=160, lmin=2, lmax=18, scale=1.55):
    """`nvol` independent volumes of seeded sizes dmin^3..dmax^3 with lmin..lmax
    nested-shell labels: the outer shell at 0.45 dim, the others 4 voxels apart
    inwards (radius at least 4), shell noise 0.02 dim; h graded from 1.0 to 4.0
    times `scale` by the distance to the nearest interface."""
    rng = np.random.default_rng(seed)
    out = []
    for v in range(nvol):
        dim = int(rng.integers(dmin, dmax + 1))
        nl = int(rng.integers(lmin, lmax + 1))
        nshell = nl - 1
        rmax = 0.45 * dim
        rmin = max(4.0, rmax - (nshell - 1) * 4.0) if nshell > 1 else rmax
        L = nested_shells(dim, nshell, rmin, rmax, 0.02 * dim, rng)
        dist = interface_distance(L)
        hlo = 1.0 * scale
        hf = np.clip(hlo + 0.3 * dist, hlo, 4.0 * scale).astype(np.float32)
        g = build_grid(L, hf, hlo, 4.0 * scale)
        nd = seed_lattice(L, hf, rng, density=1.0, hmin=hlo, hmax=4.0 * scale)
        out.append((g, nd))
    return out


def params_for(name: str) -> RelaxParams:
    """Relaxation parameters of each workload (reference defaults otherwise)."""
    if name == "sphere64":
        # 200 FP32 iterations, step dt = 0.2 (FIRE's first step sqrt(0.2)), no early stop, and a
        # fixed edge list: the first build's truss lists for the whole run (rebuild_policy 2)
        return RelaxParams(max_iters=200, dt=0.2, dptol=0.0, rebuild_policy=2)
    if name == "shells256":
        return RelaxParams(max_iters=500, dptol=0.0)
    if name == "tpm182":
        return RelaxParams(max_iters=300, dptol=0.0)
    if name == "ellipsoids128":
        return RelaxParams(max_iters=50, dptol=0.0, fire=False)
    if name == "batch64":
        return RelaxParams(max_iters=200, dptol=0.0)
    raise KeyError(name)


WORKLOADS = {
    "sphere64": lambda **kw: sphere(**kw),
    "shells256": lambda **kw: shells(**kw),
    "tpm182": lambda **kw: tpm(**kw),
    "ellipsoids128": lambda **kw: ellipsoids(**kw),
}


def gray_sphere(dim=48, seed=0, thresholds=(0.3, 0.6), widths=(0.2, 0.2), h=2.0, spacing=2.0):
    """Gray-scale input (tn::Grid gI / gTW / gm, src/v2m_grid.h:70-73): a smooth
    radial intensity with seeded noise; label = number of thresholds <= I; the
    interfaces are the iso-surfaces I = t_k."""
    rng = np.random.default_rng(seed)
    c = (dim - 1) / 2.0
    z, y, x = np.mgrid[0:dim, 0:dim, 0:dim].astype(np.float32)
    r = np.sqrt((x - c) ** 2 + (y - c) ** 2 + (z - c) ** 2) / (0.45 * dim)
    I = (1.0 - r + 0.05 * value_noise((dim, dim, dim), 2, 2, rng)).astype(np.float32)
    t = np.asarray(thresholds, np.float32)
    L = np.zeros(I.shape, np.uint16)
    for tk in t:
        L += (I >= tk).astype(np.uint16)
    hf = np.full(L.shape, h, np.float32)
    g = build_grid(L, hf, h, h)
    g.gI = np.ascontiguousarray(I.reshape(-1))
    g.gTW = np.concatenate([t, np.asarray(widths, np.float32)]).astype(np.float32)
    g.gm = int(t.size)
    nd = seed_lattice(L, hf, rng, density=h / spacing, hmin=h, hmax=h)
    return g, nd


def sizing_grid(shape=(64, 64, 64), lo=1.5, hi=4.0, seed=0):
    """A seeded smooth sizing grid G [m2, m1, m0] (x fastest) with values in [lo, hi]."""
    rng = np.random.default_rng(seed)
    nz = value_noise(tuple(shape[::-1]), 2, 3, rng)
    nz = (nz - nz.min()) / max(1e-12, float(nz.max() - nz.min()))
    return (lo + (hi - lo) * nz).astype(np.float32)


def sample_sizing(G: np.ndarray, cs, dims) -> np.ndarray:
    """G interpolated trilinearly at every voxel centre of a (nx, ny, nz) grid (x fastest)."""
    nx, ny, nz = dims
    m = G.shape[::-1]
    coords = []
    for n, c, mm in zip((nz, ny, nx), (cs[2], cs[1], cs[0]), (m[2], m[1], m[0])):
        coords.append(np.clip(np.arange(n) / c, 0, mm - 1))
    zz, yy, xx = np.meshgrid(*coords, indexing="ij")
    return ndimage.map_coordinates(G.astype(np.float64), [zz, yy, xx], order=1, mode="nearest").astype(np.float32)


def ellipsoids_adjoint(dim=128, m=64, nlab=4, lo=1.5, hi=4.0, density=1.66, seed=0):
    """The adjoint workload: nested ellipsoids (nlab labels) in a dim^3 volume,
    a seeded m^3 sizing grid in [lo, hi] spanning the volume (cell (dim-1)/(m-1)),
    the per-voxel h sampled from it, and lattice seeds graded by it."""
    rng = np.random.default_rng(seed)
    L = nested_shells(dim, nlab - 1, 0.22 * dim, 0.44 * dim, 0.04 * dim, rng)
    G = sizing_grid((m, m, m), lo, hi, seed + 1)
    cs = ((dim - 1) / (m - 1),) * 3
    hf = sample_sizing(G, cs, (dim, dim, dim))
    g = build_grid(L, hf, lo, hi)
    nd = seed_lattice(L, hf, rng, density=density, hmin=lo, hmax=hi)
    return g, nd, G, cs
