"""Seeded test inputs shared by the CPU and GPU tests (small enough for the
CPU checkers to finish in seconds)."""
from __future__ import annotations

import functools

import numpy as np

from trussnet_b200 import synth
from trussnet_b200.types import Nodes, RelaxParams


@functools.lru_cache(maxsize=None)
def sphere_small():
    """48^3 sphere r=18, h=2, 2-voxel lattice: ~3k nodes."""
    g, nd = synth.sphere(dim=48, radius=18.0, h=2.0, spacing=2.0, seed=1)
    return g, nd


@functools.lru_cache(maxsize=None)
def sphere64():
    """The 64^3 sphere workload (r=24, h=2, 2-voxel lattice)."""
    return synth.sphere(dim=64, radius=24.0, h=2.0, spacing=2.0, seed=0)


@functools.lru_cache(maxsize=None)
def shells_small():
    """64^3, 3 nested noisy shells, graded h in [1.5, 4]: multi-level hash, interfaces, junctions."""
    return synth.shells(dim=64, nshell=3, rmin=14.0, rmax=28.0, amp=2.0, hlo=1.5, hhi=4.0, seed=2)


@functools.lru_cache(maxsize=None)
def tpm_small():
    """40x44x36 argmax of 5 smoothed noise fields: many junctions and corners of labels."""
    return synth.tpm(shape=(40, 44, 36), nch=5, sigma=3.0, h=1.6, seed=3)


def ref_phantom(ref, dim=40):
    """Reference-built grid and seeds (build_grid_cpu + seed_cpu) of three
    nested spheres with a slab cut: interface, junction and corner seeds."""
    c = (dim - 1) / 2.0
    z, y, x = np.mgrid[0:dim, 0:dim, 0:dim].astype(np.float32)
    r = np.sqrt((x - c) ** 2 + (y - c) ** 2 + (z - c) ** 2)
    L = np.zeros((dim, dim, dim), np.uint16)
    L[r < 0.45 * dim] = 1
    L[r < 0.32 * dim] = 2
    L[(r < 0.45 * dim) & (x > c + 3)] = 3
    L[r < 0.15 * dim] = 4
    g, nd = ref.build_and_seed(L, sigma=1.0, hbase=2.5, hmin=1.5, hmax=3.0)
    return g, nd


def params(max_iters=30, **kw) -> RelaxParams:
    return RelaxParams(max_iters=max_iters, **kw)


def same_bits(a: np.ndarray, b: np.ndarray) -> bool:
    a = np.ascontiguousarray(a)
    b = np.ascontiguousarray(b)
    if a.shape != b.shape or a.dtype != b.dtype:
        return False
    return bool(np.array_equal(a.view(np.uint8), b.view(np.uint8)))


def first_diff(a: np.ndarray, b: np.ndarray):
    a = np.asarray(a).reshape(-1)
    b = np.asarray(b).reshape(-1)
    if a.dtype.kind == "f":
        d = np.nonzero(a.view(np.uint32 if a.itemsize == 4 else np.uint64) !=
                       b.view(np.uint32 if b.itemsize == 4 else np.uint64))[0]
    else:
        d = np.nonzero(a != b)[0]
    if d.size == 0:
        return None
    i = int(d[0])
    return f"{d.size} differ; first at {i}: {a[i]!r} vs {b[i]!r}"


def copy_nodes(nd: Nodes) -> Nodes:
    return nd.copy()


@functools.lru_cache(maxsize=None)
def gray_small():
    """48^3 gray-scale sphere, 2 thresholds (labels 0..2)."""
    return synth.gray_sphere(dim=48, seed=6)


# ---- shape input (analytic fields, gm < 0) ------------------------------------------
# JSON scenes for the reference's shape compiler (src/v2m_sdfshape.cpp), chosen so
# that together they reach every primitive the relaxation meets in practice and
# the program's opcodes: MCX and JMesh vocabularies, CSG (CMIN / CMAX), the
# "split" overlap rule (ADD, SCALE, CONST), per-brick programs and bounding-box
# culling (BBOX, MCONST), crease blending and gap closing.
SHAPE_SCENES = {
    "mcx": ('{"Shapes": ['
            '{"Grid": {"Tag": 0, "Size": [40, 40, 40]}},'
            '{"Sphere": {"O": [20, 20, 20], "R": 14, "Tag": 1}},'
            '{"Box": {"O": [12, 12, 17], "Size": [16, 16, 7], "Tag": 2}},'
            '{"Cylinder": {"C0": [20, 20, 3], "C1": [20, 20, 37], "R": 4, "Tag": 3}},'
            '{"Lens": {"O": [20, 20, 31], "Dir": [0, 0, 1], "R": 5, "Front": {"D": 2, "R": 8},'
            ' "Back": {"D": 2, "R": 8}, "Tag": 4}}]}',
            dict(overlap="overwrite", bricks=True, gap=0.0)),
    "jmesh": ('{"ShapeBox3": {"O": [0, 0, 0], "P": [36, 36, 36], "Tag": 1},'
              '"ShapePlane3": {"O": [0, 0, 30], "N": [0, 0.2, -1], "Tag": 5},'
              '"ShapeEllipsoid": {"O": [18, 18, 14], "R": [10, 7, 5], "Angle": [30, 20], "Tag": 2},'
              '"ShapeTorus": {"O": [18, 18, 24], "R": 9, "Rtube": 2.5, "N": [0, 0.3, 1], "Tag": 3},'
              '"ShapeConeFrustum": {"O": [6, 6, 4], "P": [6, 6, 30], "R": [4, 1.5], "Tag": 4}}',
              dict(overlap="overwrite", bricks=True, gap=0.0)),
    "csg": ('{"CSGObject": [{"CSGSubtract": [{"CSGUnion": [{"ShapeSphere": {"O": [18, 18, 18], "R": 12}},'
            '{"ShapeBox3": {"O": [8, 8, 15], "P": [28, 28, 21]}}]},'
            '{"ShapeCylinder": {"O": [18, 18, 0], "P": [18, 18, 36], "R": 4}}]}, {"Tag": 1}],'
            '"ShapeSphereShell": {"O": [18, 18, 18], "R": [6, 9], "Tag": 2}}',
            dict(overlap="overwrite", bricks=False, gap=0.0)),
    "split": ('{"Shapes": ['
              '{"Grid": {"Tag": 0, "Size": [36, 36, 36]}},'
              '{"ZSlabs": {"Bound": [[10, 20]], "Tag": 2}},'
              '{"Sphere": {"O": [14, 18, 18], "R": 9, "Tag": 3}},'
              '{"Sphere": {"O": [23, 18, 18], "R": 9, "Tag": 4}}]}',
              dict(overlap="split", bricks=True, gap=2.0)),
}


def shape_case(ref, name, exact=False):
    """A shape-input grid (gm = -1, gTW = the compiled program) and the
    reference's seeds on it. exact: crease blending off (exact CSG)."""
    scene, kw = SHAPE_SCENES[name]
    g, nd = ref.shape_and_seed(scene, voxel=1.0, hbase=2.5, hmin=1.5, hmax=3.5, **kw)
    if exact:
        g.gTW = g.gTW.copy()
        g.gTW[5 + int(g.gTW[0])] = 0.0
    return g, nd


def shape_opcodes(prog: np.ndarray):
    """The primitive types and opcodes a compiled program holds (its documented
    layout: src/opencl/v2m_sdf_body.cl:9-45), over every label's code and every
    brick's."""
    nparam = {1: 4, 2: 6, 3: 7, 4: 6, 5: 8, 6: 8, 7: 15, 8: 8, 9: 7}
    N = int(prog[0])
    starts = {int(prog[5 + l]) for l in range(N)}
    T = int(prog[8 + N])
    if T > 0:
        nb = int(prog[T]) * int(prog[T + 1]) * int(prog[T + 2])
        for b in range(nb):
            off = int(prog[T + 4 + b])
            starts.update(int(prog[off + l]) for l in range(N))
    prims, ops = set(), set()
    for pc in starts:
        while True:
            op = int(prog[pc])
            ops.add(op)
            if op == 0:
                break
            if op == 1:
                t = int(prog[pc + 1])
                prims.add(t)
                pc += 2 + nparam[t]
            elif op == 6:
                pc += 9
            elif op in (5, 7, 9):
                pc += 2
            else:
                pc += 1
    return prims, ops


# ---- seeding --------------------------------------------------------------------------
def phantom_labels(dim=40):
    """Three nested spheres with a slab cut (the ref_phantom volume)."""
    c = (dim - 1) / 2.0
    z, y, x = np.mgrid[0:dim, 0:dim, 0:dim].astype(np.float32)
    r = np.sqrt((x - c) ** 2 + (y - c) ** 2 + (z - c) ** 2)
    L = np.zeros((dim, dim, dim), np.uint16)
    L[r < 0.45 * dim] = 1
    L[r < 0.32 * dim] = 2
    L[(r < 0.45 * dim) & (x > c + 3)] = 3
    L[r < 0.15 * dim] = 4
    return L


def noise_labels(dim=36, nlab=5, seed=3):
    """argmax of smoothed seeded noise fields inside a ball: many junction lines
    and 4-label corners."""
    rng = np.random.default_rng(seed)
    f = rng.standard_normal((nlab, dim, dim, dim)).astype(np.float32)
    for _ in range(3):   # cheap smoothing: box filters along each axis
        for ax in (1, 2, 3):
            f = (np.roll(f, 1, ax) + f + np.roll(f, -1, ax)) / 3.0
    L = (np.argmax(f, axis=0) + 1).astype(np.uint16)
    c = (dim - 1) / 2.0
    z, y, x = np.mgrid[0:dim, 0:dim, 0:dim].astype(np.float32)
    L[np.sqrt((x - c) ** 2 + (y - c) ** 2 + (z - c) ** 2) > 0.46 * dim] = 0
    return L


def seed_case(ref, name, prm):
    """A reference-built grid (with its size grades) and the reference's own
    seed_cpu on it for params prm (the seeds carry part3)."""
    if name == "phantom":
        return ref.build_and_seed(phantom_labels(), sigma=1.0, hbase=2.5, hmin=1.5, hmax=3.0, prm=prm)
    if name == "noise":
        return ref.build_and_seed(noise_labels(), sigma=1.0, hbase=2.0, hmin=1.2, hmax=3.0, prm=prm)
    scene, kw = SHAPE_SCENES[name]
    return ref.shape_and_seed(scene, voxel=1.0, hbase=2.5, hmin=1.5, hmax=3.5, prm=prm, **kw)
