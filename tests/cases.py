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
