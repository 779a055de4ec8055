"""Loading the golden fixtures written by tests/golden/make_golden.py."""
import glob
import os

import numpy as np

from trussnet_b200.types import Grid, Nodes, RelaxParams

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
PARAM_FIELDS = ("max_iters", "dt", "dptol", "fire", "voxel_trap")


def names():
    """The relaxation fixtures."""
    return sorted(n for n in (os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "*.npz")))
                  if not n.startswith("seed_"))


def seed_names():
    """The seeding fixtures."""
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "seed_*.npz")))


def grid_of(d):
    nx, ny, nz = (int(x) for x in d["grid_dims"])
    g = Grid(nx=nx, ny=ny, nz=nz, vs=tuple(float(v) for v in d["grid_vs"]), L=d["grid_L"], bl_cnt=d["grid_bl_cnt"],
             bl_lab=d["grid_bl_lab"], bl_slot=d["grid_bl_slot"], phi=d["grid_phi"], h=d["grid_h"],
             hmin=float(d["grid_hrange"][0]), hmax=float(d["grid_hrange"][1]))
    if "grid_gTW" in d:   # shape input: the compiled program
        g.gTW, g.gm = d["grid_gTW"], int(d["grid_gm"][0])
    if "grid_grade" in d:
        g.grade = d["grid_grade"]
    return g


def load_seed(name):
    """A seeding fixture: the grid, the parameters and seed_cpu's nodes (with part3)."""
    d = dict(np.load(os.path.join(GOLDEN, name + ".npz")))
    nseed, jseed, corners, voxel_trap = d["seed_params"]
    prm = RelaxParams(nseed=int(nseed), jseed=float(jseed), corners=bool(corners), voxel_trap=bool(voxel_trap))
    nd = Nodes(P=d["seeds_P"], lab=d["seeds_lab"], typ=d["seeds_typ"], part=d["seeds_part"])
    nd.part3 = d["seeds_part3"]
    return grid_of(d), prm, nd


def load(name):
    d = dict(np.load(os.path.join(GOLDEN, name + ".npz")))
    g = grid_of(d)
    nd = Nodes(P=d["seed_P"], lab=d["seed_lab"], typ=d["seed_typ"], part=d["seed_part"])
    vals = dict(zip(PARAM_FIELDS, d["params"]))
    prm = RelaxParams(max_iters=int(vals["max_iters"]), dt=float(vals["dt"]), dptol=float(vals["dptol"]),
                      fire=bool(vals["fire"]), voxel_trap=bool(vals["voxel_trap"]))
    # float parameters round-trip through float64 exactly; the library takes them as float
    return g, nd, prm, d
