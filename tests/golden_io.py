"""Loading the golden fixtures written by tests/golden/make_golden.py."""
import glob
import os

import numpy as np

from trussnet_b200.types import Grid, Nodes, RelaxParams

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
PARAM_FIELDS = ("max_iters", "dt", "dptol", "fire", "voxel_trap")


def names():
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "*.npz")))


def load(name):
    d = dict(np.load(os.path.join(GOLDEN, name + ".npz")))
    nx, ny, nz = (int(x) for x in d["grid_dims"])
    g = Grid(nx=nx, ny=ny, nz=nz, vs=tuple(float(v) for v in d["grid_vs"]), L=d["grid_L"], bl_cnt=d["grid_bl_cnt"],
             bl_lab=d["grid_bl_lab"], bl_slot=d["grid_bl_slot"], phi=d["grid_phi"], h=d["grid_h"],
             hmin=float(d["grid_hrange"][0]), hmax=float(d["grid_hrange"][1]))
    nd = Nodes(P=d["seed_P"], lab=d["seed_lab"], typ=d["seed_typ"], part=d["seed_part"])
    vals = dict(zip(PARAM_FIELDS, d["params"]))
    prm = RelaxParams(max_iters=int(vals["max_iters"]), dt=float(vals["dt"]), dptol=float(vals["dptol"]),
                      fire=bool(vals["fire"]), voxel_trap=bool(vals["voxel_trap"]))
    # float parameters round-trip through float64 exactly; the library takes them as float
    return g, nd, prm, d
