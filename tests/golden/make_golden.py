"""Generate the golden fixtures of the relaxation from the reference's own CPU
path (oracle/_ref/libv2m_ref.so: relax_cpu and its stages, compiled from
fangq/trussnet's sources by oracle/Makefile).

The reference ships no golden vectors for this path (its tests check
determinism and mesh conformity only), so these fixtures are outputs of the
reference itself, run here on small seeded inputs; the inputs are stored too,
so the fixtures do not depend on the generator's numpy/scipy versions.

  python tests/golden/make_golden.py [NAME ...]   (needs oracle/_ref built; default: all)

Each fixture <name>.npz holds
  grid_*            the grid arrays (v2m_grid_view) and node seeds
  key, sorted, cstart, nbr, nnb, Ps      after the first list build
  F                 after the first force pass
  it1_P, it1_typ, it1_part, it1_mv       after one whole iteration
  run_P, run_typ, run_part, run_stats    after relax_cpu with the stored parameters
  grid_gTW, grid_gm (shape input only)    the compiled shape program

and each seeding fixture seed_<name>.npz holds the grid (with grid_grade), the
seeding parameters and seed_cpu's nodes (P, lab, typ, part, part3).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

from oracle.ref import RefLib  # noqa: E402
from trussnet_b200 import synth  # noqa: E402
from trussnet_b200.types import RelaxParams  # noqa: E402
import cases as test_cases  # noqa: E402

PARAM_FIELDS = ("max_iters", "dt", "dptol", "fire", "voxel_trap")
SEED_FIELDS = ("nseed", "jseed", "corners", "voxel_trap")


def cases(ref):
    out = {}
    out["sphere24"] = synth.sphere(dim=24, radius=9.0, h=2.0, spacing=2.0, seed=11) + (
        RelaxParams(max_iters=40, dt=0.2, dptol=0.0),)
    out["tpm28"] = synth.tpm(shape=(28, 30, 26), nch=4, sigma=2.5, h=1.6, seed=12) + (RelaxParams(max_iters=30),)
    out["shells32_jacobi"] = synth.shells(dim=32, nshell=2, rmin=7.0, rmax=13.0, amp=1.0, hlo=1.5, hhi=3.0,
                                          density=1.0, seed=13) + (RelaxParams(max_iters=30, fire=False),)
    out["shells32_voxel"] = synth.shells(dim=32, nshell=2, rmin=7.0, rmax=13.0, amp=1.0, hlo=1.5, hhi=3.0,
                                         density=1.0, seed=14) + (RelaxParams(max_iters=15, voxel_trap=True),)
    # shape input: the CSG scene of the tests, compiled and seeded by the reference
    out["shape_csg"] = test_cases.shape_case(ref, "csg") + (RelaxParams(max_iters=15),)
    return out


def seed_cases(ref):
    """Seeding fixtures: a reference-built 5-label noise volume (every node kind)."""
    prm = RelaxParams()
    g, nd = test_cases.seed_case(ref, "noise", prm)
    return {"seed_noise": (g, nd, prm)}


def grid_arrays(g):
    d = {}
    for a in ("L", "bl_cnt", "bl_lab", "bl_slot", "phi", "h"):
        d["grid_" + a] = getattr(g, a)
    d["grid_dims"] = np.array([g.nx, g.ny, g.nz], np.int32)
    d["grid_vs"] = np.array(g.vs, np.float32)
    d["grid_hrange"] = np.array([g.hmin, g.hmax], np.float32)
    if g.gm < 0:
        d["grid_gTW"], d["grid_gm"] = g.gTW, np.array([g.gm], np.int32)
    if g.grade is not None:
        d["grid_grade"] = g.grade
    return d


def main():
    ref = RefLib()
    only = set(sys.argv[1:])
    for name, (g, nd, prm) in seed_cases(ref).items():
        if only and name not in only:
            continue
        d = grid_arrays(g)
        d["seed_params"] = np.array([float(getattr(prm, f)) for f in SEED_FIELDS], np.float64)
        for a in ("P", "lab", "typ", "part", "part3"):
            d["seeds_" + a] = getattr(nd, a)
        path = os.path.join(HERE, name + ".npz")
        np.savez_compressed(path, **d)
        print(f"{name}: {nd.size()} seeds -> {os.path.getsize(path)} B")
    for name, (g, nd, prm) in cases(ref).items():
        if only and name not in only:
            continue
        d = grid_arrays(g)
        d.pop("grid_grade", None)
        d["seed_P"], d["seed_lab"], d["seed_typ"], d["seed_part"] = nd.P, nd.lab, nd.typ, nd.part
        d["params"] = np.array([float(getattr(prm, f)) for f in PARAM_FIELDS], np.float64)
        s = ref.state(g, prm, nd.copy())
        s.rebuild()
        for a in ("key", "sorted", "cstart", "nbr", "nnb", "Ps"):
            d[a] = s.read(a)
        s.force()
        d["F"] = s.read("F")
        s.tail()
        for a in ("P", "typ", "part", "mv"):
            d["it1_" + a] = s.read(a)
        x = nd.copy()
        st = ref.relax_cpu(g, prm, x)
        d["run_P"], d["run_typ"], d["run_part"] = x.P, x.typ, x.part
        d["run_stats"] = np.array([st.iters, st.rebuilds, st.fire_resets, st.n_interior, st.n_interface,
                                   st.n_junction, st.n_corner], np.int64)
        path = os.path.join(HERE, name + ".npz")
        np.savez_compressed(path, **d)
        print(f"{name}: {nd.size()} nodes, {st.iters} iterations, {st.rebuilds} builds -> {os.path.getsize(path)} B")


if __name__ == "__main__":
    main()
