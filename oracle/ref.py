"""TEST INFRASTRUCTURE ONLY: ctypes access to the two CPU checkers.

  RefLib     oracle/_ref/libv2m_ref.so -- the reference's own relax_cpu,
             build_grid_cpu and seed_cpu (fangq/trussnet src/v2m_particles.cpp,
             src/v2m_grid.cpp), compiled from its sources by oracle/Makefile,
             and relax_cpu's loop split into stages (ref_harness.cpp).
  OracleLib  oracle/liboracle.so -- the plain-C restatement (v2m_oracle.c), in
             FP32 without contraction ("f32") and in FP64 ("f64").

Only tests, the smoke check and the benchmark's CPU-baseline leg use this module.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from trussnet_b200.types import ARR, V2M_K, Grid, GridView, Nodes, NodesView, RelaxParams, RelaxStats, RelaxStatsC

HERE = os.path.dirname(os.path.abspath(__file__))
REF_SO = os.path.join(HERE, "_ref", "libv2m_ref.so")
ORACLE_SO = os.path.join(HERE, "liboracle.so")

_DT = {"key": np.int32, "sorted": np.int32, "cstart": np.int32, "Ps": np.float32, "nbr": np.int32, "nnb": np.int32,
       "F": np.float32, "hn": np.float32, "mv": np.float32, "V": np.float32, "pw": np.float32, "P0": np.float32,
       "hist": np.int32, "P": np.float32, "typ": np.uint8, "part": np.uint16}


def _per_node(name):
    return {"key": 1, "sorted": 1, "Ps": 4, "nbr": V2M_K, "nnb": 1, "F": 4, "hn": 1, "mv": 1, "V": 3, "pw": 1,
            "P0": 3, "P": 3, "typ": 1, "part": 2}.get(name)


def available() -> bool:
    return os.path.exists(REF_SO)


class RefLib:
    def __init__(self, path: str = REF_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} is not built (make -f oracle/Makefile ref)")
        L = C.CDLL(path)
        self.L = L
        vp = C.c_void_p
        L.ref_last_error.restype = C.c_char_p
        L.ref_relax_cpu.argtypes = [C.POINTER(GridView), vp, C.POINTER(NodesView), C.POINTER(RelaxStatsC)]
        L.ref_grid_build.restype = vp
        L.ref_grid_build.argtypes = [vp, C.c_int, C.c_int, C.c_int, vp, C.c_float, C.c_float, C.c_float, C.c_float]
        L.ref_grid_view.argtypes = [vp, C.POINTER(GridView)]
        L.ref_grid_build_p.restype = vp
        L.ref_grid_build_p.argtypes = [vp, C.c_int, C.c_int, C.c_int, vp, vp]
        L.ref_shape_grid.restype = vp
        L.ref_shape_grid.argtypes = [C.c_char_p, C.c_char_p, C.c_double, C.c_double, C.c_double, C.c_int, C.c_float,
                                     C.c_float, C.c_float, C.c_float, C.c_int]
        L.ref_grid_free.argtypes = [vp]
        L.ref_seed.restype = vp
        L.ref_seed.argtypes = [vp, vp, C.POINTER(C.c_int64)]
        L.ref_seed_copy.argtypes = [vp, vp, vp, vp, vp]
        L.ref_seed_free.argtypes = [vp]
        L.ref_seed_part3.argtypes = [vp, vp]
        L.ref_seed_view.restype = vp
        L.ref_seed_view.argtypes = [C.POINTER(GridView), vp, C.POINTER(C.c_int64)]
        L.ref_state_create.restype = vp
        L.ref_state_create.argtypes = [C.POINTER(GridView), vp, C.POINTER(NodesView)]
        L.ref_state_free.argtypes = [vp]
        L.ref_state_info.argtypes = [vp, C.POINTER(C.c_int64), C.POINTER(C.c_int32), C.POINTER(C.c_float)]
        for f in ("ref_state_rebuild", "ref_state_force", "ref_state_move_only", "ref_state_tail", "ref_state_run"):
            getattr(L, f).argtypes = [vp]
        L.ref_state_counts.argtypes = [vp] + [C.POINTER(C.c_int32)] * 6 + [C.POINTER(C.c_float)] * 2 + \
            [C.POINTER(C.c_double)] + [C.POINTER(C.c_float)] * 2
        L.ref_state_read.restype = C.c_int64
        L.ref_state_read.argtypes = [vp, C.c_int, vp, C.c_int64]
        L.ref_state_write.argtypes = [vp, C.c_int, vp, C.c_int64]

    def err(self):
        return self.L.ref_last_error().decode()

    def relax_cpu(self, g: Grid, prm: RelaxParams, nd: Nodes) -> RelaxStats:
        """tn::relax_cpu on copies; nd is updated in place."""
        gv = g.view()
        pv = prm.to_c()
        nv = nd.view()
        sv = RelaxStatsC()
        if self.L.ref_relax_cpu(C.byref(gv), C.byref(pv), C.byref(nv), C.byref(sv)) != 0:
            raise RuntimeError(self.err())
        return RelaxStats.from_c(sv)

    def build_grid(self, L: np.ndarray, vs=(1.0, 1.0, 1.0), sigma=1.0, hbase=0.0, hmin=0.0, hmax=0.0) -> Grid:
        """tn::build_grid_cpu of label volume L [nz, ny, nx] with those GridParams."""
        L = np.ascontiguousarray(L, np.uint16)
        nz, ny, nx = L.shape
        vsa = np.array(vs, np.float32)
        h = self.L.ref_grid_build(L.ctypes.data, nx, ny, nz, vsa.ctypes.data, sigma, hbase, hmin, hmax)
        if not h:
            raise RuntimeError(self.err())
        try:
            gv = GridView()
            self.L.ref_grid_view(h, C.byref(gv))
            g = Grid.from_view(gv)
        finally:
            self.L.ref_grid_free(h)
        return g

    def build_grid_p(self, L: np.ndarray, vs=(1.0, 1.0, 1.0), prm=None) -> Grid:
        """tn::build_grid_cpu of label volume L [nz, ny, nx] with every field of
        GridParams (trussnet_b200.types.GridParams, hlab included)."""
        from trussnet_b200.types import GridParams, GridParamsC
        prm = prm or GridParams()
        L = np.ascontiguousarray(L, np.uint16)
        nz, ny, nx = L.shape
        pc = GridParamsC()
        for f in ("sigma", "sigma_thin", "thin_lo", "thin_hi", "thick", "thin_floor", "preserve", "sigma_curv",
                  "hbase", "hmin", "hmax", "K", "g"):
            setattr(pc, f, float(getattr(prm, f)))
        hl = np.ascontiguousarray(prm.hlab, np.float32)
        pc.hlab = hl.ctypes.data if hl.size else None
        pc.nhlab = int(hl.size)
        vsa = np.array(vs, np.float32)
        h = self.L.ref_grid_build_p(L.ctypes.data, nx, ny, nz, vsa.ctypes.data, C.byref(pc))
        if not h:
            raise RuntimeError(self.err())
        try:
            gv = GridView()
            self.L.ref_grid_view(h, C.byref(gv))
            g = Grid.from_view(gv)
        finally:
            self.L.ref_grid_free(h)
        return g

    def seed(self, g: Grid, prm: RelaxParams) -> Nodes:
        """tn::seed_cpu on grid g (g.grade required); the nodes carry part3."""
        gv, pv = g.view(), prm.to_c()
        n = C.c_int64()
        sh = self.L.ref_seed_view(C.byref(gv), C.byref(pv), C.byref(n))
        if not sh:
            raise RuntimeError(self.err())
        try:
            m = n.value
            nd = Nodes(P=np.zeros((m, 3), np.float32), lab=np.zeros(m, np.uint16), typ=np.zeros(m, np.uint8),
                       part=np.zeros((m, 2), np.uint16))
            self.L.ref_seed_copy(sh, nd.P.ctypes.data, nd.lab.ctypes.data, nd.typ.ctypes.data, nd.part.ctypes.data)
            nd.part3 = np.zeros(m, np.uint16)
            self.L.ref_seed_part3(sh, nd.part3.ctypes.data)
        finally:
            self.L.ref_seed_free(sh)
        return nd

    def build_and_seed(self, L, vs=(1.0, 1.0, 1.0), sigma=1.0, hbase=0.0, hmin=0.0, hmax=0.0,
                       prm: RelaxParams | None = None):
        """build_grid_cpu + seed_cpu of the reference (the pipeline's stages 2-3)."""
        L = np.ascontiguousarray(L, np.uint16)
        nz, ny, nx = L.shape
        vsa = np.array(vs, np.float32)
        h = self.L.ref_grid_build(L.ctypes.data, nx, ny, nz, vsa.ctypes.data, sigma, hbase, hmin, hmax)
        if not h:
            raise RuntimeError(self.err())
        return self._grid_and_seeds(h, prm)

    def shape_and_seed(self, scene: str, voxel=1.0, gap=0.0, margin=3.0, bricks=True, sigma=1.0, hbase=0.0,
                       hmin=0.0, hmax=0.0, prm: RelaxParams | None = None, overlap="overwrite", feat=False):
        """Shape input: the reference's shape compiler on a JSON scene, a grid
        over its raster with the compiled program as the fields (gm = -1), and
        seed_cpu on it (ref_shape_grid). feat: the grid build also takes the
        scene's sharp features, as the shape front end hands them over (sizing
        refined near them, tn::Grid::feat set), so seed_cpu pins nodes on them."""
        h = self.L.ref_shape_grid(scene.encode(), overlap.encode(), voxel, gap, margin, int(bricks), sigma, hbase,
                                  hmin, hmax, int(feat))
        if not h:
            raise RuntimeError(self.err())
        return self._grid_and_seeds(h, prm)

    def _grid_and_seeds(self, h, prm):
        prm = prm or RelaxParams()
        try:
            gv = GridView()
            self.L.ref_grid_view(h, C.byref(gv))
            g = Grid.from_view(gv)
            pv = prm.to_c()
            n = C.c_int64()
            sh = self.L.ref_seed(h, C.byref(pv), C.byref(n))
            if not sh:
                raise RuntimeError(self.err())
            n = n.value
            nd = Nodes(P=np.zeros((n, 3), np.float32), lab=np.zeros(n, np.uint16), typ=np.zeros(n, np.uint8),
                       part=np.zeros((n, 2), np.uint16))
            self.L.ref_seed_copy(sh, nd.P.ctypes.data, nd.lab.ctypes.data, nd.typ.ctypes.data, nd.part.ctypes.data)
            nd.part3 = np.zeros(n, np.uint16)   # (a CORNER node's fourth label)
            self.L.ref_seed_part3(sh, nd.part3.ctypes.data)
            self.L.ref_seed_free(sh)
        finally:
            self.L.ref_grid_free(h)
        return g, nd

    def state(self, g: Grid, prm: RelaxParams, nd: Nodes) -> "RefState":
        return RefState(self, g, prm, nd)


class RefState:
    """relax_cpu's loop, stage by stage (ref_harness.cpp)."""

    def __init__(self, lib: RefLib, g: Grid, prm: RelaxParams, nd: Nodes):
        self.lib = lib
        self.n = nd.size()
        gv, pv, nv = g.view(), prm.to_c(), nd.view()
        self.h = lib.L.ref_state_create(C.byref(gv), C.byref(pv), C.byref(nv))
        if not self.h:
            raise RuntimeError(lib.err())
        nk, nl, b0 = C.c_int64(), C.c_int32(), C.c_float()
        lib.L.ref_state_info(self.h, C.byref(nk), C.byref(nl), C.byref(b0))
        self.nkeys, self.nlev, self.b0 = nk.value, nl.value, b0.value

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.L.ref_state_free(self.h)
            self.h = None

    def rebuild(self):
        self.lib.L.ref_state_rebuild(self.h)

    def force(self):
        self.lib.L.ref_state_force(self.h)

    def move_only(self):
        self.lib.L.ref_state_move_only(self.h)

    def tail(self) -> bool:
        return bool(self.lib.L.ref_state_tail(self.h))

    def run(self):
        self.lib.L.ref_state_run(self.h)

    def counts(self) -> dict:
        i32 = [C.c_int32() for _ in range(6)]
        f = [C.c_float() for _ in range(2)]
        p = C.c_double()
        f2 = [C.c_float() for _ in range(2)]
        self.lib.L.ref_state_counts(self.h, *[C.byref(x) for x in i32], *[C.byref(x) for x in f], C.byref(p),
                                    *[C.byref(x) for x in f2])
        names = ("it", "stopped", "nhalf", "nrefresh", "rebuilds", "fire_resets")
        d = {k: v.value for k, v in zip(names, i32)}
        d.update(fire_dt=f[0].value, fire_alpha=f[1].value, power=p.value, mmax=f2[0].value, p99=f2[1].value)
        return d

    def read(self, name: str) -> np.ndarray:
        dt = _DT[name]
        if name == "cstart":
            count = self.nkeys + 1
        elif name == "hist":
            count = 34
        else:
            count = self.n * _per_node(name)
            if name in ("V", "pw") and count == 0:
                count = 1
        out = np.zeros(max(count, 1) + 64, dt)
        nb = self.lib.L.ref_state_read(self.h, ARR[name], out.ctypes.data, out.nbytes)
        if nb < 0:
            raise RuntimeError(self.lib.err())
        return out[: nb // out.itemsize].copy()

    def write(self, name: str, a: np.ndarray):
        a = np.ascontiguousarray(a, _DT[name])
        if self.lib.L.ref_state_write(self.h, ARR[name], a.ctypes.data, a.nbytes) != 0:
            raise RuntimeError(self.lib.err())
