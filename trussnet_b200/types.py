"""Host-side mirrors of the reference's relaxation types and their C views.

``Grid``, ``RelaxParams``, ``Nodes`` and ``RelaxStats`` carry the same fields,
names and meaning as tn::Grid (src/v2m_grid.h:45-81), tn::RelaxParams
(src/v2m_particles.h:21-41), tn::Nodes (src/v2m_particles.h:78-87) and
tn::RelaxStats (src/v2m_particles.h:89-96) of fangq/trussnet; the ctypes
structures are the POD views of include/v2m_cuda.h that cross the C ABI.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field, fields

import numpy as np

V2M_K = 24
V2M_MAXLEV = 8
V2M_BS = 8
V2M_SLOT = 512
V2M_BL = 16
V2M_NOLAB = 0xFFFF
V2M_INTERIOR, V2M_INTERFACE, V2M_JUNCTION, V2M_CORNER = 0, 1, 2, 3

# internal arrays (V2M_ARR_* of include/v2m_cuda.h)
ARR = dict(key=1, sorted=2, cstart=3, Ps=4, nbr=5, nnb=6, F=7, hn=8, mv=9, V=10, pw=11, P0=12, hist=13, serial_sums=14, dirs=15,
           P=20, typ=21, part=22)


class GridView(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
                ("nbx", C.c_int32), ("nby", C.c_int32), ("nbz", C.c_int32),
                ("vs", C.c_float * 3),
                ("L", C.c_void_p), ("bl_cnt", C.c_void_p), ("bl_lab", C.c_void_p), ("bl_slot", C.c_void_p),
                ("phi", C.c_void_p), ("nslots", C.c_int64), ("h", C.c_void_p),
                ("hmin", C.c_float), ("hmax", C.c_float),
                ("gI", C.c_void_p), ("gTW", C.c_void_p), ("gm", C.c_int32), ("ngTW", C.c_int64),
                ("grade", C.c_void_p), ("feat", C.c_void_p), ("nfeat", C.c_int64)]


class RelaxParamsC(C.Structure):
    _fields_ = [("nseed", C.c_int32), ("t", C.c_float), ("skin", C.c_float), ("fscale", C.c_float),
                ("fsurf", C.c_float), ("dt", C.c_float), ("maxstep", C.c_float), ("snap", C.c_float),
                ("max_iters", C.c_int32), ("dptol", C.c_float), ("jseed", C.c_float),
                ("corners", C.c_int32), ("voxel_trap", C.c_int32), ("thin", C.c_float),
                ("fire", C.c_int32), ("fire_dtmax", C.c_float), ("verbose", C.c_int32),
                ("h_mode", C.c_int32), ("rebuild_div", C.c_int32), ("rebuild_policy", C.c_int32)]


class NodesView(C.Structure):
    _fields_ = [("n", C.c_int64), ("P", C.c_void_p), ("lab", C.c_void_p), ("typ", C.c_void_p),
                ("part", C.c_void_p)]


class RelaxStatsC(C.Structure):
    _fields_ = [("iters", C.c_int32), ("rebuilds", C.c_int32), ("last_move", C.c_float), ("last_p99", C.c_float),
                ("fire_resets", C.c_int32), ("fire_dt", C.c_float),
                ("n_interior", C.c_int64), ("n_interface", C.c_int64), ("n_junction", C.c_int64),
                ("n_corner", C.c_int64),
                ("ms_seed", C.c_double), ("ms_hash", C.c_double), ("ms_force", C.c_double), ("ms_move", C.c_double)]


@dataclass
class RelaxParams:
    """tn::RelaxParams (src/v2m_particles.h:21-41) plus three extensions (0 = reference)."""
    nseed: int = 8
    t: float = 1.3
    skin: float = 0.3
    fscale: float = 1.2
    fsurf: float = 1.0
    dt: float = 0.5
    maxstep: float = 0.2
    snap: float = 0.5
    max_iters: int = 500
    dptol: float = 2e-3
    jseed: float = 0.8
    corners: bool = True
    voxel_trap: bool = False
    thin: float = 0.0
    fire: bool = True
    fire_dtmax: float = 2.0
    verbose: bool = False
    h_mode: int = 0          # 0: nearest-voxel h (reference), 1: trilinear h
    rebuild_div: int = 0     # 0: V2M_REBUILD_DIV or 300
    rebuild_policy: int = 0  # 0: reference Verlet trigger, 1: max |dp| since build > 0.1 h, 2: fixed lists

    def to_c(self) -> RelaxParamsC:
        c = RelaxParamsC()
        for f in fields(self):
            v = getattr(self, f.name)
            setattr(c, f.name, int(v) if isinstance(v, bool) else v)
        return c


@dataclass
class RelaxStats:
    """tn::RelaxStats (src/v2m_particles.h:89-96)."""
    iters: int = 0
    rebuilds: int = 0
    last_move: float = 0.0
    last_p99: float = 0.0
    fire_resets: int = 0
    fire_dt: float = 0.0
    n_interior: int = 0
    n_interface: int = 0
    n_junction: int = 0
    n_corner: int = 0
    ms_seed: float = 0.0
    ms_hash: float = 0.0
    ms_force: float = 0.0
    ms_move: float = 0.0

    @classmethod
    def from_c(cls, c: RelaxStatsC) -> "RelaxStats":
        return cls(**{f.name: getattr(c, f.name) for f in fields(cls)})


class GridParamsC(C.Structure):
    """v2m_grid_params: tn::GridParams (src/v2m_grid.h:21-43), label input."""
    _fields_ = [(f, C.c_float) for f in ("sigma", "sigma_thin", "thin_lo", "thin_hi", "thick", "thin_floor", "preserve",
                                         "sigma_curv", "hbase", "hmin", "hmax", "K", "g")] + \
        [("hlab", C.c_void_p), ("nhlab", C.c_int32)]


@dataclass
class GridParams:
    """tn::GridParams (src/v2m_grid.h:21-43): the reference's defaults."""
    sigma: float = 1.0
    sigma_thin: float = 0.35
    thin_lo: float = 2.0
    thin_hi: float = 4.0
    thick: float = 0.0
    thin_floor: float = 0.5
    preserve: float = 0.0
    sigma_curv: float = 2.0
    hbase: float = 0.0
    hmin: float = 0.0
    hmax: float = 0.0
    K: float = 3.0
    g: float = 0.3
    hlab: tuple = ()


@dataclass
class Grid:
    """The relaxation's read-only fields: tn::Grid (src/v2m_grid.h:45-81)."""
    nx: int
    ny: int
    nz: int
    vs: tuple
    L: np.ndarray            # uint16 [nz, ny, nx] (x fastest)
    bl_cnt: np.ndarray       # int32 [nb]
    bl_lab: np.ndarray       # uint16 [nb * 16]
    bl_slot: np.ndarray      # int32 [nb]
    phi: np.ndarray          # float32 [nslots * 512]
    h: np.ndarray            # float32 [nz, ny, nx] (mm)
    hmin: float
    hmax: float
    gI: np.ndarray | None = None
    gTW: np.ndarray | None = None   # gray: thresholds, widths; gm < 0: the analytic shape program
    gm: int = 0                     # gray thresholds; 0: label volume; < 0: analytic shape fields
    R: int = 6
    grade: np.ndarray | None = None  # uint8 [nz, ny, nx] size grades (seeding only)
    feat: np.ndarray | None = None   # float32: shape input's sharp features (tn::Grid::feat; seeding only)

    @property
    def nbx(self):
        return (self.nx + V2M_BS - 1) // V2M_BS

    @property
    def nby(self):
        return (self.ny + V2M_BS - 1) // V2M_BS

    @property
    def nbz(self):
        return (self.nz + V2M_BS - 1) // V2M_BS

    def view(self) -> GridView:
        """A C view over this grid's arrays (they must stay alive while it is used)."""
        for a in ("L", "bl_cnt", "bl_lab", "bl_slot", "phi", "h"):
            arr = getattr(self, a)
            assert arr.flags.c_contiguous, a
        v = GridView()
        v.nx, v.ny, v.nz = self.nx, self.ny, self.nz
        v.nbx, v.nby, v.nbz = self.nbx, self.nby, self.nbz
        v.vs[:] = [float(x) for x in self.vs]
        v.L = self.L.ctypes.data
        v.bl_cnt = self.bl_cnt.ctypes.data
        v.bl_lab = self.bl_lab.ctypes.data
        v.bl_slot = self.bl_slot.ctypes.data
        v.phi = self.phi.ctypes.data
        v.nslots = self.phi.size // V2M_SLOT
        v.h = self.h.ctypes.data
        v.hmin, v.hmax = float(self.hmin), float(self.hmax)
        v.gI = self.gI.ctypes.data if self.gI is not None else None
        if self.gTW is not None:
            assert self.gTW.dtype == np.float32 and self.gTW.flags.c_contiguous
        v.gTW = self.gTW.ctypes.data if self.gTW is not None else None
        v.gm = int(self.gm)
        v.ngTW = int(self.gTW.size) if self.gTW is not None else 0
        if self.grade is not None:
            assert self.grade.dtype == np.uint8 and self.grade.flags.c_contiguous
            assert self.grade.size == self.nx * self.ny * self.nz
        v.grade = self.grade.ctypes.data if self.grade is not None else None
        if self.feat is not None and self.feat.size:
            assert self.feat.dtype == np.float32 and self.feat.flags.c_contiguous
            v.feat = self.feat.ctypes.data
            v.nfeat = int(self.feat.size)
        return v

    @classmethod
    def from_view(cls, v: GridView, owner=None) -> "Grid":
        """A Grid of a C view's arrays: copies, or (owner given) views of the
        view's own memory that keep `owner`, the holder of that memory, alive
        for as long as any of them lives."""
        nv = v.nx * v.ny * v.nz
        nb = v.nbx * v.nby * v.nbz

        def arr(ptr, dtype, count):
            if not ptr or count == 0:
                return np.zeros(0, dtype)
            if owner is not None:
                buf = (C.c_char * (count * np.dtype(dtype).itemsize)).from_address(ptr)
                buf._owner = owner
                return np.frombuffer(buf, dtype, count)
            return np.ctypeslib.as_array(C.cast(ptr, C.POINTER(np.ctypeslib.as_ctypes_type(dtype))),
                                         shape=(count,)).copy()
        g = cls(nx=v.nx, ny=v.ny, nz=v.nz, vs=tuple(v.vs),
                L=arr(v.L, np.uint16, nv).reshape(v.nz, v.ny, v.nx),
                bl_cnt=arr(v.bl_cnt, np.int32, nb), bl_lab=arr(v.bl_lab, np.uint16, nb * V2M_BL),
                bl_slot=arr(v.bl_slot, np.int32, nb), phi=arr(v.phi, np.float32, v.nslots * V2M_SLOT),
                h=arr(v.h, np.float32, nv).reshape(v.nz, v.ny, v.nx), hmin=v.hmin, hmax=v.hmax, gm=v.gm)
        if v.gm > 0:
            g.gI = arr(v.gI, np.float32, nv)
            g.gTW = arr(v.gTW, np.float32, 2 * v.gm)
        elif v.gm < 0:
            g.gTW = arr(v.gTW, np.float32, v.ngTW)
        if v.grade:
            g.grade = arr(v.grade, np.uint8, nv).reshape(v.nz, v.ny, v.nx)
        if v.feat and v.nfeat > 0:
            g.feat = arr(v.feat, np.float32, v.nfeat)
        return g

    def nbytes(self) -> int:
        n = sum(getattr(self, a).nbytes for a in ("L", "bl_cnt", "bl_lab", "bl_slot", "phi", "h"))
        if self.gI is not None:
            n += self.gI.nbytes
        if self.gTW is not None:
            n += self.gTW.nbytes
        return n


@dataclass
class Nodes:
    """tn::Nodes (src/v2m_particles.h:78-87): P float32 [n,3], lab uint16, typ uint8, part uint16 [n,2]."""
    P: np.ndarray
    lab: np.ndarray
    typ: np.ndarray
    part: np.ndarray

    def size(self) -> int:
        return int(self.lab.shape[0])

    def copy(self) -> "Nodes":
        return Nodes(self.P.copy(), self.lab.copy(), self.typ.copy(), self.part.copy())

    def view(self) -> NodesView:
        for a in ("P", "lab", "typ", "part"):
            assert getattr(self, a).flags.c_contiguous, a
        assert self.P.dtype == np.float32 and self.lab.dtype == np.uint16
        assert self.typ.dtype == np.uint8 and self.part.dtype == np.uint16
        v = NodesView()
        v.n = self.size()
        v.P = self.P.ctypes.data
        v.lab = self.lab.ctypes.data
        v.typ = self.typ.ctypes.data
        v.part = self.part.ctypes.data
        return v

    def nbytes(self) -> int:
        return self.P.nbytes + self.lab.nbytes + self.typ.nbytes + self.part.nbytes
