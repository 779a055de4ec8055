"""The relaxation's public Python surface, mirroring the reference's C++ one.

  relax_cl(g, prm, nd, st=None, device=-1)
      tn::relax_cl (src/v2m_gpu.h:16-18 of fangq/trussnet): relax the nodes in
      place on a CUDA device; same contract as tn::relax_cpu
      (src/v2m_particles.h:99). Raises V2mError (a RuntimeError, as the
      reference throws std::runtime_error) when the device path fails; there is
      no CPU fallback inside -- the caller decides, as run_pipeline does
      (src/v2m_pipeline.cpp:492-526).
  relax_cl_batch(grids, prms, nodes, device=-1)
      many independent volumes in one set of launches (no reference counterpart).
  seed_cl(g, prm, device=-1)
      tn::seed_cpu (src/v2m_particles.cpp:625-726) on a CUDA device, without its
      shape-feature pass: the seeds as Nodes, and their part3 labels.
  Session
      the relaxation state kept on the device: the stages one at a time, repeated
      runs from the same seeds, internal arrays for checks.
"""
from __future__ import annotations

import ctypes as C
from typing import Sequence

import numpy as np

from . import _lib
from .types import (ARR, V2M_K, Grid, GridParams, GridParamsC, GridView, Nodes, NodesView, RelaxParams, RelaxParamsC, RelaxStats,
                    RelaxStatsC)

_ARR_DTYPE = {"key": np.int32, "sorted": np.int32, "cstart": np.int32, "Ps": np.float32, "nbr": np.int32,
              "nnb": np.int32, "F": np.float32, "hn": np.float32, "mv": np.float32, "V": np.float32, "pw": np.float32,
              "P0": np.float32, "hist": np.int32, "serial_sums": np.int32, "dirs": np.float32, "P": np.float32, "typ": np.uint8, "part": np.uint16}
_PER_NODE = {"key": 1, "sorted": 1, "Ps": 4, "nbr": V2M_K, "nnb": 1, "F": 4, "hn": 1, "mv": 1, "V": 3, "pw": 1,
             "P0": 3, "P": 3, "typ": 1, "part": 2, "dirs": 3}


def device_count() -> int:
    return int(_lib.load().v2m_cuda_device_count())


def _views(grids, prms, nodes):
    gv = (GridView * len(grids))(*[g.view() for g in grids])
    pv = (RelaxParamsC * len(prms))(*[p.to_c() for p in prms])
    nv = (NodesView * len(nodes))(*[nd.view() for nd in nodes])
    return gv, pv, nv


def relax_cl(g: Grid, prm: RelaxParams, nd: Nodes, st: RelaxStats | None = None, device: int = -1) -> RelaxStats:
    """tn::relax_cl: relax `nd` in place on CUDA device `device` (-1 = the first)."""
    L = _lib.load()
    gv, pv, nv = _views([g], [prm], [nd])
    sv = (RelaxStatsC * 1)()
    _lib.check(L.v2m_relax_cuda(gv, pv, nv, sv, device))
    out = RelaxStats.from_c(sv[0])
    if st is not None:
        st.__dict__.update(out.__dict__)
    return out


def relax_cl_batch(grids: Sequence[Grid], prms: Sequence[RelaxParams], nodes: Sequence[Nodes],
                   device: int = -1) -> list[RelaxStats]:
    """Relax many independent volumes together; each volume's result is the one
    relax_cl gives for it alone."""
    L = _lib.load()
    if not (len(grids) == len(prms) == len(nodes)):
        raise ValueError("grids, params and nodes must have the same length")
    gv, pv, nv = _views(grids, prms, nodes)
    sv = (RelaxStatsC * len(grids))()
    _lib.check(L.v2m_relax_cuda_batch(len(grids), gv, pv, nv, sv, device))
    return [RelaxStats.from_c(s) for s in sv]


def seed_cl(g: Grid, prm: RelaxParams, device: int = -1) -> tuple[Nodes, np.ndarray]:
    """Seed grid g on a CUDA device (g.grade is required): the nodes of
    tn::seed_cpu in its order (the shape-feature nodes excepted), and part3 (a
    CORNER node's fourth label, else V2M_NOLAB)."""
    L = _lib.load()
    gv = g.view()
    pv = prm.to_c()
    h = C.c_void_p()
    n = C.c_int64()
    _lib.check(L.v2m_seed_cuda(C.byref(gv), C.byref(pv), device, C.byref(h), C.byref(n)))
    try:
        nd, part3 = _copy_seed_result(L, h, n.value)
    finally:
        L.v2m_seed_free(h)
    return nd, part3


def _copy_seed_result(L, h, m: int) -> tuple[Nodes, np.ndarray]:
    nd = Nodes(P=np.zeros((m, 3), np.float32), lab=np.zeros(m, np.uint16), typ=np.zeros(m, np.uint8),
               part=np.zeros((m, 2), np.uint16))
    part3 = np.zeros(m, np.uint16)
    _lib.check(L.v2m_seed_copy(h, nd.P.ctypes.data, nd.lab.ctypes.data, nd.typ.ctypes.data, nd.part.ctypes.data,
                               part3.ctypes.data))
    return nd, part3


def grid_cl(L: np.ndarray, vs=(1.0, 1.0, 1.0), prm: GridParams | None = None, device: int = -1) -> Grid:
    """tn::build_grid_cpu of label volume L (uint16 [nz, ny, nx], x fastest) on a
    CUDA device, bit for bit: bricks, slots, smoothed indicators, sizing field
    and size grades (the returned grid carries grade, ready for seed_cl)."""
    lib = _lib.load()
    L = np.ascontiguousarray(L, np.uint16)
    nz, ny, nx = L.shape
    prm = prm or GridParams()
    pc = GridParamsC()
    for f in ("sigma", "sigma_thin", "thin_lo", "thin_hi", "thick", "thin_floor", "preserve", "sigma_curv", "hbase",
              "hmin", "hmax", "K", "g"):
        setattr(pc, f, float(getattr(prm, f)))
    hl = np.ascontiguousarray(prm.hlab, np.float32)
    pc.hlab = hl.ctypes.data if hl.size else None
    pc.nhlab = int(hl.size)
    vsa = np.asarray(vs, np.float32)
    h = C.c_void_p()
    _lib.check(lib.v2m_grid_build_cuda(L.ctypes.data, nx, ny, nz, vsa.ctypes.data, C.byref(pc), device, C.byref(h)))
    owner = _GridResult(lib, h)
    gv = GridView()
    _lib.check(lib.v2m_grid_result_view(h, C.byref(gv)))
    g = Grid.from_view(gv, owner)   # the grid's arrays are the result's host memory, no copy
    R = C.c_int32()
    _lib.check(lib.v2m_grid_result_info(h, None, C.byref(R), None, None))
    g.R = R.value
    return g


class _GridResult:
    """Owner of a v2m_grid_result's host arrays: freed when the last array
    viewing them is gone (the result holds host memory only)."""

    def __init__(self, lib, h):
        self.lib, self.h = lib, h

    def __del__(self):
        if self.h:
            self.lib.v2m_grid_free(self.h)
            self.h = None


def points_cl(L: np.ndarray, vs=(1.0, 1.0, 1.0), gprm: GridParams | None = None, prm: RelaxParams | None = None,
              device: int = -1) -> tuple[Nodes, np.ndarray, RelaxStats]:
    """The pipeline's points mode on a CUDA device (v2m_points_cuda): the label
    volume uploaded once, grid built, seeded and relaxed from device arrays,
    the relaxed nodes copied back once -- build_grid_cpu -> seed_cpu ->
    relax_cpu bit for bit. Returns (nodes, part3, stats)."""
    lib = _lib.load()
    L = np.ascontiguousarray(L, np.uint16)
    nz, ny, nx = L.shape
    gprm = gprm or GridParams()
    prm = prm or RelaxParams()
    pc = GridParamsC()
    for f in ("sigma", "sigma_thin", "thin_lo", "thin_hi", "thick", "thin_floor", "preserve", "sigma_curv", "hbase",
              "hmin", "hmax", "K", "g"):
        setattr(pc, f, float(getattr(gprm, f)))
    hl = np.ascontiguousarray(gprm.hlab, np.float32)
    pc.hlab = hl.ctypes.data if hl.size else None
    pc.nhlab = int(hl.size)
    vsa = np.asarray(vs, np.float32)
    pv = prm.to_c()
    sv = RelaxStatsC()
    h = C.c_void_p()
    n = C.c_int64()
    _lib.check(lib.v2m_points_cuda(L.ctypes.data, nx, ny, nz, vsa.ctypes.data, C.byref(pc), C.byref(pv), device,
                                   C.byref(h), C.byref(n), C.byref(sv)))
    try:
        nd, part3 = _copy_seed_result(lib, h, n.value)
    finally:
        lib.v2m_seed_free(h)
    return nd, part3, RelaxStats.from_c(sv)


def validate_lists(nbr: np.ndarray, nnb: np.ndarray, pi: np.ndarray, pj: np.ndarray) -> str:
    """Host-side check of truss lists (v2m_validate_lists; no device): lengths,
    ids in range, no self-edges or repeats, and (distance, id) order from the
    positions the lists were built from (pi: each node's position at its build,
    pj: the bin-order snapshot's). Returns "" when valid, else the first
    violation."""
    L = _lib.load()
    n = int(nnb.size)
    nbr = np.ascontiguousarray(nbr, np.int32).reshape(-1)
    nnb = np.ascontiguousarray(nnb, np.int32)
    pi = np.ascontiguousarray(pi, np.float32).reshape(-1)
    pj = np.ascontiguousarray(pj, np.float32).reshape(-1)
    if nbr.size != n * V2M_K or pi.size != 3 * n or pj.size != 3 * n:
        raise ValueError("validate_lists: array sizes do not match the node count")
    rep = C.create_string_buffer(512)
    rc = L.v2m_validate_lists(n, nbr.ctypes.data, nnb.ctypes.data, pi.ctypes.data, pj.ctypes.data, rep, len(rep))
    if rc not in (0, _lib.V2M_ERR_KERNEL):
        _lib.check(rc)
    return rep.value.decode()


def build_positions(Ps: np.ndarray, sorted_ids: np.ndarray) -> np.ndarray:
    """Each node's position in the bin-order snapshot (Ps, 4 floats per slot,
    slot s holding node sorted_ids[s]), in node order (3 floats per node)."""
    n = sorted_ids.size
    out = np.zeros((n, 3), np.float32)
    out[sorted_ids] = Ps.reshape(-1, 4)[:n, :3]
    return out


class Session:
    """Device-resident relaxation state of one or more volumes."""

    def __init__(self, grids, prms, nodes, device: int = -1):
        if isinstance(grids, Grid):
            grids, prms, nodes = [grids], [prms], [nodes]
        self.L = _lib.load()
        self.nvol = len(grids)
        self.n = [nd.size() for nd in nodes]
        gv, pv, nv = _views(grids, prms, nodes)
        h = C.c_void_p()
        _lib.check(self.L.v2m_session_create(self.nvol, gv, pv, nv, device, C.byref(h)))
        self.h = h
        self.nkeys = []
        self.nlev = []
        for v in range(self.nvol):
            n, nk, nl = C.c_int64(), C.c_int64(), C.c_int32()
            _lib.check(self.L.v2m_session_info(self.h, v, C.byref(n), C.byref(nk), C.byref(nl)))
            self.nkeys.append(nk.value)
            self.nlev.append(nl.value)

    def close(self):
        if getattr(self, "h", None):
            self.L.v2m_session_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def reset(self):
        _lib.check(self.L.v2m_session_reset(self.h))

    def rebuild(self):
        _lib.check(self.L.v2m_session_rebuild(self.h))

    def force(self):
        _lib.check(self.L.v2m_session_force(self.h))

    def step_tail(self):
        _lib.check(self.L.v2m_session_step_tail(self.h))

    def iterate(self, iters: int, graph: bool = True):
        _lib.check(self.L.v2m_session_iterate(self.h, int(iters), int(graph)))

    def run(self, graph: bool = True):
        _lib.check(self.L.v2m_session_run(self.h, int(graph)))

    def synchronize(self):
        _lib.check(self.L.v2m_session_synchronize(self.h))

    def stats(self, vol: int = 0) -> RelaxStats:
        sv = RelaxStatsC()
        _lib.check(self.L.v2m_session_stats(self.h, vol, C.byref(sv)))
        return RelaxStats.from_c(sv)

    def read_nodes(self, nd: Nodes, vol: int = 0) -> Nodes:
        v = nd.view()
        _lib.check(self.L.v2m_session_read_nodes(self.h, vol, C.byref(v)))
        return nd

    def read(self, name: str, vol: int = 0) -> np.ndarray:
        dt = _ARR_DTYPE[name]
        if name == "cstart":
            count = self.nkeys[vol] + 1
        elif name == "hist":
            count = 34
        elif name == "serial_sums":
            count = 1
        else:
            count = self.n[vol] * _PER_NODE[name]
        out = np.zeros(max(count, 1), dt)
        _lib.check(self.L.v2m_session_read_array(self.h, vol, ARR[name], out.ctypes.data, out.nbytes))
        return out[:count]

    def write(self, name: str, a: np.ndarray, vol: int = 0):
        a = np.ascontiguousarray(a, _ARR_DTYPE[name])
        _lib.check(self.L.v2m_session_write_array(self.h, vol, ARR[name], a.ctypes.data, a.nbytes))

    def write_lists(self, nbr: np.ndarray, nnb: np.ndarray, vol: int = 0):
        nbr = np.ascontiguousarray(nbr, np.int32)
        nnb = np.ascontiguousarray(nnb, np.int32)
        _lib.check(self.L.v2m_session_write_lists(self.h, vol, nbr.ctypes.data, nnb.ctypes.data))

    def validate_lists(self, vol: int = 0) -> str:
        """The session's current truss lists through validate_lists ("" when valid)."""
        return validate_lists(self.read("nbr", vol), self.read("nnb", vol), self.read("P0", vol),
                              build_positions(self.read("Ps", vol), self.read("sorted", vol)))

    def timed_runs(self, runs: int, graph: bool = True, time_force: bool = False) -> float:
        """Device milliseconds of `runs` whole relaxations from the seeds (CUDA events)."""
        ms = C.c_float()
        _lib.check(self.L.v2m_session_timed_runs(self.h, int(runs), int(graph), int(time_force), C.byref(ms)))
        return ms.value

    def autotune(self, reps: int = 20) -> str:
        """Time the result-neutral launch shapes, keep the fastest (cached); the
        session is reset to its seeds."""
        buf = C.create_string_buffer(4096)
        _lib.check(self.L.v2m_session_autotune(self.h, int(reps), buf, len(buf)))
        return buf.value.decode()

    def shapes(self):
        a, b = C.c_int32(), C.c_int32()
        _lib.check(self.L.v2m_session_shapes(self.h, C.byref(a), C.byref(b)))
        return dict(force_threads=a.value, nbr_threads=b.value)

    def profile_stages(self, iters: int) -> dict:
        """Device ms per stage over `iters` plain-launch iterations from the current state."""
        ms = np.zeros(5, np.float64)
        _lib.check(self.L.v2m_session_profile_stages(self.h, int(iters), ms.ctypes.data))
        return dict(zip(("force", "move", "control_refresh", "rebuild", "total"), ms.tolist()))

    def queue_sizes(self):
        """(trapped, interior) nodes the last iteration's move sent to the trapped-move stage."""
        a, b = C.c_int32(), C.c_int32()
        _lib.check(self.L.v2m_session_queue_sizes(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def clear_counters(self):
        _lib.check(self.L.v2m_session_clear_counters(self.h))

    def counters(self):
        a, b, c = C.c_int64(), C.c_int64(), C.c_double()
        _lib.check(self.L.v2m_session_counters(self.h, C.byref(a), C.byref(b), C.byref(c)))
        return dict(launches=a.value, force_launches=b.value, force_ms=c.value)
