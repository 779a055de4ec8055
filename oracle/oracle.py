"""TEST INFRASTRUCTURE ONLY: ctypes access to oracle/liboracle.so, the plain-C
restatement of the relaxation (v2m_oracle.c / v2m_oracle_body.h) in FP32
without contraction ("f32") and in FP64 ("f64").

Only tests, the smoke check and the benchmark's CPU-baseline leg use it.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from trussnet_b200.types import ARR, V2M_K, Grid, GridView, Nodes, NodesView, RelaxParams, RelaxStats, RelaxStatsC

HERE = os.path.dirname(os.path.abspath(__file__))
SO = os.path.join(HERE, "liboracle.so")
_lib = None


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(SO):
            raise FileNotFoundError(f"{SO} is not built (make -f oracle/Makefile)")
        L = C.CDLL(SO)
        vp = C.c_void_p
        for suf in ("f32", "f64"):
            getattr(L, f"orc_create_{suf}").restype = vp
            getattr(L, f"orc_create_{suf}").argtypes = [C.POINTER(GridView), vp, C.POINTER(NodesView)]
            getattr(L, f"orc_free_{suf}").argtypes = [vp]
            for f in ("rebuild", "force", "move", "tail", "run"):
                getattr(L, f"orc_{f}_{suf}").argtypes = [vp]
            getattr(L, f"orc_info_{suf}").argtypes = [vp, C.POINTER(C.c_int64), C.POINTER(C.c_int32)]
            getattr(L, f"orc_counts_{suf}").argtypes = [vp, vp, vp]
            getattr(L, f"orc_read_{suf}").restype = C.c_int64
            getattr(L, f"orc_read_{suf}").argtypes = [vp, C.c_int, vp, C.c_int64]
            getattr(L, f"orc_write_{suf}").argtypes = [vp, C.c_int, vp, C.c_int64]
        L.orc_relax_f32.argtypes = [C.POINTER(GridView), vp, C.POINTER(NodesView), C.POINTER(RelaxStatsC)]
        L.orc_seed_f32.restype = C.c_int64
        L.orc_seed_f32.argtypes = [C.POINTER(GridView), vp, C.c_int64, vp, vp, vp, vp, vp]
        _lib = L
    return _lib


_INT = {"key": np.int32, "sorted": np.int32, "cstart": np.int32, "nbr": np.int32, "nnb": np.int32,
        "typ": np.uint8, "part": np.uint16, "hist": np.int32}
_PER = {"key": 1, "sorted": 1, "Ps": 4, "nbr": V2M_K, "nnb": 1, "F": 4, "hn": 1, "mv": 1, "V": 3, "pw": 1,
        "P0": 3, "P": 3, "typ": 1, "part": 2, "dirs": 3}


class Oracle:
    """One precision of the restatement: Oracle('f32') or Oracle('f64')."""

    def __init__(self, variant: str = "f32"):
        assert variant in ("f32", "f64")
        self.v = variant
        self.real = np.float32 if variant == "f32" else np.float64
        self.L = load()

    def relax(self, g: Grid, prm: RelaxParams, nd: Nodes) -> RelaxStats:
        """A whole relaxation (float) into nd, like relax_cpu."""
        assert self.v == "f32"
        gv, pv, nv, sv = g.view(), prm.to_c(), nd.view(), RelaxStatsC()
        if self.L.orc_relax_f32(C.byref(gv), C.byref(pv), C.byref(nv), C.byref(sv)) != 0:
            raise RuntimeError("oracle relax failed")
        return RelaxStats.from_c(sv)

    def seed(self, g: Grid, prm: RelaxParams) -> Nodes:
        """tn::seed_cpu restated (float; g.grade required); the nodes carry part3."""
        assert self.v == "f32"
        gv, pv = g.view(), prm.to_c()
        n = self.L.orc_seed_f32(C.byref(gv), C.byref(pv), 0, None, None, None, None, None)
        if n < 0:
            raise RuntimeError("oracle seeding failed")
        nd = Nodes(P=np.zeros((n, 3), np.float32), lab=np.zeros(n, np.uint16), typ=np.zeros(n, np.uint8),
                   part=np.zeros((n, 2), np.uint16))
        nd.part3 = np.zeros(n, np.uint16)
        m = self.L.orc_seed_f32(C.byref(gv), C.byref(pv), n, nd.P.ctypes.data, nd.lab.ctypes.data,
                                nd.typ.ctypes.data, nd.part.ctypes.data, nd.part3.ctypes.data)
        if m != n:
            raise RuntimeError("oracle seeding failed")
        return nd

    def state(self, g: Grid, prm: RelaxParams, nd: Nodes) -> "OracleState":
        return OracleState(self, g, prm, nd)


class OracleState:
    def __init__(self, o: Oracle, g: Grid, prm: RelaxParams, nd: Nodes):
        self.o, self.L, self.v = o, o.L, o.v
        self._keep = (g, nd)     # the oracle reads the grid arrays in place
        gv, pv, nv = g.view(), prm.to_c(), nd.view()
        self.h = getattr(self.L, f"orc_create_{self.v}")(C.byref(gv), C.byref(pv), C.byref(nv))
        if not self.h:
            raise RuntimeError("oracle create failed")
        self.n = nd.size()
        nk, nl = C.c_int64(), C.c_int32()
        getattr(self.L, f"orc_info_{self.v}")(self.h, C.byref(nk), C.byref(nl))
        self.nkeys, self.nlev = nk.value, nl.value

    def __del__(self):
        if getattr(self, "h", None):
            getattr(self.L, f"orc_free_{self.v}")(self.h)
            self.h = None

    def _call(self, f):
        return getattr(self.L, f"orc_{f}_{self.v}")(self.h)

    def rebuild(self):
        self._call("rebuild")

    def force(self):
        self._call("force")

    def move_only(self):
        self._call("move")

    def tail(self) -> bool:
        return bool(self._call("tail"))

    def run(self):
        self._call("run")

    def counts(self) -> dict:
        iv = np.zeros(8, np.int32)
        dv = np.zeros(5, np.float64)
        getattr(self.L, f"orc_counts_{self.v}")(self.h, iv.ctypes.data, dv.ctypes.data)
        return dict(it=int(iv[0]), stopped=int(iv[1]), nhalf=int(iv[2]), nrefresh=int(iv[3]), rebuilds=int(iv[4]),
                    fire_resets=int(iv[5]), fire_dt=dv[0], fire_alpha=dv[1], power=dv[2], mmax=dv[3], p99=dv[4])

    def read(self, name: str) -> np.ndarray:
        dt = _INT.get(name, self.o.real)
        count = self.nkeys + 1 if name == "cstart" else (32 if name == "hist" else self.n * _PER[name])
        out = np.zeros(max(count, 1), dt)
        nb = getattr(self.L, f"orc_read_{self.v}")(self.h, ARR[name], out.ctypes.data, out.nbytes)
        if nb < 0:
            raise RuntimeError(f"oracle read {name} failed")
        return out[:count]

    def write(self, name: str, a: np.ndarray):
        a = np.ascontiguousarray(a, _INT.get(name, self.o.real))
        if getattr(self.L, f"orc_write_{self.v}")(self.h, ARR[name], a.ctypes.data, a.nbytes) != 0:
            raise RuntimeError(f"oracle write {name} failed")


# ---- the differentiable unroll (v2m_unroll_oracle.c), FP64 ----------------------
def _unroll_args(nbr, nnb, typ, G, cs):
    L = load()
    if not hasattr(L, "_unroll_set"):
        vp = C.c_void_p
        for f in ("orc_unroll_forward_f64", "orc_unroll_grad_f64"):
            getattr(L, f).restype = C.c_double
            getattr(L, f).argtypes = [C.c_int, vp, vp, vp, vp, vp, vp, C.c_double, C.c_double, C.c_double, C.c_int,
                                      vp, vp] + ([vp] if f.endswith("grad_f64") else []) + [vp, C.c_int, vp]
        L._unroll_set = True
    nbr = np.ascontiguousarray(nbr, np.int32).reshape(-1)
    nnb = np.ascontiguousarray(nnb, np.int32)
    typ = np.ascontiguousarray(typ, np.uint8)
    G = np.ascontiguousarray(G, np.float64)
    m = np.array(G.shape[::-1], np.int32)          # G is [m2, m1, m0] (x fastest)
    cs = np.ascontiguousarray(cs, np.float64)
    return L, nbr, nnb, typ, G, m, cs


def unroll_dirs(typ, dirs):
    """The taped constraints as the oracle takes them, [n, 4] float64: each
    INTERFACE (kind 1) and JUNCTION (kind 2) node's direction normalised in
    double and rounded to float32 (as v2m_unroll_set_constraints stores it),
    zero rows for other types and zero directions; None stays None."""
    if dirs is None:
        return None
    typ = np.asarray(typ, np.uint8).reshape(-1)
    d = np.asarray(dirs, np.float32).reshape(-1, 3).astype(np.float64)
    r = np.sqrt((d * d).sum(1))
    kind = np.where(typ == 1, 1.0, np.where(typ == 2, 2.0, 0.0))
    kind[r == 0.0] = 0.0
    out = np.zeros((len(typ), 4))
    ok = kind > 0
    out[ok, :3] = (d[ok] / r[ok, None]).astype(np.float32)
    out[:, 3] = kind
    return np.ascontiguousarray(out)


def _dptr(d):
    return None if d is None else d.ctypes.data


def unroll_forward_f64(nbr, nnb, typ, G, cs, fscale, fsurf, dt, K, x0, tape=None, dirs=None):
    """FP64: K unroll steps from x0 [n,3]; returns (xK, loss at xK, tape). With
    tape=None the active bars are decided and recorded; with a tape (uint32
    [K, n]) they are replayed (the taped function). dirs [n, 3]: taped
    constraints (unroll_dirs)."""
    dd = unroll_dirs(typ, dirs)
    L, nbr, nnb, typ, G, m, cs = _unroll_args(nbr, nnb, typ, G, cs)
    x0 = np.ascontiguousarray(x0, np.float64)
    xK = np.zeros_like(x0)
    replay = tape is not None
    tape = np.zeros((K, len(nnb)), np.uint32) if tape is None else np.ascontiguousarray(tape, np.uint32)
    loss = L.orc_unroll_forward_f64(len(nnb), nbr.ctypes.data, nnb.ctypes.data, typ.ctypes.data, m.ctypes.data,
                                    cs.ctypes.data, G.ctypes.data, fscale, fsurf, dt, K, x0.ctypes.data,
                                    xK.ctypes.data, tape.ctypes.data, int(replay), _dptr(dd))
    return xK, loss, tape


def unroll_grad_f64(nbr, nnb, typ, G, cs, fscale, fsurf, dt, K, x0, tape=None, dirs=None):
    """FP64: (loss, dloss/dx0 [n,3], dloss/dG [shape of G], tape) by reverse mode
    of the taped function (recorded here when tape is None); dirs as in
    unroll_forward_f64."""
    dd = unroll_dirs(typ, dirs)
    L, nbr, nnb, typ, G, m, cs = _unroll_args(nbr, nnb, typ, G, cs)
    x0 = np.ascontiguousarray(x0, np.float64)
    gx = np.zeros_like(x0)
    gG = np.zeros_like(G)
    replay = tape is not None
    tape = np.zeros((K, len(nnb)), np.uint32) if tape is None else np.ascontiguousarray(tape, np.uint32)
    loss = L.orc_unroll_grad_f64(len(nnb), nbr.ctypes.data, nnb.ctypes.data, typ.ctypes.data, m.ctypes.data,
                                 cs.ctypes.data, G.ctypes.data, fscale, fsurf, dt, K, x0.ctypes.data, gx.ctypes.data,
                                 gG.ctypes.data, tape.ctypes.data, int(replay), _dptr(dd))
    return loss, gx, gG, tape
