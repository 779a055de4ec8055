"""pyv2mesh's points-mode call on the B200 path.

`points` mirrors v2mesh.points (pyv2mesh/v2mesh/__init__.py:185-199 of
fangq/trussnet): a label volume indexed vol[x, y, z] in, the relaxed nodes of
the mesher out (before tessellation), with the same keys. Here the grid build,
the seeding and the relaxation all run on the device in one call
(points_cl: one upload of the labels, one copy back of the nodes), bit for bit
the reference's CPU stages. `optimize_sizing` is the sizing-by-gradient step
the reference does not have: descent on a sizing grid through the
differentiable relaxation unroll (trussnet_b200.adjoint). `dump_nodes` /
`load_nodes` write and read the relaxed nodes in the reference's node-dump
format (its --dump-nodes), the on-disk hand-off to its tessellation tools.
"""
from __future__ import annotations

import numpy as np

from .relax import points_cl
from .types import V2M_NOLAB, GridParams, RelaxParams


def _grid_params(opts) -> GridParams:
    p = GridParams()
    size = opts.pop("size", None)
    if size is not None:
        p.hbase = float(size)
    for key, name in (("hmin", "hmin"), ("hmax", "hmax"), ("K", "K"), ("grad", "g"), ("sigma", "sigma"),
                      ("sigma_thin", "sigma_thin"), ("thick", "thick"), ("thin_floor", "thin_floor"),
                      ("preserve", "preserve")):
        if key in opts:
            setattr(p, name, float(opts.pop(key)))
    lsize = opts.pop("lsize", None)
    if lsize is not None:
        if isinstance(lsize, dict):
            n = max(lsize) + 1
            hl = [0.0] * n
            for k, v in lsize.items():
                hl[int(k)] = float(v)
        else:   # a sequence for labels 1, 2, ...
            hl = [0.0] + [float(v) for v in lsize]
        p.hlab = tuple(hl)
    return p


def _relax_params(opts) -> RelaxParams:
    p = RelaxParams()
    for key, name in (("iters", "max_iters"), ("dt", "dt"), ("fscale", "fscale"), ("fsurf", "fsurf"),
                      ("snap", "snap"), ("dptol", "dptol"), ("fire_dtmax", "fire_dtmax"), ("jseed", "jseed")):
        if key in opts:
            v = opts.pop(key)
            setattr(p, name, int(v) if name == "max_iters" else float(v))
    relax = opts.pop("relax", None)
    if relax is not None:
        p.fire = relax == "fire"
    if "trap" in opts:
        p.voxel_trap = opts.pop("trap") == "voxel"
    if "corners" in opts:
        p.corners = bool(opts.pop("corners"))
    return p


def points(vol, *, voxelsize=None, gpuid: int = 1, **opts):
    """The mesher's relaxed nodes, before tessellation (v2mesh.points).

    vol: 3-D integer labels indexed vol[x, y, z] (0 = exterior). voxelsize: a
    float or three (mm, default 1). opts: size, hmin, hmax, lsize, K, grad,
    sigma, sigma_thin, thick, thin_floor, preserve (the grid); iters, dt,
    fscale, fsurf, snap, dptol, relax ('fire' | 'jacobi'), trap ('voxel'),
    jseed, corners (the seeding and the relaxation). gpuid: 1-based device.
    Returns node (N, 3), label (N,), type (N,), partner (N, 3) (-1 = none) and
    info, as v2mesh.points.
    """
    vol = np.asarray(vol)
    if vol.ndim != 3:
        raise ValueError("points: a 3-D label volume vol[x, y, z]")
    opts = dict(opts)
    vs = (1.0, 1.0, 1.0) if voxelsize is None else tuple(np.broadcast_to(np.asarray(voxelsize, float), (3,)))
    gp = _grid_params(opts)
    rp = _relax_params(opts)
    if opts:
        raise TypeError(f"points: options not supported on the device path: {sorted(opts)}")
    L = np.ascontiguousarray(vol.astype(np.uint16).transpose(2, 1, 0))   # x fastest
    nd, part3, st = points_cl(L, vs, gp, rp, device=int(gpuid) - 1)
    partner = np.stack([nd.part[:, 0], nd.part[:, 1], part3], axis=1).astype(np.int64)
    partner[partner == V2M_NOLAB] = -1
    info = {"iters": st.iters, "rebuilds": st.rebuilds, "fire_resets": st.fire_resets, "last_move": st.last_move,
            "types": [st.n_interior, st.n_interface, st.n_junction, st.n_corner]}
    return {"node": nd.P.astype(np.float64), "label": nd.lab.astype(np.int64), "type": nd.typ.astype(np.int64),
            "partner": partner, "info": info}


def optimize_sizing(nbr, nnb, typ, x0, G0, cs, *, K=50, ckpt=10, steps=20, step=0.05, fscale=1.2, fsurf=1.0,
                    dt=0.2, gpuid: int = 1):
    """Sizing by gradient (no counterpart in v2mesh): descent on the sizing grid
    G0 (float32 [m2, m1, m0], x fastest, value at (a cs0, b cs1, c cs2)) so that
    the nodes x0 (N, 3) relaxed K steps on the frozen lists nbr / nnb make bars
    of their target lengths (trussnet_b200.adjoint.optimize_sizing). Returns
    (G, losses) as numpy arrays / floats."""
    import torch
    from .adjoint import Unroll, optimize_sizing as _opt
    dev = int(gpuid) - 1
    G0 = np.ascontiguousarray(G0, np.float32)
    u = Unroll(nbr, nnb, typ, G0.shape[::-1], cs, fscale, fsurf, dt, K, ckpt, device=dev)
    try:
        x = torch.tensor(np.ascontiguousarray(x0, np.float32), device=f"cuda:{dev}")
        G = torch.tensor(G0, device=f"cuda:{dev}")
        Gout, losses = _opt(u, x, G, steps=steps, step=step)
        return Gout.cpu().numpy(), losses
    finally:
        u.close()


# ---- the node dump: the relaxation's on-disk hand-off --------------------------------
_DUMP_FIELDS = (("P", "float32", 3), ("Label", "uint16", 1), ("Type", "uint8", 1), ("Partner", "uint16", 2))


def dump_nodes(path, nodes) -> None:
    """Write nodes as v2mesh's node dump (``--dump-nodes``,
    src/v2m_pipeline.cpp:58-73 of fangq/trussnet; read by its
    tools/v2mview.py): one JSON header line {name: [dtype, shape, byte
    offset]} -- compact, keys in sorted order as the reference's JSON library
    writes them -- then the raw little-endian arrays in the order P float32
    [n, 3], Label uint16 [n], Type uint8 [n], Partner uint16 [n, 2], the
    offsets counted from the end of the header line. (The reference's dump has
    no part3: a CORNER node's fourth label stays in memory.)"""
    import json
    n = int(nodes.size())
    arrays = (np.ascontiguousarray(nodes.P, np.float32).reshape(n, 3), np.ascontiguousarray(nodes.lab, np.uint16),
              np.ascontiguousarray(nodes.typ, np.uint8), np.ascontiguousarray(nodes.part, np.uint16).reshape(n, 2))
    head, off = {}, 0
    for (name, dt, w), a in zip(_DUMP_FIELDS, arrays):
        head[name] = [dt, [n, w] if w > 1 else [n], off]
        off += a.nbytes
    with open(path, "wb") as f:
        f.write(json.dumps(head, separators=(",", ":"), sort_keys=True).encode())
        f.write(b"\n")
        for a in arrays:
            f.write(a.astype(a.dtype.newbyteorder("<"), copy=False).tobytes())


def load_nodes(path):
    """Nodes from a v2mesh node dump (the reference's or dump_nodes'): P, lab,
    typ, part as tn::Nodes holds them."""
    import json
    from .types import Nodes
    with open(path, "rb") as f:
        head = json.loads(f.readline())
        buf = f.read()
    out = {}
    for name, dt, w in _DUMP_FIELDS:
        dtype, shape, off = head[name]
        cnt = int(np.prod(shape))
        out[name] = np.frombuffer(buf, dtype=np.dtype(dtype).newbyteorder("<"), count=cnt, offset=int(off)).reshape(shape)
    n = int(head["Label"][1][0])
    return Nodes(P=out["P"].astype(np.float32).reshape(n, 3).copy(), lab=out["Label"].astype(np.uint16).copy(),
                 typ=out["Type"].astype(np.uint8).copy(), part=out["Partner"].astype(np.uint16).reshape(n, 2).copy())
