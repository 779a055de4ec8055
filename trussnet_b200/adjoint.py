"""The differentiable relaxation unroll behind torch.autograd.Function.

  u = Unroll(nbr, nnb, typ, m, cs, fscale=1.2, fsurf=1.0, dt=0.2, K=50, ckpt=10)
  xK = RelaxUnroll.apply(x0, G, u)          # K taped relaxation steps
  L = EdgeLoss.apply(xK, G, u)              # sum over list entries (l/h - 1)^2
  L.backward()                              # x0.grad, G.grad by the hand-written adjoint

x0 is a float32 CUDA tensor [n, 3]; G the float32 CUDA sizing grid [m2, m1, m0]
(x fastest), value G[c, b, a] at x = (a cs0, b cs1, c cs2). The lists come from
a list build (Session.read('nbr'), Session.read('nnb')) and stay frozen; the
active bars of every step are taped by the forward pass (see
csrc/v2m_adjoint.cu for the step). The reference has no adjoint; its
relaxation step is src/opencl/v2m_particle_body.cl:161-184 / 898-900 of
fangq/trussnet. One backward per forward: the handle keeps the last forward
pass's checkpoints and tape.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib


class Unroll:
    def __init__(self, nbr, nnb, typ, m, cs, fscale=1.2, fsurf=1.0, dt=0.2, K=50, ckpt=10, device=0):
        self.L = _lib.load()
        nbr = np.ascontiguousarray(nbr, np.int32).reshape(-1)
        nnb = np.ascontiguousarray(nnb, np.int32)
        typ = np.ascontiguousarray(typ, np.uint8)
        self.n = int(nnb.size)
        self.m = np.ascontiguousarray(m, np.int32)
        self.cs = np.ascontiguousarray(cs, np.float32)
        self.K, self.ckpt, self.device = int(K), int(ckpt), int(device)
        h = C.c_void_p()
        _lib.check_unroll(self.L.v2m_unroll_create(self.n, nbr.ctypes.data, nnb.ctypes.data, typ.ctypes.data,
                                                   self.m.ctypes.data, self.cs.ctypes.data, float(fscale),
                                                   float(fsurf), float(dt), self.K, self.ckpt, self.device,
                                                   C.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.L.v2m_unroll_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def _ptr(t):
        assert t.is_cuda and t.is_contiguous() and str(t.dtype) == "torch.float32"
        return t.data_ptr()

    @staticmethod
    def _sync():
        import torch
        torch.cuda.current_stream().synchronize()

    def forward(self, x0, G, replay=False):
        import torch
        xK = torch.empty_like(x0)
        self._sync()
        _lib.check_unroll(self.L.v2m_unroll_forward(self.h, self._ptr(x0), self._ptr(G), self._ptr(xK), int(replay)))
        return xK

    def loss(self, x, G) -> float:
        self._sync()
        out = C.c_double()
        _lib.check_unroll(self.L.v2m_unroll_loss(self.h, self._ptr(x), self._ptr(G), C.byref(out)))
        return out.value

    def loss_backward(self, x, G, gscale=1.0):
        import torch
        gx = torch.empty_like(x)
        gG = torch.empty_like(G)
        self._sync()
        _lib.check_unroll(self.L.v2m_unroll_loss_backward(self.h, self._ptr(x), self._ptr(G), float(gscale),
                                                          self._ptr(gx), self._ptr(gG), 0))
        return gx, gG

    def backward(self, G, gxK):
        import torch
        gxK = gxK.contiguous()
        gx0 = torch.empty_like(gxK)
        gG = torch.empty_like(G)
        self._sync()
        _lib.check_unroll(self.L.v2m_unroll_backward(self.h, self._ptr(G), self._ptr(gxK), self._ptr(gx0),
                                                     self._ptr(gG), None))
        return gx0, gG

    def set_constraints(self, dirs=None):
        """Taped constraints (see v2m_unroll_set_constraints): dirs float [n, 3],
        each INTERFACE node's interface normal and each JUNCTION node's
        junction-line direction (Session.read('dirs')); None removes them."""
        if dirs is None:
            _lib.check_unroll(self.L.v2m_unroll_set_constraints(self.h, None))
            return
        d = np.ascontiguousarray(dirs, np.float32).reshape(-1)
        if d.size != 3 * self.n:
            raise ValueError("dirs needs 3 values per node")
        _lib.check_unroll(self.L.v2m_unroll_set_constraints(self.h, d.ctypes.data))

    def tape(self) -> np.ndarray:
        out = np.zeros((self.K, self.n), np.uint32)
        _lib.check_unroll(self.L.v2m_unroll_tape(self.h, out.ctypes.data, out.size))
        return out

    def timing(self):
        a, b = C.c_float(), C.c_float()
        _lib.check_unroll(self.L.v2m_unroll_timing(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value


def _function_classes():
    import torch

    class RelaxUnroll(torch.autograd.Function):
        """x0 [n,3], G -> xK after the unroll's K taped steps; adjoint in backward."""

        @staticmethod
        def forward(ctx, x0, G, unroll):
            ctx.unroll = unroll
            ctx.save_for_backward(G)
            return unroll.forward(x0.detach().contiguous(), G.detach().contiguous())

        @staticmethod
        def backward(ctx, gxK):
            (G,) = ctx.saved_tensors
            gx0, gG = ctx.unroll.backward(G.detach().contiguous(), gxK)
            return gx0, gG, None

    class EdgeLoss(torch.autograd.Function):
        """x [n,3], G -> sum over list entries of (l_ij / h_ij - 1)^2 (float64 scalar)."""

        @staticmethod
        def forward(ctx, x, G, unroll):
            ctx.unroll = unroll
            ctx.save_for_backward(x, G)
            return torch.tensor(unroll.loss(x.detach().contiguous(), G.detach().contiguous()), dtype=torch.float64,
                                device=x.device)

        @staticmethod
        def backward(ctx, g):
            x, G = ctx.saved_tensors
            gx, gG = ctx.unroll.loss_backward(x.detach().contiguous(), G.detach().contiguous(), float(g))
            return gx, gG, None

    return RelaxUnroll, EdgeLoss


class _Lazy:
    """The Function classes, created on first use (torch is imported lazily)."""

    def __getattr__(self, name):
        r, e = _function_classes()
        globals()["RelaxUnroll"], globals()["EdgeLoss"] = r, e
        return {"RelaxUnroll": r, "EdgeLoss": e}[name]


def __getattr__(name):
    if name in ("RelaxUnroll", "EdgeLoss"):
        return getattr(_Lazy(), name)
    raise AttributeError(name)


def unrolled_loss(x0, G, unroll):
    """EdgeLoss(RelaxUnroll(x0, G)): the loss after K steps, differentiable in x0 and G."""
    import sys
    mod = sys.modules[__name__]
    return mod.EdgeLoss.apply(mod.RelaxUnroll.apply(x0, G, unroll), G, unroll)


def optimize_sizing(unroll, x0, G0, steps=20, step=0.05, hmin=None, hmax=None):
    """Sizing by gradient: descent on the sizing grid G so that the nodes after
    the K-step unroll from x0 make bars of their target lengths (the unroll's
    edge loss, sum over list entries of (l_ij / h_ij - 1)^2). Each step
    evaluates the loss and dL/dG by the hand-written adjoint (RelaxUnroll +
    EdgeLoss), moves G by `step` times the largest grid value against the
    gradient normalised by its largest magnitude, and clamps G to
    [hmin, hmax] (default: G0's range). Returns (G, losses): the final grid
    and the loss before each step and after the last."""
    import torch
    G = G0.detach().clone().contiguous()
    lo = float(G0.min()) if hmin is None else float(hmin)
    hi = float(G0.max()) if hmax is None else float(hmax)
    scale = step * hi
    losses = []
    for _ in range(steps):
        Gv = G.clone().requires_grad_(True)
        L = unrolled_loss(x0, Gv, unroll)
        L.backward()
        losses.append(float(L.detach()))
        g = Gv.grad
        with torch.no_grad():
            G = (G - scale * g / g.abs().max().clamp_min(1e-30)).clamp_(lo, hi).contiguous()
    with torch.no_grad():
        losses.append(float(unrolled_loss(x0, G, unroll)))
    return G, losses


def optimize_positions(unroll, x0, G, steps=20, step=0.05):
    """Node positions by gradient: descent on the starting positions x0 of the
    unroll (the relaxation's state fed to a mesh-quality optimiser) against
    the same edge loss after K steps, each node moved by at most `step` times
    its local grid spacing. Returns (x, losses)."""
    import torch
    x = x0.detach().clone().contiguous()
    cell = float(min(unroll.cs))
    losses = []
    for _ in range(steps):
        xv = x.clone().requires_grad_(True)
        L = unrolled_loss(xv, G, unroll)
        L.backward()
        losses.append(float(L.detach()))
        g = xv.grad
        with torch.no_grad():
            x = (x - step * cell * g / g.norm(dim=1).max().clamp_min(1e-30)).contiguous()
    with torch.no_grad():
        losses.append(float(unrolled_loss(x, G, unroll)))
    return x, losses
