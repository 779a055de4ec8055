"""GPU: the hand-written adjoint of the relaxation unroll (csrc/v2m_adjoint.cu)
behind torch.autograd.Function (trussnet_b200/adjoint.py).

Checks, on the taped function (active bars recorded by the GPU forward pass and
replayed by every evaluation):
  * the loss and the gradients w.r.t. the node positions and the sizing grid
    against the FP64 reverse-mode gradient (oracle/v2m_unroll_oracle.c):
    relative error (2-norm) <= 1e-4;
  * directional derivatives against FP64 central finite differences with
    eps = 1e-3: along the gradient direction, relative error <= 1e-4; along
    random directions, error <= 1e-4 of the gradient's norm;
  * run-to-run bit-identical gradients (fixed-point accumulation);
  * the adjoint costs <= 3x a forward step (backward time / K against
    forward time / K, both CUDA-event timed).
"""
import numpy as np
import pytest

from oracle.oracle import unroll_forward_f64, unroll_grad_f64
from cases import first_diff, same_bits
from trussnet_b200 import Session, synth
from trussnet_b200.types import RelaxParams

pytestmark = pytest.mark.gpu

FSCALE, FSURF, DT = 1.2, 1.0, 0.2


def setup(dim, m, K, ckpt, density=1.66, seed=0):
    import torch
    from trussnet_b200.adjoint import Unroll
    g, nd, G, cs = synth.ellipsoids_adjoint(dim=dim, m=m, density=density, seed=seed)
    with Session(g, RelaxParams(max_iters=1), nd) as s:
        s.rebuild()
        nbr, nnb = s.read("nbr"), s.read("nnb")
    u = Unroll(nbr, nnb, nd.typ, G.shape[::-1], cs, FSCALE, FSURF, DT, K, ckpt)
    x0 = torch.tensor(nd.P, device="cuda")
    Gt = torch.tensor(G, device="cuda")
    return u, x0, Gt, nd, nbr, nnb, G, cs


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("cfg", [(48, 16, 12, 5), (128, 64, 50, 10)], ids=["small", "ellipsoids128_K50"])
def test_adjoint_against_fp64_and_fd(cfg, cuda_lib, record_property):
    dim, m, K, ckpt = cfg
    u, x0, Gt, nd, nbr, nnb, G, cs = setup(dim, m, K, ckpt)
    xK = u.forward(x0, Gt)
    loss = u.loss(xK, Gt)
    gxK, gG1 = u.loss_backward(xK, Gt)
    gx0, gG2 = u.backward(Gt, gxK)
    gx0 = gx0.cpu().numpy().astype(np.float64)
    gG = (gG1 + gG2).cpu().numpy().astype(np.float64)
    tape = u.tape()
    args = (nbr, nnb, nd.typ, G.astype(np.float64), cs, FSCALE, FSURF, DT, K)
    L64, gx64, gG64, _ = unroll_grad_f64(*args, nd.P.astype(np.float64), tape)
    e_loss = abs(loss - L64) / abs(L64)
    e_x, e_G = rel(gx0, gx64), rel(gG, gG64)
    record_property("loss_rel_err", e_loss)
    record_property("grad_x_rel_err_vs_fp64", e_x)
    record_property("grad_G_rel_err_vs_fp64", e_G)
    assert e_loss <= 1e-4 and e_x <= 1e-4 and e_G <= 1e-4, (e_loss, e_x, e_G)
    # central finite differences (FP64, the same tape), eps = 1e-3: along the
    # gradient's own direction (relative to the directional derivative), and
    # along random directions (relative to |g|: a random unit direction projects
    # a gradient of norm |g| down to about |g| / sqrt(dimension), so its own
    # value is no scale for the error)
    rng = np.random.default_rng(1)
    eps = 1e-3
    x64, G64 = nd.P.astype(np.float64), G.astype(np.float64)

    def fd_x(d):
        lp = unroll_forward_f64(*args, x64 + eps * d, tape)[1]
        lm = unroll_forward_f64(*args, x64 - eps * d, tape)[1]
        return (lp - lm) / (2 * eps)

    def fd_G(d):
        lp = unroll_forward_f64(nbr, nnb, nd.typ, G64 + eps * d, cs, FSCALE, FSURF, DT, K, x64, tape)[1]
        lm = unroll_forward_f64(nbr, nnb, nd.typ, G64 - eps * d, cs, FSCALE, FSURF, DT, K, x64, tape)[1]
        return (lp - lm) / (2 * eps)

    along = 0.0
    for g, fd in ((gx0, fd_x), (gG, fd_G)):
        d = g / np.linalg.norm(g)
        an = float(np.sum(g * d))
        along = max(along, abs(fd(d) - an) / abs(an))
    rand = 0.0
    for _ in range(2):
        for g, fd, shape in ((gx0, fd_x, nd.P.shape), (gG, fd_G, G.shape)):
            d = rng.standard_normal(shape)
            d /= np.linalg.norm(d)
            rand = max(rand, abs(fd(d) - float(np.sum(g * d))) / np.linalg.norm(g))
    record_property("fd_rel_err_along_gradient", along)
    record_property("fd_err_random_over_gradient_norm", rand)
    assert along <= 1e-4 and rand <= 1e-4, (along, rand)


def test_adjoint_deterministic_and_cost(cuda_lib, record_property):
    u, x0, Gt, *_ = setup(128, 64, 50, 10)
    outs = []
    for _ in range(2):
        xK = u.forward(x0, Gt)
        gxK, _ = u.loss_backward(xK, Gt)
        gx0, gG = u.backward(Gt, gxK)
        outs.append((gx0.cpu().numpy(), gG.cpu().numpy()))
    assert np.array_equal(outs[0][0].view(np.uint32), outs[1][0].view(np.uint32))
    assert np.array_equal(outs[0][1].view(np.uint32), outs[1][1].view(np.uint32))
    # timing: warm runs
    for _ in range(3):
        xK = u.forward(x0, Gt)
        gxK, _ = u.loss_backward(xK, Gt)
        u.backward(Gt, gxK)
    fwd, bwd = u.timing()
    ratio = bwd / fwd
    record_property("forward_ms_per_step", fwd / 50)
    record_property("adjoint_ms_per_step", bwd / 50)
    record_property("adjoint_over_forward", ratio)
    assert ratio <= 3.0, ratio


def test_autograd_function(cuda_lib):
    import torch
    from trussnet_b200.adjoint import unrolled_loss
    u, x0, Gt, *_ = setup(48, 16, 12, 5)
    x = x0.clone().requires_grad_(True)
    G = Gt.clone().requires_grad_(True)
    L = unrolled_loss(x, G, u)
    L.backward()
    xK = u.forward(x0, Gt)
    gxK, gG1 = u.loss_backward(xK, Gt)
    gx0, gG2 = u.backward(Gt, gxK)
    assert torch.equal(x.grad, gx0)
    assert torch.allclose(G.grad, gG1 + gG2, rtol=0, atol=0)
    assert float(L.detach()) == pytest.approx(u.loss(xK, Gt), rel=0, abs=0)


def test_sizing_by_gradient_lowers_the_loss(cuda_lib):
    """The adjoint's consumer: descent on the sizing grid through the K-step
    unroll (adjoint.optimize_sizing) lowers the edge loss after K steps; the
    same for descent on the starting positions (adjoint.optimize_positions)."""
    from trussnet_b200.adjoint import optimize_positions, optimize_sizing
    u, x0, Gt, nd, nbr, nnb, G, cs = setup(48, 16, 12, 5)
    G1, lg = optimize_sizing(u, x0, Gt, steps=12, step=0.02)
    assert min(lg[1:]) < lg[0] and lg[-1] < 0.99 * lg[0], lg
    assert float(G1.min()) >= float(Gt.min()) and float(G1.max()) <= float(Gt.max())
    x1, lx = optimize_positions(u, x0, Gt, steps=12, step=0.02)
    assert lx[-1] < lx[0], lx
    u.close()


def test_constrained_adjoint(cuda_lib, record_property):
    """Taped constraints (Unroll.set_constraints): the session's constraint
    directions (V2M_ARR_DIRS) after 3 relaxation iterations of tpm_small equal
    the oracle's bit for bit; the constrained unroll keeps INTERFACE nodes in
    their tangent planes and JUNCTION nodes on their lines; its loss and
    gradients match the FP64 constrained unroll (relative 2-norm <= 1e-4) and
    FP64 finite differences along the gradient (<= 1e-4); removing the
    constraints gives back the unconstrained unroll bit for bit."""
    import cases
    import torch
    from oracle.oracle import Oracle
    from trussnet_b200.adjoint import Unroll
    g, nd = cases.tpm_small()
    prm = RelaxParams(max_iters=3)
    o = Oracle("f32").state(g, prm, nd.copy())
    o.run()
    with Session(g, prm, nd.copy()) as s:
        s.run()
        P, typ = s.read("P").reshape(-1, 3), s.read("typ")
        nbr, nnb, dirs = s.read("nbr"), s.read("nnb"), s.read("dirs").reshape(-1, 3)
    assert same_bits(P, o.read("P").reshape(-1, 3)) and same_bits(typ, o.read("typ"))
    d = first_diff(dirs, o.read("dirs").reshape(-1, 3))
    assert d is None, f"constraint directions vs the oracle: {d}"
    m, K = 10, 12
    G = synth.sizing_grid((m, m, m), 1.4, 2.0, seed=5)
    cs = tuple((v - 1) / (m - 1) for v in (g.nx, g.ny, g.nz))
    u = Unroll(nbr, nnb, typ, G.shape[::-1], cs, FSCALE, FSURF, DT, K, 5)
    x0, Gt = torch.tensor(P, device="cuda"), torch.tensor(G, device="cuda")
    free = u.forward(x0, Gt).cpu().numpy()
    u.set_constraints(dirs)
    from trussnet_b200._lib import V2mError
    with pytest.raises(V2mError):
        u.forward(x0, Gt, replay=True)   # the constraints invalidate the tape
    xK = u.forward(x0, Gt)
    loss = u.loss(xK, Gt)
    gxK, gG1 = u.loss_backward(xK, Gt)
    gx0, gG2 = u.backward(Gt, gxK)
    disp = xK.cpu().numpy().astype(np.float64) - P
    itf, jun = typ == 1, typ == 2
    un = dirs.astype(np.float64) / np.maximum(np.linalg.norm(dirs.astype(np.float64), axis=1), 1e-30)[:, None]
    along = np.abs((disp[itf] * un[itf]).sum(1)).max()
    across = np.linalg.norm(np.cross(disp[jun], un[jun]), axis=1).max()
    record_property("interface_normal_motion_max", float(along))
    record_property("junction_off_line_motion_max", float(across))
    # float32 positions: each of the K steps rounds x + increment (|x| < 44: half
    # an ulp is 1.9e-6), against free motions of order 1e-2
    assert along <= 1e-4 and across <= 1e-4, (along, across)
    assert np.abs(((free - P)[itf] * un[itf]).sum(1)).max() > 1e-2
    assert np.all(disp[typ == 3] == 0.0)
    tape = u.tape()
    args = (nbr, nnb, typ, G.astype(np.float64), cs, FSCALE, FSURF, DT, K)
    x64 = P.astype(np.float64)
    L64, gx64, gG64, _ = unroll_grad_f64(*args, x64, tape, dirs=dirs)
    gx = gx0.cpu().numpy().astype(np.float64)
    gG = (gG1 + gG2).cpu().numpy().astype(np.float64)
    e_loss, e_x, e_G = abs(loss - L64) / abs(L64), rel(gx, gx64), rel(gG, gG64)
    record_property("constrained_loss_rel_err", e_loss)
    record_property("constrained_grad_x_rel_err_vs_fp64", e_x)
    record_property("constrained_grad_G_rel_err_vs_fp64", e_G)
    assert e_loss <= 1e-4 and e_x <= 1e-4 and e_G <= 1e-4, (e_loss, e_x, e_G)
    eps = 1e-3
    dx = gx / np.linalg.norm(gx)
    lp = unroll_forward_f64(*args, x64 + eps * dx, tape, dirs=dirs)[1]
    lm = unroll_forward_f64(*args, x64 - eps * dx, tape, dirs=dirs)[1]
    an = float(np.sum(gx * dx))
    e_fd = abs((lp - lm) / (2 * eps) - an) / abs(an)
    record_property("constrained_fd_rel_err_along_gradient", e_fd)
    assert e_fd <= 1e-4, e_fd
    u.set_constraints(None)
    again = u.forward(x0, Gt).cpu().numpy()
    assert same_bits(again, free)
    u.close()
