"""CPU: the FP64 reverse-mode gradient of the relaxation unroll
(oracle/v2m_unroll_oracle.c) against central finite differences of the same
FP64 unroll (the taped function: active bars replayed from the unperturbed
forward pass), on a small volume: the checker of the CUDA adjoint is itself
checked first."""
import numpy as np
import pytest

from oracle.oracle import Oracle, unroll_dirs, unroll_forward_f64, unroll_grad_f64
from trussnet_b200 import synth
from trussnet_b200.types import RelaxParams


@pytest.fixture(scope="module")
def small():
    g, nd, G, cs = synth.ellipsoids_adjoint(dim=40, m=12, density=1.0, seed=3)
    s = Oracle("f32").state(g, RelaxParams(max_iters=1), nd)
    s.rebuild()
    return nd, G, cs, s.read("nbr"), s.read("nnb")


@pytest.mark.parametrize("K", [1, 6])
def test_fp64_gradient_matches_finite_differences(small, K):
    nd, G, cs, nbr, nnb = small
    x0 = nd.P.astype(np.float64)
    args = (nbr, nnb, nd.typ, G.astype(np.float64), cs, 1.2, 1.0, 0.2, K)
    loss, gx, gG, tape = unroll_grad_f64(*args, x0)
    _, l2, tape2 = unroll_forward_f64(*args, x0)
    assert loss == l2 and np.array_equal(tape, tape2)
    rng = np.random.default_rng(0)
    eps = 1e-6
    for _ in range(4):
        d = rng.standard_normal(x0.shape)
        lp = unroll_forward_f64(*args[:-1], K, x0 + eps * d, tape)[1]
        lm = unroll_forward_f64(*args[:-1], K, x0 - eps * d, tape)[1]
        fd = (lp - lm) / (2 * eps)
        an = float(np.sum(gx * d))
        assert abs(fd - an) <= 1e-5 * max(1.0, abs(an)), (fd, an)
        dG = rng.standard_normal(G.shape)
        Gp = (G.astype(np.float64) + eps * dG, G.astype(np.float64) - eps * dG)
        lp = unroll_forward_f64(nbr, nnb, nd.typ, Gp[0], cs, 1.2, 1.0, 0.2, K, x0, tape)[1]
        lm = unroll_forward_f64(nbr, nnb, nd.typ, Gp[1], cs, 1.2, 1.0, 0.2, K, x0, tape)[1]
        fd = (lp - lm) / (2 * eps)
        an = float(np.sum(gG * dG))
        assert abs(fd - an) <= 1e-5 * max(1.0, abs(an)), (fd, an)


@pytest.fixture(scope="module")
def constrained():
    """tpm_small after 3 relaxation iterations (its seeds classified as
    INTERFACE and JUNCTION nodes by their first moves), its lists, the oracle's
    constraint directions there and a seeded sizing grid over the box."""
    import types
    import cases
    g, nd = cases.tpm_small()
    s = Oracle("f32").state(g, RelaxParams(max_iters=3), nd)
    s.run()
    st = types.SimpleNamespace(P=s.read("P").reshape(-1, 3), typ=s.read("typ"))
    dims = (g.nx, g.ny, g.nz)
    m = 10
    G = synth.sizing_grid((m, m, m), 1.4, 2.0, seed=5)
    cs = tuple((d - 1) / (m - 1) for d in dims)
    return st, G, cs, s.read("nbr"), s.read("nnb"), s.read("dirs").reshape(-1, 3)


def test_oracle_constraint_directions(constrained):
    """Unit directions on every INTERFACE and JUNCTION seed, zero elsewhere."""
    nd, _, _, _, _, dirs = constrained
    r = np.linalg.norm(dirs.astype(np.float64), axis=1)
    con = (nd.typ == 1) | (nd.typ == 2)
    assert con.sum() > 1000 and (nd.typ == 2).sum() > 100
    assert np.all(np.abs(r[con] - 1.0) < 1e-6)
    assert np.all(r[~con] == 0.0)


@pytest.mark.parametrize("K", [1, 6])
def test_fp64_constrained_unroll(constrained, K):
    """Taped constraints: INTERFACE nodes move in their tangent planes, JUNCTION
    nodes along their lines, CORNER nodes stay; the reverse-mode gradient of the
    constrained unroll matches its central finite differences."""
    nd, G, cs, nbr, nnb, dirs = constrained
    x0 = nd.P.astype(np.float64)
    args = (nbr, nnb, nd.typ, G.astype(np.float64), cs, 1.2, 1.0, 0.2, K)
    xK, loss, tape = unroll_forward_f64(*args, x0, dirs=dirs)
    d = xK - x0
    free = unroll_forward_f64(*args, x0)[0] - x0
    # the directions are unit to float32 rounding, so a projected step keeps
    # about 1e-7 of the unprojected one along them
    tol = 1e-6 * np.abs(free).max()
    u = unroll_dirs(nd.typ, dirs)[:, :3]
    moved = np.linalg.norm(d, axis=1)
    itf, jun = nd.typ == 1, nd.typ == 2
    assert moved[itf].max() > 1e-2 and moved[jun].max() > 1e-2
    assert np.abs((d[itf] * u[itf]).sum(1)).max() <= tol
    assert np.linalg.norm(np.cross(d[jun], u[jun]), axis=1).max() <= tol
    assert np.all(d[nd.typ == 3] == 0.0)
    assert np.abs((free[itf] * u[itf]).sum(1)).max() > 1e-2   # the constraint changes the motion
    loss2, gx, gG, _ = unroll_grad_f64(*args, x0, tape, dirs=dirs)
    assert loss2 == loss
    rng = np.random.default_rng(2)
    eps = 1e-6
    for _ in range(3):
        v = rng.standard_normal(x0.shape)
        lp = unroll_forward_f64(*args, x0 + eps * v, tape, dirs=dirs)[1]
        lm = unroll_forward_f64(*args, x0 - eps * v, tape, dirs=dirs)[1]
        fd, an = (lp - lm) / (2 * eps), float(np.sum(gx * v))
        assert abs(fd - an) <= 1e-5 * max(1.0, abs(an)), (fd, an)
        dG = rng.standard_normal(G.shape)
        G64 = G.astype(np.float64)
        lp = unroll_forward_f64(nbr, nnb, nd.typ, G64 + eps * dG, cs, 1.2, 1.0, 0.2, K, x0, tape, dirs=dirs)[1]
        lm = unroll_forward_f64(nbr, nnb, nd.typ, G64 - eps * dG, cs, 1.2, 1.0, 0.2, K, x0, tape, dirs=dirs)[1]
        fd, an = (lp - lm) / (2 * eps), float(np.sum(gG * dG))
        assert abs(fd - an) <= 1e-5 * max(1.0, abs(an)), (fd, an)
