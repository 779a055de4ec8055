"""CPU: the FP64 reverse-mode gradient of the relaxation unroll
(oracle/v2m_unroll_oracle.c) against central finite differences of the same
FP64 unroll (the taped function: active bars replayed from the unperturbed
forward pass), on a small volume: the checker of the CUDA adjoint is itself
checked first."""
import numpy as np
import pytest

from oracle.oracle import Oracle, unroll_forward_f64, unroll_grad_f64
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
