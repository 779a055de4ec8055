"""The host-side truss-list checker (v2m_validate_lists, no device): the
reference's own lists (relax_cpu's rebuild, oracle/_ref) pass, after the build
and after iterations with self-refreshes; mistakes planted in copies of them,
on the CPU, are each reported."""
import numpy as np
import pytest

import cases
from trussnet_b200 import validate_lists
from trussnet_b200.relax import build_positions
from trussnet_b200.types import V2M_K


def ref_lists(ref, name, iters=0):
    g, nd = cases.shells_small() if name == "shells_small" else cases.tpm_small()
    rs = ref.state(g, cases.params(10), nd.copy())
    rs.rebuild()
    for _ in range(iters):
        rs.force()
        rs.tail()
    n = nd.size()
    nbr = rs.read("nbr").reshape(n, V2M_K).copy()
    nnb = rs.read("nnb").astype(np.int32)
    pi = rs.read("P0").reshape(n, 3)
    pj = build_positions(rs.read("Ps"), rs.read("sorted"))
    return nbr, nnb, pi, pj


@pytest.mark.parametrize("name,iters", [("shells_small", 0), ("tpm_small", 0), ("shells_small", 4)])
def test_reference_lists_are_valid(ref, name, iters):
    nbr, nnb, pi, pj = ref_lists(ref, name, iters)
    assert validate_lists(nbr, nnb, pi, pj) == ""


def test_planted_mistakes_are_reported(ref):
    nbr, nnb, pi, pj = ref_lists(ref, "shells_small")
    i = int(np.argmax(nnb >= 5))
    cases_ = []
    a = nbr.copy()
    a[i, [1, 2]] = a[i, [2, 1]]
    cases_.append((a, nnb, "order"))
    a = nbr.copy()
    a[i, 3] = i
    cases_.append((a, nnb, "self-edge"))
    a = nbr.copy()
    a[i, 4] = a[i, 0]
    cases_.append((a, nnb, "repeated"))
    a = nbr.copy()
    a[i, 0] = nnb.size
    cases_.append((a, nnb, "outside [0, n)"))
    b = nnb.copy()
    b[i] = V2M_K + 1
    cases_.append((nbr, b, "length"))
    for lists, lens, what in cases_:
        rep = validate_lists(lists, lens, pi, pj)
        assert rep and what in rep and f"node {i}" in rep, (what, rep)
