"""GPU parity on shape input (analytic fields, gm < 0): the CUDA relaxation
against the reference's own relax_cpu (oracle/_ref) on grids whose fields are
programs compiled by the reference's shape compiler from JSON scenes
(tests/cases.py SHAPE_SCENES). Every point query of the move then evaluates the
labels' signed distance programs (src/opencl/v2m_sdf_body.cl) instead of the
sampled fields.

The bar is bit-exact, as for the sampled fields: positions, types, partner
labels and the iteration statistics.
"""
import numpy as np
import pytest

import cases
from cases import first_diff
from trussnet_b200 import Session, relax_cl

pytestmark = pytest.mark.gpu

SCENES = list(cases.SHAPE_SCENES)


def check_same(nd, rd):
    for a in ("P", "typ", "part"):
        d = first_diff(getattr(nd, a), getattr(rd, a))
        assert d is None, f"{a}: {d}"


@pytest.mark.parametrize("name", SCENES)
def test_shape_relax_bit_exact(name, ref, cuda_lib):
    g, nd = cases.shape_case(ref, name)
    prm = cases.params(30)
    rd = nd.copy()
    rs = ref.relax_cpu(g, prm, rd)
    st = relax_cl(g, prm, nd)
    check_same(nd, rd)
    assert (st.iters, st.rebuilds, st.fire_resets) == (rs.iters, rs.rebuilds, rs.fire_resets)
    assert st.last_move == rs.last_move and st.last_p99 == rs.last_p99
    assert (st.n_interface, st.n_junction) == (rs.n_interface, rs.n_junction)


@pytest.mark.parametrize("name", ["mcx", "split"])
@pytest.mark.parametrize("fire", [0, 1])
def test_shape_iterations_bit_exact(name, fire, ref, cuda_lib):
    """Stage by stage: after each iteration's move the node arrays agree."""
    g, nd = cases.shape_case(ref, name)
    prm = cases.params(10, fire=fire)
    rs = ref.state(g, prm, nd.copy())
    rs.rebuild()
    with Session(g, prm, nd.copy()) as s:
        s.rebuild()
        for it in range(4):
            rs.force()
            rs.tail()
            s.force()
            s.step_tail()
            for a in ("P", "typ", "part", "mv", "hn"):
                d = first_diff(s.read(a), rs.read(a))
                assert d is None, f"iteration {it}, {a}: {d}"


def test_shape_exact_csg(ref, cuda_lib):
    """Crease blending off: the min / max of exact CSG, with T-junctions."""
    g, nd = cases.shape_case(ref, "mcx", exact=True)
    prm = cases.params(25, fire=0)
    rd = nd.copy()
    ref.relax_cpu(g, prm, rd)
    relax_cl(g, prm, nd)
    check_same(nd, rd)


def test_shape_batch_equals_single(ref, cuda_lib):
    """A shape volume batched with a label volume relaxes as it does alone."""
    from trussnet_b200 import relax_cl_batch
    g1, n1 = cases.shape_case(ref, "csg")
    g2, n2 = cases.sphere_small()
    prm = cases.params(20)
    a = n1.copy()
    relax_cl(g1, prm, a)
    b1, b2 = n1.copy(), n2.copy()
    relax_cl_batch([g1, g2], [prm, prm], [b1, b2])
    check_same(b1, a)
    c = n2.copy()
    relax_cl(g2, prm, c)
    check_same(b2, c)


def test_shape_handmade_program(ref, cuda_lib):
    """A program written by hand in the documented layout (a sphere and its
    complement) over the 48^3 sphere grid: nodes seeded as interior lattice
    points, so the interface forms by trapping."""
    from test_shapes_cpu import sphere_program
    g, nd = cases.sphere_small()
    c = (48 - 1) / 2.0
    g = type(g)(**{**g.__dict__, "gm": -1, "gTW": sphere_program((c, c, c), 17.6)})
    prm = cases.params(30)
    rd = nd.copy()
    rs = ref.relax_cpu(g, prm, rd)
    st = relax_cl(g, prm, nd)
    check_same(nd, rd)
    assert st.n_interface == rs.n_interface and st.n_interface > 0
