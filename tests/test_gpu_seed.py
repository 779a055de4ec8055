"""GPU parity of seeding: seed_cl (the CUDA seeding, through the C ABI) against
the reference's own seed_cpu (oracle/_ref) on reference-built grids -- label
volumes and shape input -- with junction-line seeds and corners on and off and
in voxel-trap mode. The bar is bit-exact: the node count and order, positions,
labels, types and the three partner labels."""
import numpy as np
import pytest

import cases
from cases import first_diff
from trussnet_b200 import seed_cl
from trussnet_b200.types import V2M_CORNER, V2M_JUNCTION, RelaxParams

pytestmark = pytest.mark.gpu


def check_seeds(ref_nd, nd, part3):
    assert nd.size() == ref_nd.size()
    for a in ("P", "lab", "typ", "part"):
        d = first_diff(getattr(nd, a), getattr(ref_nd, a))
        assert d is None, f"{a}: {d}"
    d = first_diff(part3, ref_nd.part3)
    assert d is None, f"part3: {d}"


@pytest.mark.parametrize("name", ["phantom", "noise", "mcx", "csg"])
def test_seed_bit_exact(name, ref, cuda_lib):
    prm = RelaxParams()
    g, rnd = cases.seed_case(ref, name, prm)
    nd, part3 = seed_cl(g, prm)
    check_seeds(rnd, nd, part3)
    assert (nd.typ == V2M_JUNCTION).any()


@pytest.mark.parametrize("variant", ["no_junction_seeds", "no_corners", "voxel_trap", "one_level"])
def test_seed_variants_bit_exact(variant, ref, cuda_lib):
    prm = {"no_junction_seeds": RelaxParams(jseed=0.0), "no_corners": RelaxParams(corners=False),
           "voxel_trap": RelaxParams(voxel_trap=True, fire=False), "one_level": RelaxParams(nseed=1)}[variant]
    g, rnd = cases.seed_case(ref, "noise", prm)
    nd, part3 = seed_cl(g, prm)
    check_seeds(rnd, nd, part3)
    if variant == "no_corners":
        assert not (nd.typ == V2M_CORNER).any()


def test_seeded_relax_matches_reference(ref, cuda_lib):
    """Seeds made on the device, then relaxed on the device: the reference's
    seed_cpu + relax_cpu result."""
    from trussnet_b200 import relax_cl
    prm = RelaxParams(max_iters=20)
    g, rnd = cases.seed_case(ref, "phantom", prm)
    nd, _ = seed_cl(g, prm)
    ref.relax_cpu(g, prm, rnd)
    relax_cl(g, prm, nd)
    for a in ("P", "typ", "part"):
        d = first_diff(getattr(nd, a), getattr(rnd, a))
        assert d is None, f"{a}: {d}"


@pytest.mark.parametrize("name", ["mcx", "csg", "jmesh", "split"])
def test_seed_shape_features_bit_exact(name, ref, cuda_lib):
    """Shape input with its sharp features handed to the grid (as the shape
    front end does): seed_cpu's feature pass -- CORNER nodes pinned on the
    primitives' corners, edges and rims, the seeds near them dropped -- against
    the device's."""
    scene, kw = cases.SHAPE_SCENES[name]
    prm = RelaxParams()
    g, rnd = ref.shape_and_seed(scene, voxel=1.0, hbase=2.5, hmin=1.5, hmax=3.5, prm=prm, feat=True, **kw)
    assert g.feat is not None and g.feat.size > 0
    nd, part3 = seed_cl(g, prm)
    check_seeds(rnd, nd, part3)
    assert (nd.typ == V2M_CORNER).sum() > 0


def test_shape_features_seeded_relax_matches_reference(ref, cuda_lib):
    """Feature-pinned seeds made on the device, relaxed on the device: the
    reference's seed_cpu + relax_cpu result (the CORNER nodes stay put)."""
    from trussnet_b200 import relax_cl
    scene, kw = cases.SHAPE_SCENES["csg"]
    prm = RelaxParams(max_iters=15)
    g, rnd = ref.shape_and_seed(scene, voxel=1.0, hbase=2.5, hmin=1.5, hmax=3.5, prm=prm, feat=True, **kw)
    nd, _ = seed_cl(g, prm)
    corner = nd.typ == V2M_CORNER
    P0 = nd.P.copy()
    ref.relax_cpu(g, prm, rnd)
    relax_cl(g, prm, nd)
    for a in ("P", "typ", "part"):
        d = first_diff(getattr(nd, a), getattr(rnd, a))
        assert d is None, f"{a}: {d}"
    assert np.array_equal(nd.P[corner], P0[corner])
