"""Shape input (analytic fields, gm < 0) without a GPU: the test scenes reach
the whole program language of src/opencl/v2m_sdf_body.cl, and the C ABI checks
a shape program before any device work."""
import numpy as np
import pytest

import cases
from trussnet_b200 import V2mError, _lib, relax_cl
from trussnet_b200.types import RelaxParams


def sphere_program(c, r, w=1.5):
    """A two-label program in the documented layout (src/opencl/v2m_sdf_body.cl:9-21):
    label 1 inside the sphere, label 0 (its complement) outside; no brick table."""
    N = 2
    head = [N, w, 0.0, 0.0, 0.0, 0, 0, 0.0, 0.0, 3.0, 0.0]
    code1 = [1, 1, c[0], c[1], c[2], r, 0]            # PRIM SPHERE c r, END
    code0 = [1, 1, c[0], c[1], c[2], r, 4, 0]         # PRIM SPHERE c r, NEG, END
    head[5] = len(head)
    head[6] = len(head) + len(code0)
    return np.array(head + code0 + code1, np.float32)


def test_shape_scenes_cover_the_program_language(ref):
    prims, ops = set(), set()
    for name in cases.SHAPE_SCENES:
        g, nd = cases.shape_case(ref, name)
        assert g.gm == -1 and nd.size() > 500
        assert set(np.unique(nd.lab)) <= set(range(int(g.gTW[0])))
        p, o = cases.shape_opcodes(g.gTW)
        prims |= p
        ops |= o
    assert prims == set(range(1, 10)), prims      # every primitive type
    assert ops == set(range(0, 12)), ops          # every opcode


def test_shape_relax_reference_runs(ref):
    g, nd = cases.shape_case(ref, "split")
    st = ref.relax_cpu(g, cases.params(5), nd)
    assert st.iters == 5


def shape_grid(prog):
    g, nd = cases.sphere_small()
    return type(g)(**{**g.__dict__, "gm": -1, "gTW": prog}), nd


def test_shape_program_checked_before_any_device():
    c = (16.0, 16.0, 16.0)
    good = sphere_program(c, 10.0)
    bad = {
        "label count": good.copy(),
        "width": good.copy(),
        "code offset": good.copy(),
        "brick table": good.copy(),
        "header": good[:8].copy(),
    }
    bad["label count"][0] = 0.0
    bad["width"][1] = 0.0
    bad["code offset"][5] = float(good.size)
    bad["brick table"][10] = float(good.size)
    for what, prog in bad.items():
        g, nd = shape_grid(prog)
        with pytest.raises(V2mError) as e:
            relax_cl(g, RelaxParams(max_iters=1), nd)
        assert e.value.code == _lib.V2M_ERR_ARG, what
        assert "shape" in str(e.value) or "analytic" in str(e.value), (what, str(e.value))


@pytest.mark.parametrize("name", list(cases.SHAPE_SCENES))
def test_oracle_restatement_equals_reference_on_shapes(name, ref):
    """The plain-C restatement's analytic fields (FP32) against the compiled
    reference: 15 relaxation iterations, bit for bit."""
    from oracle.oracle import Oracle
    g, nd = cases.shape_case(ref, name)
    prm = cases.params(15)
    a, b = nd.copy(), nd.copy()
    ra = ref.relax_cpu(g, prm, a)
    rb = Oracle("f32").relax(g, prm, b)
    for f in ("P", "typ", "part"):
        d = cases.first_diff(getattr(b, f), getattr(a, f))
        assert d is None, f"{f}: {d}"
    assert (rb.iters, rb.rebuilds) == (ra.iters, ra.rebuilds)


def test_oracle_restatement_handmade_program(ref):
    from oracle.oracle import Oracle
    g, nd = shape_grid(sphere_program((23.5, 23.5, 23.5), 17.6))
    prm = cases.params(15)
    a, b = nd.copy(), nd.copy()
    ref.relax_cpu(g, prm, a)
    Oracle("f32").relax(g, prm, b)
    assert cases.first_diff(b.P, a.P) is None and cases.first_diff(b.typ, a.typ) is None


def test_seed_checked_before_any_device():
    from trussnet_b200 import seed_cl
    g, _ = cases.sphere_small()            # (synthetic grids carry no size grades)
    assert g.grade is None
    with pytest.raises(V2mError) as e:
        seed_cl(g, RelaxParams())
    assert e.value.code == _lib.V2M_ERR_ARG and "grade" in str(e.value)
    g2 = type(g)(**{**g.__dict__, "grade": np.zeros((g.nz, g.ny, g.nx), np.uint8)})
    with pytest.raises(V2mError) as e:
        seed_cl(g2, RelaxParams(nseed=0))
    assert e.value.code == _lib.V2M_ERR_ARG and "nseed" in str(e.value)
    g3 = type(g2)(**{**g2.__dict__, "hmin": 0.01})   # more lattice points than int32 counts hold
    with pytest.raises(V2mError) as e:
        seed_cl(g3, RelaxParams())
    assert e.value.code == _lib.V2M_ERR_ARG and "int32" in str(e.value)


def test_seed_cases_build(ref):
    """The seeding cases' reference seeds: every node type present."""
    for name, types in (("phantom", {0, 1, 2}), ("noise", {0, 1, 2, 3})):
        g, nd = cases.seed_case(ref, name, RelaxParams())
        assert g.grade is not None and g.grade.shape == (g.nz, g.ny, g.nx)
        assert set(np.unique(nd.typ)) == types, name
        assert nd.part3.shape == (nd.size(),)


@pytest.mark.parametrize("name", ["phantom", "noise", "mcx", "csg"])
def test_oracle_seeding_equals_reference(name, ref):
    """The plain-C restatement of seed_cpu against the compiled reference."""
    from oracle.oracle import Oracle
    prm = RelaxParams()
    g, rnd = cases.seed_case(ref, name, prm)
    nd = Oracle("f32").seed(g, prm)
    assert nd.size() == rnd.size()
    for f in ("P", "lab", "typ", "part", "part3"):
        d = cases.first_diff(getattr(nd, f), getattr(rnd, f))
        assert d is None, f"{f}: {d}"


@pytest.mark.parametrize("prm", [RelaxParams(jseed=0.0), RelaxParams(corners=False),
                                 RelaxParams(voxel_trap=True, fire=False), RelaxParams(nseed=1)],
                         ids=["no_junction_seeds", "no_corners", "voxel_trap", "one_level"])
def test_oracle_seeding_variants(prm, ref):
    from oracle.oracle import Oracle
    g, rnd = cases.seed_case(ref, "noise", prm)
    nd = Oracle("f32").seed(g, prm)
    assert nd.size() == rnd.size()
    for f in ("P", "lab", "typ", "part", "part3"):
        assert cases.first_diff(getattr(nd, f), getattr(rnd, f)) is None, f


@pytest.mark.skipif(_lib.load().v2m_cuda_device_count() > 0, reason="a CUDA device is present")
def test_seed_without_device_fails_loudly():
    """No CPU fallback inside the library: seeding without a device is a CUDA error."""
    from trussnet_b200 import seed_cl
    g, _ = cases.sphere_small()
    g = type(g)(**{**g.__dict__, "grade": np.zeros((g.nz, g.ny, g.nx), np.uint8)})
    with pytest.raises(V2mError) as e:
        seed_cl(g, RelaxParams())
    assert e.value.code == _lib.V2M_ERR_CUDA
