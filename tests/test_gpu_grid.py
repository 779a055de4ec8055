"""GPU: the grid build on the device (grid_cl, the C ABI's v2m_grid_build_cuda)
against the reference's own build_grid_cpu (oracle/_ref), bit for bit: brick
label counts and lists, slot starts, the smoothed-indicator fields phi, the
sizing field h, the size grades, hmin and hmax.

Inputs: a reference phantom, a 5-label argmax-of-noise volume (junctions and
corners), the small shells and TPM cases, a stack of thin layers with more
labels than a brick lists (overflow), anisotropic voxels, the reference's
default sizes, per-label sizes; then the benchmark's own label volumes at full
size (shells256, tpm182). Last, the whole chain on the device -- grid build,
seeding, relaxation -- equals build_grid_cpu -> seed_cpu -> relax_cpu.
"""
import numpy as np
import pytest

import cases
from cases import first_diff
from trussnet_b200 import GridParams, grid_cl, relax_cl, seed_cl, synth
from trussnet_b200.types import RelaxParams

pytestmark = pytest.mark.gpu


def thin_layers(dim=32, nlab=20):
    """Parallel one-voxel layers of nlab labels: a brick's box (8 + 2R + 1 = 21
    voxels wide) meets more labels than a brick lists (the overflow count)."""
    L = np.zeros((dim, dim, dim), np.uint16)
    x = np.arange(dim)
    lab = x % nlab + 1
    L[:, :, :] = lab[None, None, :].astype(np.uint16)
    L[:2] = 0
    return L


VOLUMES = {
    "phantom": lambda: (cases.phantom_labels(), (1.0, 1.0, 1.0), GridParams(hbase=2.5, hmin=1.5, hmax=3.0)),
    "noise": lambda: (cases.noise_labels(), (1.0, 1.0, 1.0), GridParams(hbase=2.0, hmin=1.2, hmax=3.0)),
    "noise_defaults": lambda: (cases.noise_labels(), (1.0, 1.0, 1.0), GridParams()),
    "shells_small": lambda: (cases.shells_small()[0].L, (1.0, 1.0, 1.0), GridParams(hbase=3.0, hmin=1.5, hmax=4.0)),
    "tpm_small": lambda: (cases.tpm_small()[0].L, (1.0, 1.0, 1.0), GridParams(hbase=2.0, hmin=1.3, hmax=3.0)),
    "overflow": lambda: (thin_layers(), (1.0, 1.0, 1.0), GridParams(hbase=2.0, hmin=1.0, hmax=3.0)),
    "anisotropic": lambda: (cases.phantom_labels(), (1.0, 1.25, 0.8), GridParams(hbase=2.5, hmin=1.5, hmax=3.0)),
}


def ref_grid(ref, L, vs, p: GridParams):
    return ref.build_grid_p(L, vs=vs, prm=p)


def assert_same_grid(gd, gr):
    assert (gd.hmin, gd.hmax) == (gr.hmin, gr.hmax)
    for a in ("bl_cnt", "bl_lab", "bl_slot", "phi", "h", "grade"):
        x, y = getattr(gd, a), getattr(gr, a)
        assert x.shape == y.shape, a
        d = first_diff(x, y)
        assert d is None, f"{a}: {d}"


@pytest.mark.parametrize("name", list(VOLUMES))
def test_grid_build_bit_exact(name, ref, cuda_lib):
    L, vs, p = VOLUMES[name]()
    gr = ref_grid(ref, L, vs, p)
    gd = grid_cl(L, vs, p)
    if name == "overflow":
        assert (gr.bl_cnt == 17).any()
    assert_same_grid(gd, gr)


@pytest.mark.parametrize("variant", ["hlab", "preserve", "thick", "no_thin_blend", "wide_sigma"])
def test_grid_build_options_bit_exact(variant, ref, cuda_lib):
    """The GridParams options the label path has: per-label sizes, the
    label-preserving margin, thin-layer sizing, the thin-layer blend off, a
    wider interface smoothing."""
    L = cases.phantom_labels()
    base = dict(hbase=2.5, hmin=1.5, hmax=3.0)
    p = {"hlab": GridParams(**base, hlab=(0.0, 0.0, 1.2, 2.0)),
         "preserve": GridParams(**base, preserve=0.1),
         "thick": GridParams(**base, thick=2.0),
         "no_thin_blend": GridParams(**base, sigma_thin=0.0),
         "wide_sigma": GridParams(**base, sigma=1.6)}[variant]
    gr = ref_grid(ref, L, (1.0, 1.0, 1.0), p)
    gd = grid_cl(L, (1.0, 1.0, 1.0), p)
    assert_same_grid(gd, gr)


@pytest.mark.parametrize("name", ["shells256", "tpm182"])
def test_grid_build_bit_exact_at_scale(name, ref, cuda_lib):
    g0, _ = synth.shells(seed=0) if name == "shells256" else synth.tpm(seed=0)
    L = g0.L
    p = GridParams(hbase=4.0, hmin=1.5, hmax=6.0)
    gr = ref_grid(ref, L, (1.0, 1.0, 1.0), p)
    gd = grid_cl(L, (1.0, 1.0, 1.0), p)
    assert_same_grid(gd, gr)


def test_device_chain_equals_reference_chain(ref, cuda_lib):
    """grid build -> seeding -> relaxation, each on the device, against
    build_grid_cpu -> seed_cpu -> relax_cpu."""
    L = cases.noise_labels()
    p = GridParams(hbase=2.0, hmin=1.2, hmax=3.0)
    prm = RelaxParams(max_iters=40)
    g_ref, nd_ref = ref.build_and_seed(L, sigma=p.sigma, hbase=p.hbase, hmin=p.hmin, hmax=p.hmax, prm=prm)
    g_dev = grid_cl(L, (1.0, 1.0, 1.0), p)
    nd_dev, part3 = seed_cl(g_dev, prm)
    assert nd_dev.size() == nd_ref.size()
    for f in ("P", "lab", "typ", "part"):
        assert first_diff(getattr(nd_dev, f), getattr(nd_ref, f)) is None, f
    st_ref = ref.relax_cpu(g_ref, prm, nd_ref)
    st_dev = relax_cl(g_dev, prm, nd_dev)
    assert (st_dev.iters, st_dev.rebuilds) == (st_ref.iters, st_ref.rebuilds)
    for f in ("P", "typ", "part"):
        assert first_diff(getattr(nd_dev, f), getattr(nd_ref, f)) is None, f


@pytest.mark.parametrize("name", ["phantom", "noise"])
def test_points_mode_on_device_equals_reference(name, ref, cuda_lib):
    """points_cl (v2m_points_cuda): one upload of the labels, grid build,
    seeding and relaxation from device arrays, one copy back -- equals the
    reference pipeline's points mode (build_grid_cpu -> seed_cpu -> relax_cpu)."""
    from trussnet_b200 import points_cl
    L, vs, p = VOLUMES[name]()
    prm = RelaxParams(max_iters=40)
    g_ref, nd_ref = ref.build_and_seed(L, sigma=p.sigma, hbase=p.hbase, hmin=p.hmin, hmax=p.hmax, prm=prm)
    part3_ref = nd_ref.part3.copy()
    st_ref = ref.relax_cpu(g_ref, prm, nd_ref)
    nd, part3, st = points_cl(L, vs, p, prm)
    assert nd.size() == nd_ref.size()
    for f in ("P", "lab", "typ", "part"):
        assert first_diff(getattr(nd, f), getattr(nd_ref, f)) is None, f
    assert np.array_equal(part3, part3_ref)
    assert (st.iters, st.rebuilds, st.fire_resets) == (st_ref.iters, st_ref.rebuilds, st_ref.fire_resets)


def test_pyv2mesh_points_call(cuda_lib):
    """trussnet_b200.pyv2mesh.points: v2mesh.points' call (vol[x, y, z], size
    and relaxation options, keys node / label / type / partner / info) on the
    device path; equals points_cl on the transposed volume."""
    from trussnet_b200 import points_cl, pyv2mesh
    L = cases.noise_labels()
    vol = L.transpose(2, 1, 0)   # vol[x, y, z]
    out = pyv2mesh.points(vol, size=2.0, hmin=1.2, hmax=3.0, iters=30)
    nd, part3, st = points_cl(L, (1.0, 1.0, 1.0), GridParams(hbase=2.0, hmin=1.2, hmax=3.0), RelaxParams(max_iters=30))
    assert np.array_equal(out["node"].astype(np.float32), nd.P)
    assert np.array_equal(out["type"], nd.typ.astype(np.int64)) and np.array_equal(out["label"], nd.lab)
    partner = out["partner"]
    assert partner.shape == (nd.size(), 3) and (partner[nd.typ == 0] == -1).all()
    assert out["info"]["iters"] == st.iters == 30
