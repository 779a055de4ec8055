"""CPU: the seeded synthetic inputs. The brick tables built by synth.build_grid
are the reference's (build_grid_cpu, src/v2m_grid.cpp:109-146 of
fangq/trussnet): same per-brick label lists, counts and slot numbering; the
smoothed fields agree with the reference's sigma = 1 smoothing where the
reference applies no thin-layer blending."""
import numpy as np
import pytest

import cases
from trussnet_b200 import synth
from trussnet_b200.types import V2M_BL, V2M_NOLAB


def test_bricks_match_reference(ref):
    g, _ = cases.sphere_small()
    gr = ref.build_grid(g.L, hbase=2.0, hmin=2.0, hmax=2.0)
    assert np.array_equal(gr.bl_cnt, g.bl_cnt)
    assert np.array_equal(gr.bl_lab, g.bl_lab)
    assert np.array_equal(gr.bl_slot, g.bl_slot)
    assert gr.phi.size == g.phi.size
    assert np.abs(gr.phi - g.phi).max() < 1e-5


def test_multilabel_bricks_match_reference(ref):
    g, _ = cases.tpm_small()
    gr = ref.build_grid(g.L, hbase=1.6, hmin=1.6, hmax=1.6)
    assert np.array_equal(gr.bl_cnt, g.bl_cnt)
    assert np.array_equal(gr.bl_lab, g.bl_lab)
    assert np.array_equal(gr.bl_slot, g.bl_slot)


def test_brick_table_invariants():
    g, nd = cases.shells_small()
    nb = g.nbx * g.nby * g.nbz
    lab = g.bl_lab.reshape(nb, V2M_BL)
    for b in range(nb):
        c = min(int(g.bl_cnt[b]), V2M_BL)
        assert c >= 1
        row = lab[b]
        assert np.all(np.diff(row[:c].astype(int)) > 0)           # ascending, unique
        assert np.all(row[c:] == V2M_NOLAB)
        assert (g.bl_slot[b] >= 0) == (c >= 2)
    assert g.phi.size // 512 == int(np.sum(np.where(g.bl_slot >= 0, np.minimum(g.bl_cnt, V2M_BL), 0)))
    assert nd.size() > 1000
    assert np.all(nd.lab != 0) and np.all(nd.typ == 0)
    # seeds lie in non-zero voxels of their own label
    ijk = np.floor(nd.P + 0.5).astype(int)
    assert np.all(g.L[ijk[:, 2], ijk[:, 1], ijk[:, 0]] == nd.lab)


def test_seeds_deterministic():
    a = synth.sphere(dim=32, radius=10.0, seed=4)[1]
    b = synth.sphere(dim=32, radius=10.0, seed=4)[1]
    c = synth.sphere(dim=32, radius=10.0, seed=5)[1]
    assert np.array_equal(a.P, b.P)
    assert not np.array_equal(a.P, c.P) or a.P.shape != c.P.shape


@pytest.mark.slow
def test_shells256_size():
    g, nd = synth.shells()
    assert 0.9e6 < nd.size() < 1.1e6
    assert np.unique(g.L).size == 7
    assert g.hmin == 1.5 and g.hmax == 6.0
