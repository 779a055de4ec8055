"""CPU: the C ABI library loads, exports every function include/v2m_cuda.h
declares, validates its arguments before touching a device, and fails loudly
(V2M_ERR_CUDA, a raised V2mError) where no CUDA device exists -- no silent CPU
fallback. No compute call runs here."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import cases
from trussnet_b200 import V2mError, _lib, relax_cl
from trussnet_b200.types import NodesView, RelaxParams, RelaxParamsC

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    text = open(os.path.join(ROOT, "include", "v2m_cuda.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(v2m_[a-z0-9_]+)\s*\(", text)))


def test_every_declared_symbol_is_exported():
    L = _lib.load()
    names = header_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert sorted(_lib.EXPORTS) == names


def test_params_default_matches_reference():
    L = _lib.load()
    p = RelaxParamsC()
    L.v2m_relax_params_default(C.byref(p))
    ref = RelaxParams()
    for f in ("nseed", "t", "skin", "fscale", "fsurf", "dt", "maxstep", "snap", "max_iters", "dptol", "jseed",
              "thin", "fire_dtmax"):
        assert getattr(p, f) == pytest.approx(getattr(ref, f), rel=1e-7), f
    assert p.fire == 1 and p.voxel_trap == 0 and p.corners == 1


def test_argument_errors_before_any_device():
    g, nd = cases.sphere_small()
    bad = nd.copy()
    bad.typ[3] = 7
    with pytest.raises(V2mError) as e:
        relax_cl(g, RelaxParams(max_iters=1), bad)
    assert e.value.code == _lib.V2M_ERR_ARG and "type" in str(e.value)
    g2 = cases.sphere_small()[0]
    g2 = type(g2)(**{**g2.__dict__, "hmin": 0.0})
    with pytest.raises(V2mError) as e:
        relax_cl(g2, RelaxParams(max_iters=1), nd.copy())
    assert e.value.code == _lib.V2M_ERR_ARG
    with pytest.raises(V2mError) as e:
        relax_cl(g, RelaxParams(max_iters=-1), nd.copy())
    assert e.value.code == _lib.V2M_ERR_ARG
    g3 = cases.sphere_small()[0]
    g3 = type(g3)(**{**g3.__dict__, "gm": -1})
    with pytest.raises(V2mError) as e:
        relax_cl(g3, RelaxParams(max_iters=1), nd.copy())
    assert "analytic" in str(e.value)
    g4 = cases.sphere_small()[0]
    slot = g4.bl_slot.copy()
    slot[np.argmax(slot)] = g4.phi.size // 512
    g4 = type(g4)(**{**g4.__dict__, "bl_slot": slot})
    with pytest.raises(V2mError) as e:
        relax_cl(g4, RelaxParams(max_iters=1), nd.copy())
    assert "slot" in str(e.value)


@pytest.mark.skipif(_lib.load().v2m_cuda_device_count() > 0, reason="a CUDA device is present")
def test_no_device_fails_loudly():
    g, nd = cases.sphere_small()
    before = nd.P.copy()
    with pytest.raises(V2mError) as e:
        relax_cl(g, RelaxParams(max_iters=3), nd)
    assert e.value.code == _lib.V2M_ERR_CUDA
    assert np.array_equal(nd.P, before)      # nothing written back


def test_null_views_rejected():
    L = _lib.load()
    rc = L.v2m_relax_cuda(None, None, None, None, 0)
    assert rc == _lib.V2M_ERR_ARG
    assert L.v2m_cuda_last_error()


def test_session_create_rejects_bad_volume_count():
    L = _lib.load()
    h = C.c_void_p()
    assert L.v2m_session_create(0, None, None, None, 0, C.byref(h)) == _lib.V2M_ERR_ARG
    nv = NodesView()
    assert isinstance(nv, C.Structure)


def test_python_views_match_the_c_header(tmp_path):
    """The ctypes mirrors of the C ABI's structs have the header's size and
    field offsets (compiled with the system C compiler)."""
    import shutil
    import subprocess
    from trussnet_b200.types import GridView, NodesView, RelaxParamsC, RelaxStatsC
    cc = shutil.which("gcc") or shutil.which("cc")
    if not cc:
        pytest.skip("no C compiler")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    structs = {"v2m_grid_view": GridView, "v2m_nodes_view": NodesView, "v2m_relax_params": RelaxParamsC,
               "v2m_relax_stats": RelaxStatsC}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "v2m_cuda.h"', "int main(void) {"]
    for cname, py in structs.items():
        lines.append(f'    printf("{cname} size %zu\\n", sizeof({cname}));')
        for f in py._fields_:
            lines.append(f'    printf("{cname} {f[0]} %zu\\n", offsetof({cname}, {f[0]}));')
    lines += ["    return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run([cc, "-std=c11", "-I", os.path.join(root, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    got = {tuple(l.split()[:2]): int(l.split()[2]) for l in out if l.strip()}
    for cname, py in structs.items():
        assert got[(cname, "size")] == C.sizeof(py), cname
        for f in py._fields_:
            assert got[(cname, f[0])] == getattr(py, f[0]).offset, (cname, f[0])
