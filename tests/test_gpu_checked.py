"""The bounds-checked build (libv2m_cuda_check.so, V2M_CHECK): the same
relaxations, shape-field relaxation and seeding as the normal build, run in a
child process that loads the checked library, end without a failed check and
with the normal build's results bit for bit."""
import hashlib
import json
import os
import subprocess
import sys

import numpy as np
import pytest

import cases
from trussnet_b200 import build as b
from trussnet_b200.types import RelaxParams

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import hashlib, json, sys
sys.path.insert(0, {root!r}); sys.path.insert(0, {tests!r})
import cases
from oracle.ref import RefLib
from trussnet_b200 import relax_cl, seed_cl, _lib
from trussnet_b200.types import RelaxParams
assert _lib.load()._name.endswith("libv2m_cuda_check.so")
out = {{}}
def h(nd):
    return hashlib.md5(nd.P.tobytes() + nd.typ.tobytes() + nd.part.tobytes()).hexdigest()
for name in ("shells_small", "tpm_small"):
    g, nd = getattr(cases, name)()
    x = nd.copy()
    relax_cl(g, RelaxParams(max_iters=30), x)
    out[name] = h(x)
ref = RefLib()
g, nd = cases.shape_case(ref, "csg")
x = nd.copy()
relax_cl(g, RelaxParams(max_iters=20), x)
out["csg"] = h(x)
g, _ = cases.seed_case(ref, "phantom", RelaxParams())
s, p3 = seed_cl(g, RelaxParams())
out["seed"] = hashlib.md5(s.P.tobytes() + s.lab.tobytes() + s.typ.tobytes() + s.part.tobytes() + p3.tobytes()).hexdigest()
print(json.dumps(out))
"""


def _h(nd):
    return hashlib.md5(nd.P.tobytes() + nd.typ.tobytes() + nd.part.tobytes()).hexdigest()


def test_checked_build_runs_clean_and_equal(ref, cuda_lib):
    from trussnet_b200 import relax_cl, seed_cl
    if not os.path.exists(b.LIB_CHECK):
        pytest.fail(f"{b.LIB_CHECK} is not built (trussnet_b200.build.build_cuda(check=True))")
    want = {}
    for name in ("shells_small", "tpm_small"):
        g, nd = getattr(cases, name)()
        x = nd.copy()
        relax_cl(g, RelaxParams(max_iters=30), x)
        want[name] = _h(x)
    g, nd = cases.shape_case(ref, "csg")
    x = nd.copy()
    relax_cl(g, RelaxParams(max_iters=20), x)
    want["csg"] = _h(x)
    g, _ = cases.seed_case(ref, "phantom", RelaxParams())
    s, p3 = seed_cl(g, RelaxParams())
    want["seed"] = hashlib.md5(s.P.tobytes() + s.lab.tobytes() + s.typ.tobytes() + s.part.tobytes()
                               + p3.tobytes()).hexdigest()
    env = dict(os.environ, V2M_CUDA_LIBRARY=b.LIB_CHECK)
    code = CHILD.format(root=ROOT, tests=os.path.join(ROOT, "tests"))
    r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    got = json.loads(r.stdout.strip().splitlines()[-1])
    assert got == want
