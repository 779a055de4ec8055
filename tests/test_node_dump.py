"""The node dump (v2mesh's --dump-nodes format, src/v2m_pipeline.cpp:58-73):
dump_nodes writes the reference's layout byte for byte -- one compact JSON
header line with sorted keys, then P, Label, Type, Partner raw -- and
load_nodes reads it back."""
import numpy as np

import cases
from trussnet_b200.pyv2mesh import dump_nodes, load_nodes
from trussnet_b200.types import Nodes


def _nodes(n, seed=0):
    rng = np.random.default_rng(seed)
    return Nodes(P=rng.normal(size=(n, 3)).astype(np.float32) * 40, lab=rng.integers(0, 7, n).astype(np.uint16),
                 typ=rng.integers(0, 4, n).astype(np.uint8), part=rng.integers(0, 0xFFFF, (n, 2)).astype(np.uint16))


def test_layout_is_the_references(tmp_path):
    nd = _nodes(5)
    p = tmp_path / "n.bjd"
    dump_nodes(p, nd)
    raw = p.read_bytes()
    head, body = raw.split(b"\n", 1)
    # nlohmann::json's dump of the reference's header object: sorted keys, no spaces
    assert head == (b'{"Label":["uint16",[5],60],"P":["float32",[5,3],0],"Partner":["uint16",[5,2],75],'
                    b'"Type":["uint8",[5],70]}')
    assert body == nd.P.tobytes() + nd.lab.tobytes() + nd.typ.tobytes() + nd.part.tobytes()


def test_round_trip(tmp_path):
    g, nd = cases.sphere_small()
    p = tmp_path / "n.bjd"
    dump_nodes(p, nd)
    back = load_nodes(p)
    for a in ("P", "lab", "typ", "part"):
        assert np.array_equal(getattr(back, a), getattr(nd, a)), a
    assert back.P.dtype == np.float32 and back.part.shape == (nd.size(), 2)


def test_empty(tmp_path):
    nd = _nodes(0)
    p = tmp_path / "e.bjd"
    dump_nodes(p, nd)
    assert p.read_bytes() == (b'{"Label":["uint16",[0],0],"P":["float32",[0,3],0],"Partner":["uint16",[0,2],0],'
                              b'"Type":["uint8",[0],0]}\n')
    assert load_nodes(p).size() == 0
