"""GPU parity: the CUDA relaxation (through the C ABI) against the reference's
own CPU path (oracle/_ref, relax_cpu and its stages) on identical inputs.

The bar is bit-exact: bin keys, sorted order, bin starts, truss lists, forces,
positions, types and partner labels. Kernels compute in FP32 without FMA
contraction and with IEEE division and square root, in the reference's
operation order, so there is no tolerance to state for these stages.
"""
import numpy as np
import pytest

import cases
from cases import first_diff, same_bits
from trussnet_b200 import Session, relax_cl, relax_cl_batch
from trussnet_b200.types import V2M_CORNER, V2M_K, RelaxParams

pytestmark = pytest.mark.gpu

CASES = ["sphere_small", "shells_small", "tpm_small", "ref_phantom", "gray_small"]


def load_case(name, ref):
    if name == "ref_phantom":
        return cases.ref_phantom(ref)
    return getattr(cases, name)()


def rowmajor_lists(nbr, nnb, n):
    """Truss lists with unused slots zeroed (both sides compared this way)."""
    nbr = nbr.reshape(n, V2M_K).copy()
    k = np.arange(V2M_K)[None, :]
    nbr[k >= nnb[:, None]] = 0
    return nbr


@pytest.mark.parametrize("name", CASES)
def test_rebuild_bit_exact(name, ref, cuda_lib):
    g, nd = load_case(name, ref)
    prm = cases.params(10)
    rs = ref.state(g, prm, nd.copy())
    rs.rebuild()
    with Session(g, prm, nd.copy()) as s:
        s.rebuild()
        assert s.nkeys[0] == rs.nkeys
        for a in ("key", "sorted", "cstart", "nnb"):
            d = first_diff(s.read(a), rs.read(a))
            assert d is None, f"{a}: {d}"
        ps_ref = rs.read("Ps").reshape(-1, 4)
        assert same_bits(s.read("Ps").reshape(-1, 4), ps_ref)
        n = nd.size()
        nnb = rs.read("nnb")
        d = first_diff(rowmajor_lists(s.read("nbr"), nnb, n), rowmajor_lists(rs.read("nbr"), nnb, n))
        assert d is None, f"nbr: {d}"
        assert same_bits(s.read("P0"), rs.read("P0"))


@pytest.mark.parametrize("name", CASES)
def test_force_bit_exact(name, ref, cuda_lib):
    g, nd = load_case(name, ref)
    prm = cases.params(10)
    rs = ref.state(g, prm, nd.copy())
    rs.rebuild()
    rs.force()
    with Session(g, prm, nd.copy()) as s:
        s.rebuild()
        s.force()
        d = first_diff(s.read("F"), rs.read("F"))
        assert d is None, f"F: {d}"


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("fire", [True, False])
def test_one_iteration_bit_exact(name, fire, ref, cuda_lib):
    g, nd = load_case(name, ref)
    prm = cases.params(10, fire=fire)
    rs = ref.state(g, prm, nd.copy())
    rs.rebuild()
    with Session(g, prm, nd.copy()) as s:
        s.rebuild()
        for it in range(3):
            rs.force()
            rs.tail()
            s.force()
            s.step_tail()
            for a in ("P", "typ", "part", "mv", "hn"):
                d = first_diff(s.read(a), rs.read(a))
                assert d is None, f"iteration {it}, {a}: {d}"
            if fire:
                for a in ("V", "pw"):
                    d = first_diff(s.read(a), rs.read(a))
                    assert d is None, f"iteration {it}, {a}: {d}"
            st = s.stats()
            c = rs.counts()
            assert st.rebuilds == c["rebuilds"], it
            assert st.last_move == c["mmax"]
            assert st.last_p99 == c["p99"]
            assert st.fire_resets == c["fire_resets"]


@pytest.mark.parametrize("name", CASES)
def test_full_relax_bit_exact(name, ref, cuda_lib):
    """Whole loop in the production mode (the FIRE power's sign from the block
    tree when it is clear of rounding, else from the serial order): identical to
    relax_cpu."""
    g, nd = load_case(name, ref)
    prm = cases.params(60)
    a = nd.copy()
    st_ref = ref.relax_cpu(g, prm, a)
    b = nd.copy()
    st = relax_cl(g, prm, b)
    assert st.iters == st_ref.iters and st.rebuilds == st_ref.rebuilds
    for f in ("P", "typ", "part"):
        d = first_diff(getattr(b, f), getattr(a, f))
        assert d is None, f"{f}: {d}"
    assert st.fire_resets == st_ref.fire_resets and st.fire_dt == st_ref.fire_dt
    assert (st.n_interior, st.n_interface, st.n_junction, st.n_corner) == \
        (st_ref.n_interior, st_ref.n_interface, st_ref.n_junction, st_ref.n_corner)


@pytest.mark.parametrize("name", ["sphere64", "shells_small", "ref_phantom"])
def test_full_relax_graph_and_plain(name, ref, cuda_lib):
    """Longer runs: the graph and the plain launches agree bit for bit, and both
    equal relax_cpu."""
    g, nd = load_case(name, ref)
    prm = RelaxParams(max_iters=200, dt=0.2, dptol=0.0) if name == "sphere64" else cases.params(80)
    a = nd.copy()
    st_ref = ref.relax_cpu(g, prm, a)
    with Session(g, prm, nd.copy()) as s:
        s.run(graph=True)
        b = s.read_nodes(nd.copy())
        st = s.stats()
        s.reset()
        s.run(graph=False)
        c = s.read_nodes(nd.copy())
    for f in ("P", "typ", "part"):
        assert same_bits(getattr(b, f), getattr(c, f)), f"graph vs plain launches differ in {f}"
    assert st.iters == st_ref.iters and st.fire_resets == st_ref.fire_resets
    for f in ("P", "typ", "part"):
        d = first_diff(getattr(b, f), getattr(a, f))
        assert d is None, f"{f} vs relax_cpu: {d}"


def two_pairs():
    """Four interior nodes in a uniform label-1 volume (h = 1.25): two pairs of
    nodes one voxel apart along x, each pair's bar compressed, the pairs out of
    each other's reach. Equal and opposite forces +-f."""
    from trussnet_b200 import synth
    from trussnet_b200.types import Nodes
    L = np.ones((32, 32, 32), np.uint16)
    g = synth.build_grid(L, np.full(L.shape, 1.25, np.float32), 1.25, 1.25)
    P = np.array([[15, 16, 16], [16, 16, 16], [15, 16, 24], [16, 16, 24]], np.float32)
    nd = Nodes(P=P, lab=np.ones(4, np.uint16), typ=np.zeros(4, np.uint8), part=np.full((4, 2), 0xFFFF, np.uint16))
    return g, nd


def test_fire_power_within_rounding_of_zero(ref, cuda_lib):
    """Velocities planted so that the powers are f 2^61, -f 2^61, -2f, 0: the
    serial double sum is -2f (uphill: FIRE resets), while a pairwise tree
    rounds f 2^61 - 2f to f 2^61 and gives 0 (downhill). The sum is within the
    rounding bound of zero, so the kernel takes the serial order: the same reset
    as relax_cpu, and the fallback is counted."""
    g, nd = two_pairs()
    prm = cases.params(5, dptol=0.0)
    V = np.array([[-2.0 ** 61, 0, 0], [-2.0 ** 61, 0, 0], [2, 0, 0], [0, 0, 0]], np.float32)
    rs = ref.state(g, prm, nd.copy())
    rs.rebuild()
    rs.write("V", V.reshape(-1))
    rs.force()
    with Session(g, prm, nd.copy()) as s:
        s.rebuild()
        s.write("V", V.reshape(-1))
        s.force()
        F = s.read("F").reshape(-1, 4)
        assert F[0, 0] == -F[1, 0] and F[2, 0] == -F[3, 0] and F[0, 0] < 0
        rs.tail()
        s.step_tail()
        pw = s.read("pw").astype(np.float64)
        assert pw[0] == -pw[1] and pw[2] < 0 and pw[3] == 0
        assert sum(pw.tolist()) < 0 and (pw[0] + pw[2]) + (pw[1] + pw[3]) == 0.0
        assert s.read("serial_sums")[0] == 1
        assert s.stats().fire_resets == rs.counts()["fire_resets"] == 1
        for a in ("P", "typ", "V", "pw"):
            d = first_diff(s.read(a), rs.read(a))
            assert d is None, f"{a}: {d}"


def test_relax_cl_deterministic(cuda_lib):
    g, nd = cases.shells_small()
    prm = cases.params(50)
    a, b = nd.copy(), nd.copy()
    relax_cl(g, prm, a)
    relax_cl(g, prm, b)
    assert same_bits(a.P, b.P) and same_bits(a.typ, b.typ) and same_bits(a.part, b.part)


def test_voxel_trap_mode(ref, cuda_lib):
    g, nd = cases.shells_small()
    prm = cases.params(20, voxel_trap=True)
    a = nd.copy()
    ref.relax_cpu(g, prm, a)
    b = nd.copy()
    relax_cl(g, prm, b)
    for f in ("P", "typ", "part"):
        d = first_diff(getattr(b, f), getattr(a, f))
        assert d is None, f"{f}: {d}"


def test_corners_stay(ref, cuda_lib):
    g, nd = cases.tpm_small()
    nd = nd.copy()
    rng = np.random.default_rng(5)
    idx = rng.choice(nd.size(), 50, replace=False)
    nd.typ[idx] = V2M_CORNER
    prm = cases.params(20)
    a = nd.copy()
    ref.relax_cpu(g, prm, a)
    b = nd.copy()
    relax_cl(g, prm, b)
    assert same_bits(b.P[idx], nd.P[idx])
    assert same_bits(b.P, a.P) and same_bits(b.typ, a.typ)


def test_batch_equals_single(cuda_lib):
    vols = [cases.sphere_small(), cases.shells_small(), cases.tpm_small()]
    prms = [cases.params(40), cases.params(25), cases.params(30)]
    singles = []
    for (g, nd), p in zip(vols, prms):
        x = nd.copy()
        relax_cl(g, p, x)
        singles.append(x)
    outs = [nd.copy() for _, nd in vols]
    relax_cl_batch([g for g, _ in vols], prms, outs)
    for x, y in zip(singles, outs):
        assert same_bits(x.P, y.P) and same_bits(x.typ, y.typ) and same_bits(x.part, y.part)


def test_edge_cases(ref, cuda_lib):
    g, nd = cases.sphere_small()
    prm = cases.params(5)
    # no nodes
    empty = nd.copy()
    empty.P = empty.P[:0].copy()
    empty.lab = empty.lab[:0].copy()
    empty.typ = empty.typ[:0].copy()
    empty.part = empty.part[:0].copy()
    st = relax_cl(g, prm, empty)
    st_ref = ref.relax_cpu(g, prm, empty.copy())
    assert st.iters == st_ref.iters
    # one node
    one = nd.copy()
    one.P, one.lab, one.typ, one.part = one.P[:1].copy(), one.lab[:1].copy(), one.typ[:1].copy(), one.part[:1].copy()
    a = one.copy()
    ref.relax_cpu(g, prm, a)
    relax_cl(g, prm, one)
    assert same_bits(one.P, a.P)
    # zero iterations: nothing moves
    z = nd.copy()
    relax_cl(g, cases.params(0), z)
    assert same_bits(z.P, nd.P)


def test_trilinear_h_matches_oracle(cuda_lib):
    """Extension: h sampled trilinearly (h_mode 1) -- no reference counterpart;
    bit-exact with the FP32 restatement in the same mode."""
    from oracle.oracle import Oracle
    g, nd = cases.shells_small()
    prm = cases.params(30, h_mode=1)
    a = nd.copy()
    Oracle("f32").relax(g, prm, a)
    b = nd.copy()
    relax_cl(g, prm, b)
    for f in ("P", "typ", "part"):
        d = first_diff(getattr(b, f), getattr(a, f))
        assert d is None, f"{f}: {d}"


@pytest.mark.parametrize("name", ["sphere_small", "shells_small", "tpm_small"])
def test_step_within_tolerance_of_fp64(name, cuda_lib, record_property):
    """One step from identical positions and lists: CUDA forces within 1e-6 of the
    FP64 restatement (per-bar scale h_i * active bars), free-step positions within
    1e-6 of |P|; trapped positions within the projection tolerance (1e-2 h)."""
    from oracle.oracle import Oracle
    g, nd = getattr(cases, name)()
    prm = cases.params(1)
    o64 = Oracle("f64").state(g, prm, nd.copy())
    with Session(g, prm, nd.copy()) as s:
        s.rebuild()
        n = nd.size()
        nbr, nnb = s.read("nbr"), s.read("nnb")
        o64.write("nbr", rowmajor_lists(nbr, nnb, n).reshape(-1))
        o64.write("nnb", nnb)
        s.force()
        o64.force()
        F = s.read("F").reshape(-1, 4).astype(np.float64)
        F64 = o64.read("F").reshape(-1, 4)
        hn = o64.read("hn")
        ok = (F[:, 3] == F64[:, 3]) & (F64[:, 3] > 0)
        ferr = np.abs(F[ok, :3] - F64[ok, :3]).max(axis=1) / (hn[ok] * F64[ok, 3])
        o64.write("F", F.reshape(-1))
        s.step_tail()
        o64.move_only()
        P = s.read("P").reshape(-1, 3).astype(np.float64)
        P64 = o64.read("P").reshape(-1, 3)
        t = s.read("typ")
        same = t == o64.read("typ")
        free = same & (nd.typ == 0) & (t == 0)
        dif = np.abs(P - P64).max(axis=1)
        perr = (dif / np.maximum(np.abs(P64).max(axis=1), hn))[free]
        proj = (dif / hn)[same & ~free]
    record_property("max_force_rel_err", float(ferr.max()))
    record_property("max_free_position_rel_err", float(perr.max()))
    record_property("max_trapped_position_rel_err", float(proj.max()) if proj.size else 0.0)
    assert ferr.max() <= 1e-6 and perr.max() <= 1e-6
    assert proj.size == 0 or proj.max() <= 1e-2
    assert (~same).sum() <= n // 1000


def test_crowded_bin_rebuild_bit_exact(ref, cuda_lib):
    """3,000 nodes packed into one hash bin (sphere_small's bins are 3.2 voxels
    wide; this cube lies inside bin (7, 7, 7)): the in-bin order is sorted by
    the whole block instead of one thread, and keys, sorted ids, bin starts,
    bin-order positions and lists still equal relax_cpu's rebuild."""
    g, nd = cases.sphere_small()
    nd = nd.copy()
    rng = np.random.default_rng(21)
    idx = rng.choice(nd.size(), 3000, replace=False)
    nd.P[idx] = rng.uniform(22.0, 25.0, (3000, 3)).astype(np.float32)
    nd.typ[idx] = 0
    prm = cases.params(3)
    rs = ref.state(g, prm, nd.copy())
    rs.rebuild()
    cs = rs.read("cstart")
    assert np.diff(cs).max() >= 3000
    with Session(g, prm, nd.copy()) as s:
        s.rebuild()
        for a in ("key", "sorted", "cstart", "nnb"):
            d = first_diff(s.read(a), rs.read(a))
            assert d is None, f"{a}: {d}"
        assert same_bits(s.read("Ps"), rs.read("Ps"))
        n = nd.size()
        nnb = rs.read("nnb")
        d = first_diff(rowmajor_lists(s.read("nbr"), nnb, n), rowmajor_lists(rs.read("nbr"), nnb, n))
        assert d is None, f"nbr: {d}"
        rs.force()
        s.force()
        assert first_diff(s.read("F"), rs.read("F")) is None


@pytest.mark.parametrize("name", ["shells_small", "tpm_small", "ref_phantom"])
def test_session_lists_pass_the_host_checker(name, ref, cuda_lib):
    """The session's truss lists obey the list build's rules (host checker
    v2m_validate_lists) after the first build and after iterations in which
    nodes refreshed their own lists."""
    g, nd = load_case(name, ref)
    with Session(g, cases.params(20), nd.copy()) as s:
        s.rebuild()
        assert s.validate_lists() == ""
        s.iterate(12, graph=False)
        assert s.validate_lists() == ""


@pytest.mark.parametrize("policy", [1, 2])
@pytest.mark.parametrize("name", ["sphere64", "shells_small"])
def test_rebuild_policy_extensions_match_oracle(name, policy, cuda_lib):
    """Extensions without a reference counterpart, against the FP32 C
    restatement (which equals relax_cpu under the reference policy): policy 1
    rebuilds when some node moved more than 0.1 h since the last build; policy 2
    keeps the first build's lists for the whole run (the fixed edge list of the
    64^3 sphere workload)."""
    from oracle.oracle import Oracle
    g, nd = getattr(cases, name)()
    prm = RelaxParams(max_iters=60, dt=0.2, dptol=0.0, rebuild_policy=policy)
    a = nd.copy()
    sa = Oracle("f32").relax(g, prm, a)
    b = nd.copy()
    sb = relax_cl(g, prm, b)
    assert sa.iters == sb.iters and sa.rebuilds == sb.rebuilds
    if policy == 2:
        assert sb.rebuilds == 1
    for f in ("P", "typ", "part"):
        d = first_diff(getattr(b, f), getattr(a, f))
        assert d is None, f"{f}: {d}"
