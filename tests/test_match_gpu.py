"""The CUDA maximum matching (xb_max_match through the C ABI): the result
is a matching of the graph and its size equals the oracle's (Edmonds), the
reference CPU engine's, and scipy's on bipartite graphs.  Matchings are not
unique; the size is."""
import numpy as np
import pytest

import xbtrav
from oracle import oracle as O

from test_match_oracle import NAMED, _csr, _random_pairs

pytestmark = pytest.mark.gpu


def _check(ctx, ro, ci, init=None, want=None):
    g = ctx.upload_arrays(ro, ci)
    mate, st = ctx.max_match(g, init=init)
    g.close()
    assert O.check_matching(ro, ci, mate) == 0
    if want is None:
        want, _ = O.max_match(ro, ci)
    assert int((mate >= 0).sum()) // 2 == want
    assert st["reached"] == want
    return mate, st


def _greedy(n, ro, ci, order):
    mate = np.full(n, -1, np.int32)
    for v in order:
        if mate[v] >= 0:
            continue
        for w in ci[ro[v]:ro[v + 1]]:
            if mate[w] < 0 and w != v:
                mate[v], mate[w] = w, v
                break
    return mate


@pytest.mark.parametrize("name", sorted(NAMED))
def test_named_graphs(ctx, name):
    n, pairs = NAMED[name]
    ro, ci = _csr(n, pairs)
    _check(ctx, ro, ci)
    _check(ctx, ro, ci, init=_greedy(n, ro, ci, range(n - 1, -1, -1)))


@pytest.mark.parametrize("seed", range(30))
def test_random_graphs(ctx, seed):
    rng = np.random.default_rng(100 + seed)
    n = int(rng.integers(2, 120))
    ro, ci = _csr(n, _random_pairs(rng, n, float(rng.uniform(0.02, 0.4))))
    _check(ctx, ro, ci)
    _check(ctx, ro, ci, init=_greedy(n, ro, ci, rng.permutation(n)))


@pytest.mark.parametrize("graph", [("rmat", 12, 16), ("rmat", 14, 4), ("rmat", 16, 16), ("er", 50000, 40000)])
def test_generated_graphs(ctx, graph):
    kind, a, b = graph
    h = xbtrav.HostCSR.rmat(a, b, seed=29) if kind == "rmat" else xbtrav.HostCSR.er(a, b, seed=29)
    ro, ci = h.arrays()
    h.close()
    want = (O.ref_max_match(ro, ci, threads=8)[0] if O.ref_match_available() else O.max_match(ro, ci)[0])
    _check(ctx, ro, ci, want=want)


def test_bipartite_equals_scipy(ctx):
    from scipy.sparse import csr_matrix
    from scipy.sparse.csgraph import maximum_bipartite_matching

    rng = np.random.default_rng(8)
    a, b = 3000, 2500
    k = 9000
    pairs = {(int(x), int(y)) for x, y in zip(rng.integers(0, a, k), rng.integers(0, b, k))}
    bip = csr_matrix((np.ones(len(pairs)), ([p[0] for p in pairs], [p[1] for p in pairs])), shape=(a, b))
    want = int((maximum_bipartite_matching(bip, perm_type="column") >= 0).sum())
    ro, ci = _csr(a + b, [(x, a + y) for x, y in pairs])
    _check(ctx, ro, ci, want=want)


def test_large_rmat_against_reference(ctx):
    if not O.ref_match_available():
        pytest.skip("reference matching engine not built")
    h = xbtrav.HostCSR.rmat(18, 16, seed=31)
    ro, ci = h.arrays()
    h.close()
    want, _ = O.ref_max_match(ro, ci, threads=16)
    _, st = _check(ctx, ro, ci, want=want)
    assert st["batches"] >= 2 and st["vertices_scanned"] == want  # every augmentation from the empty matching


def test_device_mate_in_place_and_traversal_after(ctx):
    import torch

    h = xbtrav.HostCSR.rmat(13, 8, seed=4)
    ro, ci = h.arrays()
    h.close()
    g = ctx.upload_arrays(ro, ci)
    src = xbtrav.select_sources_csr(ro, 2, 64)
    r0 = ctx.traverse(g, src)
    t = torch.full((g.n,), -1, dtype=torch.int32, device="cuda")
    out, _ = ctx.max_match(g, init=t)
    mate = out.cpu().numpy()
    assert O.check_matching(ro, ci, mate) == 0
    assert int((mate >= 0).sum()) // 2 == O.max_match(ro, ci)[0]
    r1 = ctx.traverse(g, src)  # the workspace is rebuilt for the traversal
    np.testing.assert_array_equal(r1.level, r0.level)
    np.testing.assert_array_equal(r1.parent, r0.parent)
    g.close()


def test_invalid_initial_matching(ctx):
    ro, ci = _csr(4, [(0, 1), (1, 2), (2, 3)])
    g = ctx.upload_arrays(ro, ci)
    with pytest.raises(xbtrav.XbError):
        ctx.max_match(g, init=np.array([1, -1, -1, -1], np.int32))  # not symmetric
    with pytest.raises(xbtrav.XbError):
        ctx.max_match(g, init=np.array([3, -1, -1, 0], np.int32))  # not an edge
    mate, _ = ctx.max_match(g, init=np.array([-1, 2, 1, -1], np.int32))  # augments through 1-2
    assert int((mate >= 0).sum()) == 4
    g.close()


def test_cpp_engine_matches_oracle(tmp_path):
    """The reference-shaped C++ class (MaximumMatchingEngine::FindMaximumMatch,
    nnodes = exposed) through the example program."""
    import subprocess

    from test_host_abi import _build_example

    exe = _build_example(tmp_path)
    out = subprocess.run([exe, "--rmat", "12", "16", "1", "1", "--match"], capture_output=True, text=True,
                         check=True).stdout
    kv = dict(x.split("=") for x in out.split())
    h = xbtrav.HostCSR.rmat(12, 16, seed=0x5EED)
    ro, ci = h.arrays()
    h.close()
    assert int(kv["matching_size"]) == O.max_match(ro, ci)[0]


def test_degenerate_graphs(ctx):
    # one vertex; isolated vertices only; a single edge; a perfect matching given as the start
    cases = [(np.array([0, 0], np.int64), np.zeros(0, np.int32), None, 0),
             (np.zeros(6, np.int64), np.zeros(0, np.int32), None, 0),
             (np.array([0, 1, 2], np.int64), np.array([1, 0], np.int32), None, 1),
             (np.array([0, 1, 2], np.int64), np.array([1, 0], np.int32), np.array([1, 0], np.int32), 1)]
    for ro, ci, init, want in cases:
        g = ctx.upload_arrays(ro, ci)
        mate, st = ctx.max_match(g, init=init)
        g.close()
        assert O.check_matching(ro, ci, mate) == 0
        assert int((mate >= 0).sum()) // 2 == want == st["reached"]


def test_runner_cli_modes(tmp_path):
    """xbtrav_run (the reference runners' flags) on a text CSR: match, traverse
    and sssp summaries agree with the oracle."""
    import subprocess

    from test_host_abi import _build_example

    exe = _build_example(tmp_path, "xbtrav_run")
    h = xbtrav.HostCSR.rmat(11, 8, seed=0x5EED)
    ro, ci = h.arrays()
    rp, cp = str(tmp_path / "row.txt"), str(tmp_path / "col.txt")
    h.save_text(rp, cp)
    h.close()

    def run(*extra):
        out = subprocess.run([exe, f"--row_offsets={rp}", f"--col_indices={cp}", "--rounds=3", *extra],
                             capture_output=True, text=True, check=True).stdout
        return dict(line.split(": ", 1) for line in out.splitlines() if ": " in line)

    kv = run("--mode=match")
    assert int(kv["Matching Size"]) == O.max_match(ro, ci)[0]
    assert int(kv["Num of Nodes"]) == len(ro) - 1 and len([k for k in kv if k == "Average runtime"]) == 1
    src = xbtrav.select_sources_csr(ro, 99, 50)
    kv = run("--mode=traverse", "--src_count=50", "--seed=99")
    _, _, edges, reached = O.msbfs(ro, ci, src)
    assert int(kv["Number of Processed Edges"]) == edges
    assert int(kv["Reached (source, vertex) pairs"]) == reached
    kv = run("--mode=sssp", "--src_count=50", "--seed=99", "--weight_max=20")
    d = O.msssp(ro, ci, xbtrav.symmetric_weights(ro, ci, 99, 1, 20), src)
    assert int(kv["Reached Vertices"]) == int((d < 3.0e37).sum())
