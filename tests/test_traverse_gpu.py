"""Parity of the CUDA traversal (through the C ABI) with the CPU oracle.

Bar: levels bit-exact; parents bit-exact under the min-id rule (smallest-id
neighbour one level up; the source is its own parent; -1 unreached).  The
golden fixtures additionally pin levels to the reference's own
findShortestPath and reachability to the reference's Ligra BFS.
"""
import glob
import os

import numpy as np
import pytest

import xbtrav
from oracle import oracle as O

pytestmark = pytest.mark.gpu

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))
VARIANTS = [
    dict(word_bits=64, words=1),
    dict(word_bits=32, words=1),
    dict(word_bits=64, words=2),
    dict(word_bits=64, words=4),
    dict(word_bits=32, words=4),
]


def _tune(ctx, **kw):
    base = dict(word_bits=64, words=1, pull_alpha=4.0, heavy_degree=2048, timing=0, tile=0, push_beta=0.0)
    base.update(kw)
    ctx.set_tuning(**base)


def _assert_parity(ctx, ro, ci, src, res=None, check_stats=True):
    g = ctx.upload_arrays(ro, ci)
    r = ctx.traverse(g, src) if res is None else res(g)
    lv, pr, edges, reached = O.msbfs(ro, ci, src, rule=O.RULE_MINID)
    np.testing.assert_array_equal(r.level, lv)
    np.testing.assert_array_equal(r.parent, pr)
    if check_stats:
        assert r.stats["edges_traversed"] == edges
        assert r.stats["reached"] == reached
    g.close()
    return r


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
@pytest.mark.parametrize("variant", range(len(VARIANTS)))
def test_golden_fixtures(ctx, path, variant):
    z = np.load(path)
    ro, ci, src = z["ro"], z["ci"], z["sources"]
    _tune(ctx, **VARIANTS[variant])
    g = ctx.upload_arrays(ro, ci)
    r = ctx.traverse(g, src)
    # reference pins: findShortestPath levels, Ligra reachability
    S, D = z["pair_src_idx"], z["pair_dst"]
    np.testing.assert_array_equal(r.level[S, D], z["pair_level"])
    np.testing.assert_array_equal(r.level >= 0, z["ligra_parent"] >= 0)
    lv, pr, _, _ = O.msbfs(ro, ci, src)
    np.testing.assert_array_equal(r.level, lv)
    np.testing.assert_array_equal(r.parent, pr)
    g.close()


@pytest.mark.parametrize("variant", range(len(VARIANTS)))
@pytest.mark.parametrize("alpha", [1e-6, 4.0, 1e6])
@pytest.mark.parametrize("heavy", [32, 2048])
def test_rmat12_push_pull_heavy_paths(ctx, variant, alpha, heavy):
    """alpha=1e6 forces pull every level, 1e-6 push every level; heavy=32
    routes most vertices through the block-per-vertex kernels."""
    g = xbtrav.HostCSR.rmat(12, 16, seed=77)
    ro, ci = g.arrays()
    src = xbtrav.select_sources_csr(ro, 78, 100)
    _tune(ctx, pull_alpha=alpha, heavy_degree=heavy, **VARIANTS[variant])
    r = _assert_parity(ctx, ro, ci, src)
    if alpha == 1e6:
        assert r.stats["push_levels"] == 0
    if alpha == 1e-6:
        assert r.stats["pull_levels"] == 0


@pytest.mark.parametrize("k", [1, 31, 63, 64, 65, 130])
def test_ragged_source_counts(ctx, k):
    g = xbtrav.HostCSR.er(3000, 5000, seed=k)
    ro, ci = g.arrays()
    src = xbtrav.select_sources_csr(ro, k + 1, k)
    _tune(ctx)
    _assert_parity(ctx, ro, ci, src)


def test_duplicate_and_isolated_sources(ctx):
    g = xbtrav.HostCSR.rmat(10, 2, seed=5)
    ro, ci = g.arrays()
    deg = np.diff(ro)
    iso = np.nonzero(deg == 0)[0]
    assert len(iso) > 0
    src = np.array([3, 3, int(iso[0]), 7, 3, int(iso[-1])] * 12, np.int32)
    for v in VARIANTS:
        _tune(ctx, **v)
        _assert_parity(ctx, ro, ci, src)


def test_config_rmat16_k64(ctx):
    """R-MAT scale 16, edge factor 16, 64 seeded sources (the CPU-runnable config)."""
    g = xbtrav.HostCSR.rmat(16, 16, seed=0x5EED)
    ro, ci = g.arrays()
    src = xbtrav.select_sources_csr(ro, 0x5EED + 1, 64)
    for v in VARIANTS[:2]:
        _tune(ctx, **v)
        _assert_parity(ctx, ro, ci, src)


def test_config_er335k_k256_host_buffers(ctx):
    """Uniform graph, 335,000 vertices, ~1.85M undirected edges, 256 sources, one call."""
    g = xbtrav.HostCSR.er(335_000, 1_850_000, seed=0x5EED)
    ro, ci = g.arrays()
    src = xbtrav.select_sources_csr(ro, 0x5EED + 1, 256)
    _tune(ctx)
    _assert_parity(ctx, ro, ci, src)


def test_device_outputs_match_host_outputs(ctx):
    import torch

    g = xbtrav.HostCSR.rmat(14, 8, seed=9)
    ro, ci = g.arrays()
    src = xbtrav.select_sources_csr(ro, 10, 96)
    _tune(ctx)
    dg = ctx.upload_arrays(ro, ci)
    rh = ctx.traverse(dg, src)
    rd = ctx.traverse(dg, torch.from_numpy(src).cuda(), out="device")
    np.testing.assert_array_equal(rd.level.cpu().numpy(), rh.level)
    np.testing.assert_array_equal(rd.parent.cpu().numpy(), rh.parent)
    # repeated calls are identical (state fully reset between calls)
    rh2 = ctx.traverse(dg, src)
    np.testing.assert_array_equal(rh2.level, rh.level)
    np.testing.assert_array_equal(rh2.parent, rh.parent)
    dg.close()


def test_argument_errors(ctx):
    g = xbtrav.HostCSR.rmat(8, 4, seed=1)
    ro, ci = g.arrays()
    dg = ctx.upload_arrays(ro, ci)
    with pytest.raises(xbtrav.XbError) as e:
        ctx.traverse(dg, np.array([0, 256], np.int32))
    assert e.value.status == xbtrav.XB_ERR_ARG
    with pytest.raises(xbtrav.XbError) as e:
        ctx.set_tuning(word_bits=48)
    assert e.value.status == xbtrav.XB_ERR_ARG
    r = ctx.traverse(dg, np.zeros(0, np.int32))
    assert r.level.shape == (0, 256)
    dg.close()


def test_rmat20_k128_levels_and_parents(ctx):
    """Larger graph (31M entries, hubs of degree ~60k) against the oracle."""
    g = xbtrav.HostCSR.rmat(20, 16, seed=0x5EED)
    ro, ci = g.arrays()
    src = xbtrav.select_sources_csr(ro, 0x5EED + 1, 128)
    _tune(ctx, timing=1)
    r = _assert_parity(ctx, ro, ci, src)
    assert r.stats["pull_levels"] > 0 and r.stats["push_levels"] > 0


def test_cpp_host_api_matches_python_binding(ctx, tmp_path):
    """The reference-style C++ layer (host/xbtrav.hpp) gives the same tables."""
    import subprocess

    from test_host_abi import _build_example

    exe = _build_example(tmp_path)
    out = subprocess.run([exe, "--rmat", "12", "16", "64", "0x77"], capture_output=True, text=True, check=True).stdout
    kv = dict(x.split("=") for x in out.split())
    csr = xbtrav.HostCSR.rmat(12, 16, seed=0x5EED)
    ro, ci = csr.arrays()
    src = xbtrav.select_sources_csr(ro, 0x77, 64)
    _tune(ctx)
    g = ctx.upload(csr)
    r = ctx.traverse(g, src)
    h = np.uint64(1469598103934665603)
    prime = np.uint64(1099511628211)
    with np.errstate(over="ignore"):
        for x in np.concatenate([r.level.ravel(), r.parent.ravel()]).astype(np.uint32):
            h = (h ^ np.uint64(x)) * prime
    assert kv["checksum"] == f"{int(h):016x}"
    assert int(kv["edges_traversed"]) == r.stats["edges_traversed"]
    # the same sources as three queries in one batched launch (BatchedEngine)
    out_b = subprocess.run([exe, "--rmat", "12", "16", "64", "0x77", "--batched"], capture_output=True, text=True,
                           check=True).stdout
    kvb = dict(x.split("=") for x in out_b.split())
    assert kvb["checksum"] == kv["checksum"]
    assert kvb["edges_traversed"] == kv["edges_traversed"]
    g.close()


def test_autotuner_picks_a_config_that_keeps_parity(ctx, tmp_path):
    from xbtrav import autotune

    csr = xbtrav.HostCSR.rmat(12, 16, seed=31)
    ro, ci = csr.arrays()
    src = xbtrav.select_sources_csr(ro, 32, 96)
    g = ctx.upload(csr)
    space = {"word_bits": [64, 32], "words": [1, 2], "heavy_degree": [128, 256], "pull_alpha": [64.0, 256.0],
             "push_beta": [0.0, 24.0], "tile": [0, 1], "source_order": [0, 1], "chains": [1, 2]}
    for path in ("plain", "batched"):
        # the first stage keeps the current cutoffs: start inside the space
        _tune(ctx, heavy_degree=256, pull_alpha=256.0, chains=2)
        best, table = autotune.autotune(ctx, g, src, space=space, reps=1, path=path)
        assert all(best[k] in space[k] for k in space if path == "batched" or k != "chains")
        assert best == {k: ctx.tuning()[k] for k in best}
        assert len(table) >= 4 + 4 + 2 + 2 + 2
        r = ctx.traverse(g, src)
        lv, pr, _, _ = O.msbfs(ro, ci, src)
        np.testing.assert_array_equal(r.level, lv)
        np.testing.assert_array_equal(r.parent, pr)
    autotune.save(best, str(tmp_path / "t.json"))
    assert autotune.load(str(tmp_path / "t.json")) == best
    g.close()


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_fifo_parents_match_the_reference_search(ctx, path):
    """XB_PARENT_FIFO: parents equal those of the reference's own
    findShortestPath (golden pairs) and the oracle's FIFO rule; levels are
    the min-id run's."""
    z = np.load(path)
    ro, ci, src = z["ro"], z["ci"], z["sources"]
    _tune(ctx)
    g = ctx.upload_arrays(ro, ci)
    r = ctx.traverse(g, src, parent_rule="fifo")
    S, D = z["pair_src_idx"], z["pair_dst"]
    np.testing.assert_array_equal(r.parent[S, D], z["pair_parent"])
    lv, pr, _, _ = O.msbfs(ro, ci, src, rule=O.RULE_FIFO)
    np.testing.assert_array_equal(r.level, lv)
    np.testing.assert_array_equal(r.parent, pr)
    g.close()


@pytest.mark.parametrize("variant", [0, 1, 2, 4])
@pytest.mark.parametrize("out", ["host", "device"])
def test_fifo_parents_rmat_and_er(ctx, variant, out):
    _tune(ctx, **VARIANTS[variant])
    for csr, k in ((xbtrav.HostCSR.rmat(12, 16, seed=41), 150), (xbtrav.HostCSR.er(4000, 12000, seed=42), 70)):
        ro, ci = csr.arrays()
        src = xbtrav.select_sources_csr(ro, 43, k)
        g = ctx.upload(csr)
        r = ctx.traverse(g, src, out=out, parent_rule="fifo")
        lv, pr, _, _ = O.msbfs(ro, ci, src, rule=O.RULE_FIFO)
        level = r.level.cpu().numpy() if out == "device" else r.level
        parent = r.parent.cpu().numpy() if out == "device" else r.parent
        np.testing.assert_array_equal(level, lv)
        np.testing.assert_array_equal(parent, pr)
        g.close()


def test_graph_outliving_its_context():
    """A graph freed after its context was destroyed (e.g. by a garbage
    collector at exit) is released without touching the context; using it
    fails cleanly."""
    c2 = xbtrav.Context(0)
    csr = xbtrav.HostCSR.rmat(8, 4, seed=5)
    g = c2.upload(csr)
    views = c2.upload_batch([csr, csr])
    c2.close()
    c3 = xbtrav.Context(0)
    with pytest.raises(xbtrav.XbError) as e:
        c3.traverse(g, np.array([0], np.int32))
    assert e.value.status == xbtrav.XB_ERR_STATE
    g.close()
    for v in views:
        v.close()
    c3.close()