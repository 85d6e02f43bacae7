"""Parity on the configurations the benchmark numbers are quoted on.

The default benchmark workload is R-MAT scale 22 / edge factor 16 (seed
0x5EED), 1024 sources drawn with seed 0x5EED + 1, traversed by
xb_traverse_batched at the context's default tuning (64-bit words, four per
vertex = 256 sources per pass, 4 chains, heavy cutoff 256, pull factor 256).
These tests run exactly that call and compare a spread sample of source rows
bit-exactly with the CPU oracle (levels and min-id parents): every pass, every
word of a pass and bit positions 0 and 63 of each word, plus seeded random
rows (positions in the engine's pass grouping, xb_graph_source_order, mapped
to the caller's rows).  The plain path (xb_traverse) on the same inputs must give identical
tables in full.  The uneven 128-graph workload is checked the same way on
sampled queries, and R-MAT 20 at the default tuning (hubs above degree 4096,
so the chunked hub pull runs inside the captured level loop) in full.

Reference semantics: plain BFS with Parents[s] = s (apps/ligra/apps/BFS.C:42-53);
levels are hop distances; parents follow the min-id rule (a valid predecessor
one level up, the smallest id), which the oracle restates.
"""
import numpy as np
import pytest

import xbtrav
from oracle import oracle as O

pytestmark = pytest.mark.gpu

SEED = 0x5EED  # the benchmark's graph seed; sources use SEED + 1


def _sample_rows(k: int, per_pass: int, extra: int, seed: int) -> np.ndarray:
    """Rows covering every pass and word of the default layout at bit
    positions 0 and 63, plus `extra` seeded random rows."""
    rows = []
    for p0 in range(0, k, per_pass):
        for w0 in range(p0, min(k, p0 + per_pass), 64):
            rows += [w0, min(k - 1, w0 + 63)]
    rng = np.random.default_rng(seed)
    rows += list(rng.choice(k, size=extra, replace=False))
    return np.unique(np.array(rows, np.int64))


def _check_rows(ro, ci, src, rows, level_dev, parent_dev):
    import torch

    lv, pr, _, _ = O.msbfs(ro, ci, src[rows])
    idx = torch.from_numpy(rows).to(level_dev.device)
    np.testing.assert_array_equal(level_dev.index_select(0, idx).cpu().numpy(), lv)
    np.testing.assert_array_equal(parent_dev.index_select(0, idx).cpu().numpy(), pr)


@pytest.fixture(scope="module")
def rmat22():
    csr = xbtrav.HostCSR.rmat(22, 16, 0.57, 0.19, 0.19, seed=SEED)
    ro, ci = csr.arrays()
    return csr, ro, ci


def test_headline_batched_and_plain_rmat22_k1024(rmat22):
    import torch

    csr, ro, ci = rmat22
    ctx = xbtrav.Context(0)
    tun = ctx.tuning()
    assert (tun["word_bits"], tun["words"], tun["chains"], tun["heavy_degree"]) == (64, 4, 4, 256)
    g = ctx.upload(csr)
    src = g.select_sources(SEED + 1, 1024)
    assert np.array_equal(src, xbtrav.select_sources_csr(ro, SEED + 1, 1024))
    dev = torch.device("cuda", 0)
    src_dev = torch.from_numpy(src).to(dev)
    lv_b = torch.empty((1024, g.n), dtype=torch.int32, device=dev)
    pr_b = torch.empty_like(lv_b)
    _, st = ctx.traverse_batched([(g, src_dev)], outputs=[(lv_b, pr_b)])
    assert st["batches"] == 4
    # traversal positions (pass, word, bit) -> the caller's rows through the
    # pass grouping, which the engine applies to these 1024 sources
    order = g.source_order(src).astype(np.int64)
    assert np.array_equal(np.sort(order), np.arange(1024))
    rows = np.unique(order[_sample_rows(1024, 256, 8, 2024)])
    assert len(rows) >= 40
    _check_rows(ro, ci, src, rows, lv_b, pr_b)
    # the plain per-call path on the same inputs: identical tables in full
    lv_p = torch.empty_like(lv_b)
    pr_p = torch.empty_like(lv_b)
    plain = ctx.traverse(g, src_dev, out="device", level=lv_p, parent=pr_p)
    assert bool(torch.equal(lv_p, lv_b))
    assert bool(torch.equal(pr_p, pr_b))
    assert plain.stats["edges_traversed"] == st["edges_traversed"]
    g.close()
    ctx.close()


def test_rmat20_batched_default_tuning_with_hubs():
    """R-MAT 20 / ef 16 at the default tuning: vertices above degree 4096 are
    pulled in chunks by many warps (k_pull_hubs) inside the captured level
    loop; one full pass of 256 sources, every row against the oracle."""
    csr = xbtrav.HostCSR.rmat(20, 16, 0.57, 0.19, 0.19, seed=SEED)
    ro, ci = csr.arrays()
    assert int(np.diff(ro).max()) > 4096
    ctx = xbtrav.Context(0)
    g = ctx.upload(csr)
    src = g.select_sources(SEED + 1, 256)
    res, st = ctx.traverse_batched([(g, src)])
    lv, pr, edges, reached = O.msbfs(ro, ci, src)
    np.testing.assert_array_equal(res[0].level.cpu().numpy(), lv)
    np.testing.assert_array_equal(res[0].parent.cpu().numpy(), pr)
    assert st["edges_traversed"] == edges and st["reached"] == reached
    g.close()
    ctx.close()


def test_uneven_128_graph_workload_sampled_queries():
    """The uneven workload exactly as the benchmark builds it (128 R-MAT
    graphs, scales U[10,20], edge factors {4,8,16,32}, 1..512 sources each,
    one concatenated CSR, one word per pass, 8 chains): 16 sampled queries,
    up to 12 rows each, against the oracle."""
    import torch

    import bench

    specs = bench.multi_instances(128, SEED)
    hosts = [xbtrav.HostCSR.rmat(sc, ef, 0.57, 0.19, 0.19, seed=gs) for sc, ef, _, gs in specs]
    ctx = xbtrav.Context(0)
    ctx.set_tuning(words=1, chains=8)
    graphs = ctx.upload_batch(hosts)
    dev = torch.device("cuda", 0)
    queries = [(g, torch.from_numpy(g.select_sources(gs + 1, k)).to(dev)) for (_, _, k, gs), g in zip(specs, graphs)]
    res, st = ctx.traverse_batched(queries)
    assert st["batches"] >= 128
    rng = np.random.default_rng(128)
    picks = sorted(set(rng.choice(128, size=16, replace=False)) | {int(np.argmax([s[0] for s in specs]))})
    for qi in picks:
        ro, ci = hosts[qi].arrays()
        src = queries[qi][1].cpu().numpy()
        rows = np.unique(np.concatenate([[0, len(src) - 1], rng.choice(len(src), size=min(10, len(src)),
                                                                         replace=False)])).astype(np.int64)
        _check_rows(ro, ci, src, rows, res[qi].level, res[qi].parent)
    for g in graphs:
        g.close()
    ctx.close()
