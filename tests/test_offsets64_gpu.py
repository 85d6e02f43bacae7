"""The int64-offset kernels (used for graphs of 2^31 - 1 or more entries,
R-MAT 25 / ef 32 and up) on small graphs: XB_OFFSETS64=1 keeps int64 row
offsets on upload, and every path must give the same results as with int32
offsets -- traversal (plain, batched, FIFO parents), multi-source SSSP and
maximum matching, each against the oracle."""
import os

import numpy as np
import pytest

import xbtrav
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture
def wide(ctx):
    os.environ["XB_OFFSETS64"] = "1"
    try:
        h = xbtrav.HostCSR.rmat(12, 16, seed=0x64)
        ro, ci = h.arrays()
        g = ctx.upload(h)
        h.close()
    finally:
        del os.environ["XB_OFFSETS64"]
    assert g.offset_bytes == 8
    yield g, ro, ci
    g.close()


@pytest.mark.parametrize("words", [1, 2])
def test_traversal(ctx, wide, words):
    g, ro, ci = wide
    ctx.set_tuning(words=words)
    try:
        src = xbtrav.select_sources_csr(ro, 5, 100)
        lv, pr, _, _ = O.msbfs(ro, ci, src, rule=O.RULE_MINID)
        r = ctx.traverse(g, src)
        np.testing.assert_array_equal(r.level, lv)
        np.testing.assert_array_equal(r.parent, pr)
        import torch

        outs = [(torch.empty((len(src), g.n), dtype=torch.int32, device="cuda"),
                 torch.empty((len(src), g.n), dtype=torch.int32, device="cuda"))]
        ctx.traverse_batched([(g, torch.from_numpy(src).cuda())], outputs=outs)
        np.testing.assert_array_equal(outs[0][0].cpu().numpy(), lv)
        np.testing.assert_array_equal(outs[0][1].cpu().numpy(), pr)
        rf = ctx.traverse(g, src, parent_rule="fifo")
        _, prf, _, _ = O.msbfs(ro, ci, src, rule=O.RULE_FIFO)
        np.testing.assert_array_equal(rf.parent, prf)
    finally:
        ctx.set_tuning(words=4)


def test_sssp(ctx, wide):
    g, ro, ci = wide
    w = xbtrav.symmetric_weights(ro, ci, 3, 1, 50)
    g.set_weights(w)
    src = xbtrav.select_sources_csr(ro, 9, 33)
    d, _ = ctx.multi_sssp(g, src)
    np.testing.assert_array_equal(d, O.msssp(ro, ci, w, src))


def test_matching(ctx, wide):
    g, ro, ci = wide
    mate, st = ctx.max_match(g)
    assert O.check_matching(ro, ci, mate) == 0
    assert st["reached"] == O.max_match(ro, ci)[0]


def test_int32_by_default(ctx):
    h = xbtrav.HostCSR.rmat(10, 8, seed=1)
    g = ctx.upload(h)
    h.close()
    assert g.offset_bytes == 4
    g.close()


def test_serving_slots(ctx, wide):
    """Serving slots (xb_slot_launch / poll) on an int64-offset graph: tables
    and digests equal the oracle's."""
    from xbtrav import serve

    g, ro, ci = wide
    ctx.set_tuning(words=4)
    srv = serve.Server(ctx, slots=2, reserve_bytes=1 << 30)
    qs = []
    for i, k in enumerate([3, 64, 130]):
        src = g.select_sources(700 + i, k)
        qs.append((src, srv.submit(g, src, want="tables" if i != 1 else "digest")))
    srv.drain()
    for src, q in qs:
        lv, pr, _, _ = O.msbfs(ro, ci, src, rule=O.RULE_MINID)
        if q.want == "tables":
            np.testing.assert_array_equal(q.level.cpu().numpy(), lv)
            np.testing.assert_array_equal(q.parent.cpu().numpy(), pr)
        else:
            from test_serve_gpu import _oracle_digest

            np.testing.assert_array_equal(q.digest, _oracle_digest(lv, pr))
