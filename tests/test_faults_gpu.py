"""Error paths forced without faulting the GPU (host-side limits in
xb_tuning): an allocation refused as out of memory, and the device-side level
bound of the level loop firing.  Each must come back as a status -- XB_ERR_OOM,
XB_ERR_STATE -- with the call returning promptly (the level loop stops at the
bound instead of running on), and the same context must give correct tables
afterwards.  The reference engine only terminates on such errors
(apps/xb/src/include/utils/utils_gpu.h:54-63); these statuses are new."""
import numpy as np
import pytest

import xbtrav
from oracle import oracle as O
from xbtrav import serve

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rmat12():
    return xbtrav.HostCSR.rmat(12, 16, seed=606).arrays()


def _fresh_ctx(**kw):
    c = xbtrav.Context(0)
    c.set_tuning(**kw)
    return c


def _expect(status, fn):
    with pytest.raises(xbtrav.XbError) as e:
        fn()
    assert e.value.status == status, (e.value.status, str(e.value))
    return e.value


def test_workspace_cap_gives_oom_on_every_path_then_recovers(rmat12):
    ro, ci = rmat12
    src = xbtrav.select_sources_csr(ro, 7, 70)
    c = _fresh_ctx(workspace_cap=4096)
    g = c.upload_arrays(ro, ci)
    err = _expect(xbtrav.XB_ERR_OOM, lambda: c.traverse(g, src))
    assert "workspace cap" in str(err)
    _expect(xbtrav.XB_ERR_OOM, lambda: c.traverse_batched([(g, src)]))
    g.set_weights(xbtrav.symmetric_weights(ro, ci, 1, 1, 10))
    _expect(xbtrav.XB_ERR_OOM, lambda: c.multi_sssp(g, src))
    _expect(xbtrav.XB_ERR_OOM, lambda: c.max_match(g))
    _expect(xbtrav.XB_ERR_OOM, lambda: c.slot_launch(0, g, src[:10]))
    # lifting the cap: the same context and graph work again
    c.set_tuning(workspace_cap=0)
    lv, pr, _, _ = O.msbfs(ro, ci, src)
    r = c.traverse(g, src)
    np.testing.assert_array_equal(r.level, lv)
    np.testing.assert_array_equal(r.parent, pr)
    res, _ = c.traverse_batched([(g, src)])
    np.testing.assert_array_equal(res[0].level.cpu().numpy(), lv)
    g.close()
    c.close()


@pytest.mark.parametrize("words", [1, 4])
def test_level_cap_stops_the_loop_with_state_error_then_recovers(rmat12, words):
    """The cap sits below the graph's depth, so every pass still has a live
    frontier when it reaches it: the plain path's host loop, the batched
    path's device WHILE loop and a serving slot's captured loop all stop
    there and report XB_ERR_STATE."""
    ro, ci = rmat12
    src = xbtrav.select_sources_csr(ro, 8, 130)
    lv, pr, _, _ = O.msbfs(ro, ci, src)
    assert lv.max() >= 3
    c = _fresh_ctx(words=words, level_cap=2, chains=2)
    g = c.upload_arrays(ro, ci)
    err = _expect(xbtrav.XB_ERR_STATE, lambda: c.traverse(g, src))
    assert "level bound" in str(err)
    _expect(xbtrav.XB_ERR_STATE, lambda: c.traverse_batched([(g, src)]))
    c.slot_launch(0, g, src[:10])
    _expect(xbtrav.XB_ERR_STATE, lambda: c.slot_poll(0, wait=True))
    # a cap at or above the depth changes nothing
    c.set_tuning(level_cap=int(lv.max()) + 1)
    r = c.traverse(g, src)
    np.testing.assert_array_equal(r.level, lv)
    np.testing.assert_array_equal(r.parent, pr)
    # and without a cap every path gives the oracle's tables again
    c.set_tuning(level_cap=0)
    r = c.traverse(g, src)
    np.testing.assert_array_equal(r.level, lv)
    np.testing.assert_array_equal(r.parent, pr)
    res, _ = c.traverse_batched([(g, src)])
    np.testing.assert_array_equal(res[0].level.cpu().numpy(), lv)
    np.testing.assert_array_equal(res[0].parent.cpu().numpy(), pr)
    srv = serve.Server(c, slots=1, reserve_bytes=0)
    q = srv.submit(g, src[:10], want="digest")
    srv.drain()
    np.testing.assert_array_equal(q.digest, O.row_digests(lv[:10], pr[:10]))
    c.slots_release()
    g.close()
    c.close()
