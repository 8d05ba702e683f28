"""Large results (16 MB or more) are downloaded into pinned blocks that the
library lends to the caller until gqm_free_result and then reuses.  A block is
never lent twice at once, and a reused block holds the new result, not the
old one."""
import gc
import hashlib

import numpy as np
import pytest

from gpu_cdt_refine_b200 import inputs, refine

pytestmark = pytest.mark.gpu

FIELDS = ("pointlist", "trianglelist", "neighborlist", "segmentlist")


def _digests(c):
    return {f: hashlib.sha256(np.ascontiguousarray(getattr(c, f)).tobytes()).hexdigest() for f in FIELDS}


def test_results_in_reused_blocks_stay_distinct(gpu):
    big = inputs.clustered(seed=31, n=500_000, nseg=25_000)  # a result of ~45 MB
    small = inputs.clustered(seed=32, n=300_000, nseg=15_000)
    a, _ = refine.refine(big, 20.0, 1, 1)
    want_big = _digests(a)
    assert a.pointlist.nbytes + 2 * a.trianglelist.nbytes >= 16 << 20
    b, _ = refine.refine(small, 20.0, 1, 1)  # a still alive: b takes another block
    want_small = _digests(b)
    assert a.pointlist.ctypes.data != b.pointlist.ctypes.data
    del a
    gc.collect()
    c, _ = refine.refine(big, 20.0, 1, 1)  # may reuse a's block
    d, _ = refine.refine(big, 20.0, 1, 1)  # c alive: must not share its block
    assert len({b.pointlist.ctypes.data, c.pointlist.ctypes.data, d.pointlist.ctypes.data}) == 3
    assert _digests(c) == want_big and _digests(d) == want_big and _digests(b) == want_small
    del b, c, d
    gc.collect()
    e, _ = refine.refine(small, 20.0, 1, 1)  # a freed block of the larger result fits it
    assert _digests(e) == want_small


def test_batch_results_share_one_block(gpu):
    """A persistent batch whose outputs total 16 MB or more is downloaded into
    one pinned block shared by its domains: every domain's arrays lie inside
    it, the block is reused only after the last domain's result is released,
    and reused, it holds the new results."""
    doms, thetas = inputs.batch_domains(96, seed=20261231)
    got, _ = refine.refine_batch_persistent(doms, thetas)
    assert sum(g.pointlist.nbytes + 2 * g.trianglelist.nbytes for g in got) >= 16 << 20
    want = [_digests(g) for g in got]
    addrs = sorted(g.pointlist.ctypes.data for g in got)
    assert addrs[-1] - addrs[0] < sum(g.pointlist.nbytes + 3 * g.trianglelist.nbytes for g in got) + (1 << 20)
    keep = got[len(got) // 2]  # one domain still alive: the next batch takes another block
    lo = addrs[0]
    del got
    gc.collect()
    again, _ = refine.refine_batch_persistent(doms, thetas)
    assert [_digests(g) for g in again] == want and _digests(keep) == want[len(want) // 2]
    lo2 = min(g.pointlist.ctypes.data for g in again)
    assert lo2 != lo
    del keep, again
    gc.collect()
    third, _ = refine.refine_batch_persistent(doms, thetas)  # both blocks free: one is reused
    assert min(g.pointlist.ctypes.data for g in third) in (lo, lo2)
    assert [_digests(g) for g in third] == want
