"""Failure detection without a GPU fault: a bounded device wait that runs out reports
ARC_DEVERR_TIMEOUT / ARC_ERR_TIMEOUT, the work after it is skipped on the device, and the context
stays usable.  The wait made to run out is the radix sort's decoupled look-back (a tile waits for
the tiles before it to publish their digit offsets), given a limit of one poll through
ArcLbvhParams.wait_limit; with thousands of tiles started together, some tile always finds its
predecessor unpublished at that limit."""
import numpy as np
import pytest

import helpers as H
from antiradiancecuts_b200 import _lib as L
from antiradiancecuts_b200 import api
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def test_sort_lookback_timeout_is_reported_and_the_context_recovers(ctx):
    d = H.workload("boxes2_720p_64k", 64, 64, 1 << 20)
    ctx.upload_materials(d["mats"])
    dv = ctx.upload_avpls(d["avpls"])
    bvh = api.AvplBvh(ctx)
    seen = None
    for _ in range(5):
        try:
            bvh.build(dv, wait_limit=1)
        except L.ArcError as e:
            seen = e
            break
        assert ctx.synchronize() == 0  # every tile found its predecessor published: try again
    assert seen is not None, "the look-back never ran out at a limit of one poll"
    assert seen.status == L.ARC_ERR_TIMEOUT
    assert b"look-back" in L.load().arc_last_error()
    assert ctx.synchronize() & L.ARC_DEVERR_TIMEOUT
    with pytest.raises(L.ArcError) as e:  # the object holds no tree
        bvh.view()
    assert e.value.status == L.ARC_ERR_INVALID_ARG
    # the next build with the default limit is complete and bit-exact
    bvh.build(dv)
    assert ctx.synchronize() == 0
    got = bvh.host_arrays()
    ref = O.build_tree(d["avpls"], d["dif"])
    for k in ("morton", "sorted_index", "left", "right", "parents"):
        assert np.array_equal(got[k], ref[k]), k
    assert rc_ok(got)
    # and a gather over it completes without a device error
    out = api.Outputs(64, 64)
    api.gather_cut(ctx, bvh, dv, api.GBuffer(d["pos"], d["nrm"]), d["cam"], api.gather_params(),
                   api.cut_params(L.ARC_CUT_ERROR_BOUND, error_bound=0.05, cut_pool_entries=1 << 26), out)
    assert ctx.synchronize() == 0
    assert np.isfinite(out.result64.cpu().numpy()).all()
    bvh.close()


def rc_ok(tree) -> bool:
    rc, _ = O.check_tree(tree["left"], tree["right"], tree["parents"])
    return rc == 0
