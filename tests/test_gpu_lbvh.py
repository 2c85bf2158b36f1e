"""LBVH build on the GPU: Morton codes, sorted order, topology and node data equal the CPU
oracle bit for bit."""
import numpy as np
import pytest

import helpers as H
from antiradiancecuts_b200 import _lib as L
from antiradiancecuts_b200 import api, scene
from oracle import oracle as O

pytestmark = pytest.mark.gpu

INT_KEYS = ["morton", "sorted_index", "left", "right", "parents", "size", "materialIndex"]
FLOAT_KEYS = ["randomNumbers", "position", "normal", "incRadiance", "incDirection", "records", "dirstat"]


def _compare(gpu, ref, n):
    for k in INT_KEYS:
        assert np.array_equal(gpu[k], ref[k]), k
    for k in FLOAT_KEYS:
        assert np.array_equal(gpu[k], ref[k]), k  # value equality (+0 == -0)
    gb, rb = gpu["bounds"], ref["bounds"]
    assert np.array_equal(gb.view(np.uint32)[:, [3, 7]], rb.view(np.uint32)[:, [3, 7]])  # child indices
    cols = [0, 1, 2, 4, 5, 6, 8, 9, 10, 11, 12, 13, 14, 15]
    assert np.array_equal(gb[:, cols], rb[:, cols])
    rng = gpu["range"]
    assert (rng[:, 0] <= rng[:, 1]).all() and rng[0, 0] == 0 and rng[0, 1] == n - 1


def _build(ctx, avpls, mats, **kw):
    ctx.upload_materials(mats)
    dv = ctx.upload_avpls(avpls)
    bvh = api.AvplBvh(ctx)
    bvh.build(dv, **kw)
    assert ctx.synchronize() == 0
    return bvh, dv


@pytest.mark.parametrize("name,n", [("room_256_4k", 2), ("room_256_4k", 3), ("room_256_4k", 4096),
                                    ("boxes2_720p_64k", 65536), ("boxes16_1080p_256k", 262144)])
def test_lbvh_bit_exact(ctx, name, n):
    d = H.workload(name, 8, 8, n)
    bvh, _ = _build(ctx, d["avpls"], d["mats"])
    gpu = bvh.host_arrays()
    ref = O.build_tree(d["avpls"], d["dif"])
    _compare(gpu, ref, n)
    assert O.check_tree(gpu["left"], gpu["right"], gpu["parents"])[0] == 0


def test_lbvh_duplicate_positions(ctx):
    d = H.workload("room_256_4k", 8, 8, 4096)
    a = d["avpls"].copy()
    a["position"][::2] = a["position"][0]  # half of the AVPLs share one Morton cell
    bvh, _ = _build(ctx, a, d["mats"])
    gpu = bvh.host_arrays()
    _compare(gpu, O.build_tree(a, d["dif"]), len(a))
    l2, r2 = O.topdown(gpu["morton"])
    assert np.array_equal(gpu["left"], l2) and np.array_equal(gpu["right"], r2)


@pytest.mark.parametrize("consider_normals,bbox_mode", [(False, L.ARC_BBOX_AVPL_REFERENCE), (True, L.ARC_BBOX_SCENE),
                                                         (True, L.ARC_BBOX_AVPL_REFERENCE)])
def test_lbvh_modes(ctx, consider_normals, bbox_mode):
    d = H.workload("boxes2_720p_64k", 8, 8, 20000)
    bvh, _ = _build(ctx, d["avpls"], d["mats"], consider_normals=consider_normals, bbox_mode=bbox_mode)
    gpu = bvh.host_arrays()
    ref = O.build_tree(d["avpls"], d["dif"], bbox_mode=bbox_mode, consider_normals=consider_normals)
    _compare(gpu, ref, len(d["avpls"]))


def test_lbvh_1m_bit_exact_and_invariants(ctx):
    d = H.workload("variant500_1080p_1m", 8, 8)
    n = len(d["avpls"])
    bvh, _ = _build(ctx, d["avpls"], d["mats"])
    gpu = bvh.host_arrays()
    assert np.all(np.diff(gpu["morton"].astype(np.int64)) >= 0)
    assert np.array_equal(np.sort(gpu["sorted_index"]), np.arange(n))
    assert O.check_tree(gpu["left"], gpu["right"], gpu["parents"])[0] == 0
    _compare(gpu, O.build_tree(d["avpls"], d["dif"]), n)


def test_lbvh_rebuild_reuses_buffers(ctx):
    d = H.workload("room_256_4k", 8, 8, 4096)
    bvh, dv = _build(ctx, d["avpls"], d["mats"])
    first = bvh.host_arrays()
    bvh.build(dv)
    assert ctx.synchronize() == 0
    again = bvh.host_arrays()
    for k in INT_KEYS + FLOAT_KEYS:
        assert np.array_equal(first[k], again[k])


def test_lbvh_too_few_avpls(ctx):
    d = H.workload("room_256_4k", 8, 8, 16)
    ctx.upload_materials(d["mats"])
    dv = ctx.upload_avpls(d["avpls"][:1])
    bvh = api.AvplBvh(ctx)
    with pytest.raises(L.ArcError) as e:
        bvh.build(dv)
    assert e.value.status == L.ARC_ERR_TOO_FEW_AVPLS


def test_reference_views(ctx):
    d = H.workload("room_256_4k", 8, 8, 4096)
    bvh, _ = _build(ctx, d["avpls"], d["mats"])
    bp, nd = bvh.reference_views()
    assert bp.numLeafs == 4096 and bp.numNodes == 4095
    raw = ctx.d2h(bp.nodes, np.uint8, 36 * 4095).view(np.int32).reshape(-1, 9)
    gpu = bvh.host_arrays()
    assert np.array_equal(raw[:, 0], gpu["left"]) and np.array_equal(raw[:, 1], gpu["right"])
    f = raw[:, 2:8].view(np.float32)
    assert np.array_equal(f[:, :3], gpu["bounds"][:, 0:3]) and np.array_equal(f[:, 3:], gpu["bounds"][:, 4:7])
    assert np.all(raw[:, 8] == 2)
    pos = ctx.d2h(bp.positions, np.float32, 3 * 4096).reshape(-1, 3)
    assert np.array_equal(pos, d["avpls"]["position"][gpu["sorted_index"]])
