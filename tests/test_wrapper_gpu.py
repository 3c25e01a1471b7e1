"""The reference's Python search surface (parlayann_b200.wrapper) on the GPU:
build_vamana_index from a .bin file, load_index, batch_search /
single_search / batch_search_from_string against Index.search on the same
graph, and check_recall against the brute-force groundtruth."""
import numpy as np
import pytest

import parlayann_b200 as P
from conftest import random_points
from parlayann_b200 import wrapper as W

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dtype,metric", [("uint8", "Euclidian"), ("float", "Euclidian"), ("float", "mips")])
def test_build_load_and_search(dtype, metric, tmp_path, lib_built):
    npdt = {"uint8": np.uint8, "float": np.float32}[dtype]
    base = random_points(npdt, 6000, 24, 201)
    q = random_points(npdt, 300, 24, 202)
    data, graph, qf, gtf = (str(tmp_path / n) for n in ("base.bin", "g.graph", "q.bin", "gt.ibin"))
    W.vectors_to_file(data, base)
    W.vectors_to_file(qf, q)
    W.build_vamana_index(metric, dtype, data, graph, 24, 48, 1.2, True)
    assert W.graph_metadata_from_file(graph) == (6000, 24)
    gi = W.load_index(metric, dtype, data, graph)
    assert type(gi).__name__ == {"uint8": "UInt8", "float": "Float"}[dtype] + metric.replace("mips", "Mips") + "Index"
    ids, dists = gi.batch_search(q, 10, 40)
    # the same graph and points through the plain API
    pts = gi.points
    idx = P.Index(pts, 24, W._METRIC[metric])
    idx.load_graph(graph)
    r = idx.search(q, 10, 40)
    np.testing.assert_array_equal(ids, r.ids)
    np.testing.assert_array_equal(dists.view(np.uint32), r.dists.view(np.uint32))
    np.testing.assert_array_equal(gi.single_search(q[7], 10, 40), r.ids[7])
    ids2, _ = gi.batch_search_from_string(qf, 10, 40)
    np.testing.assert_array_equal(ids2, r.ids)
    # a visit limit stops early (fewer visits than without it)
    lim = idx.search(q, 10, 40, limit=5, allow_short=True)
    ids3, _ = gi.batch_search(q, 10, 40, visit_limit=5)
    np.testing.assert_array_equal(ids3, lim.ids)
    # recall with ties against the exact groundtruth, written as .ibin
    gt_ids, gt_d = idx.groundtruth(q, 50)
    W.groundtruth_to_file(gtf, gt_ids, gt_d)
    rec = gi.check_recall(qf, gtf, ids, 10)
    assert 0.5 < rec <= 1.0
    if dtype == "float" and metric == "Euclidian":
        qi, _ = gi.batch_search(q, 10, 40, quant=True)       # the precision form
        assert gi.check_recall(qf, gtf, qi, 10) > 0.5
    idx.close()
    gi.close()
