"""The reference's Python file formats and helpers (parlayann_b200.wrapper):
.bin points (point_range.h:74-117), .ibin groundtruth (types.h:38-107), the
range groundtruth file (compute_range_groundtruth.cpp:64-87), the reference's
float distance and normalisation. CPU only."""
import numpy as np
import pytest

from conftest import random_points
from oracle import oracle as O
from parlayann_b200 import wrapper as W


@pytest.mark.parametrize("dtype", [np.float32, np.uint8, np.int8])
def test_vectors_file_round_trip(dtype, tmp_path):
    x = random_points(dtype, 37, 11, 1)
    f = str(tmp_path / "x.bin")
    W.vectors_to_file(f, x)
    raw = np.fromfile(f, dtype=np.uint8)
    assert raw[:8].view(np.int32).tolist() == [37, 11] and len(raw) == 8 + x.nbytes
    assert W.vectors_metadata_from_file(f) == (37, 11)
    np.testing.assert_array_equal(W.vectors_from_file(f, dtype), x)


def test_groundtruth_files_round_trip(tmp_path):
    rng = np.random.default_rng(2)
    ids = rng.integers(0, 1000, (9, 5)).astype(np.uint32)
    dists = rng.random((9, 5)).astype(np.float32)
    f = str(tmp_path / "gt.ibin")
    W.groundtruth_to_file(f, ids, dists)
    a, b = W.groundtruth_from_file(f)
    np.testing.assert_array_equal(a, ids)
    np.testing.assert_array_equal(b, dists)
    offs = np.array([0, 3, 3, 7], np.uint64)
    rids = np.arange(7, dtype=np.uint32) * 3
    g = str(tmp_path / "range.gt")
    W.range_groundtruth_to_file(g, offs, rids)
    head = np.fromfile(g, dtype=np.int32)
    assert head[:2].tolist() == [3, 7] and head[2:5].tolist() == [3, 0, 4]
    o2, r2 = W.range_groundtruth_from_file(g)
    np.testing.assert_array_equal(o2, offs)
    np.testing.assert_array_equal(r2, rids)


@pytest.mark.parametrize("dtype,metric", [(np.uint8, 0), (np.int8, 1), (np.float32, 0), (np.float32, 1)])
def test_reference_distances(dtype, metric):
    base = random_points(dtype, 200, 13, 3)
    q = random_points(dtype, 3, 13, 4)
    for i in range(3):
        got = W._distances(q[i], base, metric)
        want = np.array([O.olib().oracle_distance(O._DT[base.dtype], metric, 13, q[i].ctypes.data,
                                                  np.ascontiguousarray(base[j]).ctypes.data) for j in range(200)],
                        np.float32)
        np.testing.assert_array_equal(got.view(np.uint32), want.view(np.uint32))


def test_normalize_and_alpha_rule():
    x = random_points(np.float32, 50, 96, 5) * 3.0
    y = W._normalize(x)
    assert np.allclose(np.linalg.norm(y, axis=1), 1.0, atol=1e-5)
    z = W._normalize(np.zeros((2, 4), np.float32))
    assert not z.any()
    assert W._mips_prepare(x, 1.2)[1] == 1.0                 # < 100 dimensions
    assert W._mips_prepare(random_points(np.float32, 4, 150, 6), 1.2)[1] == 0.98
    assert W._mips_prepare(random_points(np.float32, 4, 256, 7), 1.2)[1] == 1.2


def test_graph_index_needs_a_type():
    with pytest.raises(ValueError):
        W.GraphIndex("points.bin", "index.graph")
