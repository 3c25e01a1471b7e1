"""Parity of the CUDA Vamana build (through the C ABI) with the oracle.

The oracle's build is pinned to the reference's own build compiled in place
(tests/test_oracle_pin.py). Given the same insertion order and the same stable
grouping of reverse edges, the GPU build produces the same graph: identical
neighbour lists (the final distance sort orders ties by id on both sides).
"""
import os

import numpy as np
import pytest

import parlayann_b200 as P
from conftest import random_points
from oracle import oracle as O

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def live(g):
    return [tuple(r[1:1 + r[0]].tolist()) for r in g]


@pytest.mark.parametrize("dtype,metric", [(np.uint8, P.L2), (np.int8, P.L2), (np.float32, P.L2),
                                          (np.float32, P.MIPS), (np.uint8, P.MIPS)])
def test_build_matches_oracle(dtype, metric, lib_built):
    base = random_points(dtype, 2500, 24, 71)
    idx = P.Index(base, 12, metric)
    st = idx.build(24, 1.2, num_passes=2)
    g = idx.get_graph()
    o, tot = O.build_graph("oracle", base, 12, 24, 1.2, 2, metric=metric)
    assert live(g) == live(o)
    assert st.dist_cmps == tot
    idx.close()


def test_build_mixture_u8_c0_shape(lib_built):
    """uint8 mixture with the C0 generator's parameters at reduced n."""
    base = P.synth_mixture(P.U8, 6000, 128, 64, 0, 0)
    idx = P.Index(base, 32)
    idx.build(64, 1.2, num_passes=2)
    o, _ = O.build_graph("oracle", base, 32, 64, 1.2, 2)
    assert live(idx.get_graph()) == live(o)
    idx.close()


def test_build_explicit_permutation(lib_built):
    base = random_points(np.float32, 1500, 16, 81)
    perm = np.random.default_rng(3).permutation(1500).astype(np.uint32)
    idx = P.Index(base, 10)
    idx.build(20, 1.3, num_passes=1, perm=perm)
    o, _ = O.build_graph("oracle", base, 10, 20, 1.3, 1, perm=perm)
    assert live(idx.get_graph()) == live(o)
    idx.close()


@pytest.mark.parametrize("nm", ["u8_l2", "f32_l2", "f32_mips"])
def test_build_matches_golden(nm, lib_built):
    z = np.load(os.path.join(GOLD, f"build_{nm}.npz"))
    idx = P.Index(z["base"], int(z["R"]), int(z["metric"]))
    st = idx.build(int(z["L"]), float(z["alpha"]), num_passes=int(z["passes"]), perm=z["perm"])
    g = live(idx.get_graph())
    ref = live(z["graph"])
    for a, b in zip(g, ref):
        assert sorted(a) == sorted(b)
    assert st.dist_cmps == int(z["dist_total"])
    idx.close()


def test_build_then_search_recall(lib_built):
    base = P.synth_mixture(P.F32, 20000, 96, 64, 1, 0, sigma=0.3, normalize=True)
    q = P.synth_mixture(P.F32, 500, 96, 64, 1, 1, sigma=0.3, normalize=True)
    idx = P.Index(base, 32)
    idx.build(64, 1.2, num_passes=1)
    gt, _ = idx.groundtruth(q, 10)
    r = idx.search(q, 10, 64)
    assert P.recall_at_k(r.ids, gt, 10) > 0.9
    idx.close()


_BLOCK_SCRIPT = r"""
import sys
import numpy as np
sys.path.insert(0, {root!r})
sys.path.insert(0, {tests!r})
import parlayann_b200 as P
from conftest import random_points
from oracle import oracle as O
for dtype, metric in [(np.uint8, P.L2), (np.float32, P.L2), (np.float32, P.MIPS), (np.int8, P.MIPS)]:
    base = random_points(dtype, 2500, 24, 71)
    idx = P.Index(base, 12, metric)
    st = idx.build(24, 1.2, num_passes=2)
    g = idx.get_graph()
    o, tot = O.build_graph("oracle", base, 12, 24, 1.2, 2, metric=metric)
    live = lambda g: [tuple(r[1:1 + r[0]].tolist()) for r in g]
    assert live(g) == live(o), (dtype, metric)
    assert st.dist_cmps == tot, (dtype, metric)
    idx.close()
print("BLOCK_OK")
"""


def test_build_block_prune_kernel_matches_oracle(lib_built):
    """The block-per-job greedy prune kernel (PANN_PRUNE_KERNEL=block, read once per process, so
    run in a child process) gives the oracle's graph and distance-comparison count."""
    import subprocess
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    code = _BLOCK_SCRIPT.format(root=os.path.dirname(here), tests=here)
    env = dict(os.environ, PANN_PRUNE_KERNEL="block")
    r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and "BLOCK_OK" in r.stdout, r.stdout[-2000:] + r.stderr[-2000:]
