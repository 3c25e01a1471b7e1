"""pann_search_device_noalloc against pann_search_device, both through the C ABI.

pann_search_device_noalloc serves callers that cannot allocate device memory
while they run (cudaFree stalls the whole device, a framework allocator may
hold all of it, a latency-bound path cannot take a first-call allocation): it
searches with one fixed static device array as its only working memory. Its
results must be those of pann_search_device: same ids, distances (FLOAT_RTOL is
the required float bar; the assertions are bitwise), visited and comparison
counts and status bits, on consecutive calls that share the array. The file is
named to be collected last; it must pass after the other GPU tests and alone.
"""
import ctypes

import numpy as np
import pytest

import parlayann_b200 as P
from conftest import random_points
from oracle import oracle as O

pytestmark = pytest.mark.gpu
FLOAT_RTOL = 1e-5


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _run(fn, idx, dq, nq, k, qp, starts, stream):
    import torch

    dev = dq.device
    out = {  # filled with junk so that anything left unwritten shows
        "ids": torch.full((nq, k), 7, dtype=torch.int32, device=dev),
        "dists": torch.full((nq, k), -1.0, dtype=torch.float32, device=dev),
        "vis": torch.full((nq,), 9, dtype=torch.int32, device=dev),
        "cmps": torch.full((nq,), 9, dtype=torch.int32, device=dev),
        "flags": torch.full((nq,), 9, dtype=torch.int32, device=dev),
    }
    st = np.asarray(starts, np.uint32)
    rc = fn(idx.handle, _ptr(dq), nq, ctypes.byref(qp), st.ctypes.data_as(ctypes.c_void_p), len(st),
            _ptr(out["ids"]), _ptr(out["dists"]), _ptr(out["vis"]), _ptr(out["cmps"]), _ptr(out["flags"]),
            ctypes.c_void_p(stream.cuda_stream))
    if rc != 0:
        raise P.PannError(rc, P.lib().pann_last_error().decode())
    return out


def _same(a, b, msg):
    import torch

    torch.cuda.synchronize()
    for key in ("ids", "vis", "cmps", "flags"):
        np.testing.assert_array_equal(a[key].cpu().numpy(), b[key].cpu().numpy(), err_msg=f"{key} {msg}")
    da, db = a["dists"].cpu().numpy(), b["dists"].cpu().numpy()
    np.testing.assert_allclose(da, db, rtol=FLOAT_RTOL, err_msg=f"dists {msg}")
    np.testing.assert_array_equal(da.view(np.uint32), db.view(np.uint32), err_msg=f"dist bits {msg}")


def test_noalloc_matches_search_device_on_consecutive_calls(lib_built):
    import torch

    lib = P.lib()
    dev = torch.device("cuda:0")
    stream = torch.cuda.current_stream(dev)

    # call 1: a graph on which the reference's hashset grows for some queries
    base = random_points(np.uint8, 20000, 8, 1)
    g = O.random_graph(20000, 64, 3, min_deg=60)
    idx = P.Index(base, 64)
    idx.set_graph(g)
    q = random_points(np.uint8, 256, 8, 2)
    dq = torch.from_numpy(q).to(dev)
    qp = P.QueryParams(10, 40, 20000, 64, 1.0)
    ref = _run(lib.pann_search_device, idx, dq, len(q), 10, qp, (0,), stream)
    got = _run(lib.pann_search_device_noalloc, idx, dq, len(q), 10, qp, (0,), stream)
    _same(ref, got, "call 1")
    assert int(((ref["flags"] & 2) != 0).sum().item()) > 0, "no query reached the hashset-growth path"

    # call 2, straight after on the same array: other queries, beam and start points
    q2 = random_points(np.uint8, 1000, 8, 4)
    dq2 = torch.from_numpy(q2).to(dev)
    qp2 = P.QueryParams(5, 24, 20000, 64, 0.125)
    ref2 = _run(lib.pann_search_device, idx, dq2, len(q2), 5, qp2, (0, 5, 9), stream)
    got2 = _run(lib.pann_search_device_noalloc, idx, dq2, len(q2), 5, qp2, (0, 5, 9), stream)
    _same(ref2, got2, "call 2")
    # call 1 again, with call 2's leftovers in the array
    got3 = _run(lib.pann_search_device_noalloc, idx, dq, len(q), 10, qp, (0,), stream)
    _same(ref, got3, "call 1 repeated")
    idx.close()


def test_noalloc_padded_rows_and_float_metrics(lib_built):
    import torch

    lib = P.lib()
    dev = torch.device("cuda:0")
    stream = torch.cuda.current_stream(dev)
    base = random_points(np.float32, 3000, 7, 31)   # 28-byte rows: queries staged with padding
    g = O.random_graph(3000, 12, 32)
    for metric in (P.L2, P.MIPS):
        idx = P.Index(base, 12, metric)
        idx.set_graph(g)
        q = random_points(np.float32, 300, 7, 33)
        dq = torch.from_numpy(q).to(dev)
        qp = P.QueryParams(8, 32, 3000, 12, 0.125)
        for _ in range(2):
            ref = _run(lib.pann_search_device, idx, dq, len(q), 8, qp, (0, 1), stream)
            got = _run(lib.pann_search_device_noalloc, idx, dq, len(q), 8, qp, (0, 1), stream)
            _same(ref, got, f"metric {metric}")
        idx.close()


def test_noalloc_rejects_calls_beyond_the_array(lib_built):
    import torch

    lib = P.lib()
    dev = torch.device("cuda:0")
    stream = torch.cuda.current_stream(dev)
    base = random_points(np.uint8, 2000, 16, 41)
    g = O.random_graph(2000, 16, 42)
    idx = P.Index(base, 16)
    idx.set_graph(g)
    nq = P.PANN_NOALLOC_SCRATCH_BYTES // 28 + 1   # more per-query state than the array holds
    dq = torch.zeros((nq, 16), dtype=torch.uint8, device=dev)
    qp = P.QueryParams(4, 8, 2000, 16, 0.125)
    with pytest.raises(P.PannError) as e:
        _run(lib.pann_search_device_noalloc, idx, dq, nq, 4, qp, (0,), stream)
    assert e.value.code == P.PANN_EINVAL
    assert "static scratch" in str(e.value)
    # a beam and degree limit whose seen tables cannot fit are refused the same way
    qp_big = P.QueryParams(4, 4000, 2000, 1024, 0.125)
    with pytest.raises(P.PannError) as e:
        _run(lib.pann_search_device_noalloc, idx, dq[:4], 4, 4, qp_big, (0,), stream)
    assert e.value.code == P.PANN_EINVAL
    # the array is still good afterwards
    q = random_points(np.uint8, 64, 16, 43)
    dq = torch.from_numpy(q).to(dev)
    ref = _run(lib.pann_search_device, idx, dq, 64, 4, qp, (0,), stream)
    got = _run(lib.pann_search_device_noalloc, idx, dq, 64, 4, qp, (0,), stream)
    _same(ref, got, "after a refused call")
    idx.close()
