"""CPU checks of the C ABI library: it loads, exports every symbol the public
header declares, validates arguments without a GPU, and its host-side logic
(batch schedule, insertion order, synthetic data) matches the oracle."""
import os
import re

import numpy as np
import pytest

import parlayann_b200 as P
from conftest import has_gpu
from oracle import oracle as O

HEADER = os.path.join(os.path.dirname(os.path.dirname(__file__)), "include", "parlayann_b200.h")


def header_symbols():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(pann_\w+)\s*\(", txt, re.M)))


def test_header_declares_expected_symbols():
    syms = header_symbols()
    assert "pann_search" in syms and "pann_build" in syms and "pann_last_error" in syms
    assert set(syms) == set(P.SIGNATURES), set(syms) ^ set(P.SIGNATURES)


def test_library_exports_every_header_symbol(lib_built):
    L = P.lib()
    for s in header_symbols():
        assert hasattr(L, s), s


@pytest.mark.skipif(has_gpu(), reason="checks the no-device error path")
def test_index_create_without_device_fails_cleanly(lib_built):
    with pytest.raises(P.PannError) as e:
        P.Index(np.zeros((10, 4), np.uint8), 4)
    assert e.value.code in (P.PANN_EDEVICE, P.PANN_ENOMEM)
    assert "CUDA" in str(e.value) or "device" in str(e.value)


def test_argument_validation_before_device(lib_built):
    import ctypes

    h = ctypes.c_void_p()
    assert P.lib().pann_index_create(ctypes.byref(h), 7, 0, 10, 4, 4) == P.PANN_EINVAL
    assert b"dtype" in P.lib().pann_last_error()
    assert P.lib().pann_index_create(ctypes.byref(h), 0, 0, 0, 4, 4) == P.PANN_EINVAL
    assert P.lib().pann_index_create(ctypes.byref(h), 0, 0, 10, 0, 4) == P.PANN_EINVAL
    assert P.lib().pann_index_create(ctypes.byref(h), 0, 0, 10, 4, 0) == P.PANN_EINVAL
    assert P.lib().pann_search(None, None, 0, None, None, 0, None, None, None, None, None) == P.PANN_EINVAL


@pytest.mark.parametrize("n", [1, 2, 3, 100, 1000, 100000, 1000000, 10000000, 100000000])
def test_batch_schedule_matches_oracle(n, lib_built):
    assert P.batch_schedule(n) == O.batch_schedule(n)


def test_batch_schedule_shape():
    s = P.batch_schedule(100000)
    assert s[0] == (0, 1) and s[1] == (1, 3) and s[10] == (1023, 2047)
    assert s[11] == (2047, 4047)          # then fixed batches of 0.02 n
    assert s[-1][1] == 100000
    assert all(a[1] == b[0] for a, b in zip(s, s[1:]))


def test_permutation_matches_oracle(lib_built):
    for n in (1, 2, 10, 12345):
        np.testing.assert_array_equal(P.permutation(n), O.permutation(n))
    p = P.permutation(5000)
    assert sorted(p.tolist()) == list(range(5000))


def test_synth_is_deterministic_and_shaped(lib_built):
    a = P.synth_mixture(P.U8, 2000, 128, 64, 0, 0)
    b = P.synth_mixture(P.U8, 2000, 128, 64, 0, 0)
    np.testing.assert_array_equal(a, b)
    q = P.synth_mixture(P.U8, 100, 128, 64, 0, 1)
    assert not np.array_equal(a[:100], q)
    assert a.dtype == np.uint8 and a.min() >= 0 and a.max() <= 255
    assert 100 < a.mean() < 156                      # centres uniform in [32, 224]
    f = P.synth_mixture(P.F32, 1000, 96, 256, 1, 0, sigma=0.3, normalize=True)
    np.testing.assert_allclose(np.linalg.norm(f, axis=1), 1.0, rtol=1e-5)
    # a row does not depend on how many rows are generated
    np.testing.assert_array_equal(P.synth_mixture(P.F32, 10, 96, 256, 1, 0, sigma=0.3, normalize=True), f[:10])
