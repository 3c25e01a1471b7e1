"""The C++ drop-in header compiles into a ParlayANN-style program (CPU), and
that program builds, saves, reloads and searches an index on the GPU; its
host-side pieces (point files, distances, graph files and edits) run on the
CPU against restatements of the reference's formats and arithmetic."""
import math
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def compile_demo(out):
    cmd = ["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "cpp", "dropin_demo.cpp"), "-o", out,
           "-L", os.path.join(ROOT, "parlayann_b200"), "-lparlayann_b200",
           "-Wl,-rpath," + os.path.join(ROOT, "parlayann_b200")]
    subprocess.run(cmd, check=True, capture_output=True)


def test_dropin_header_compiles_and_links(tmp_path, lib_built):
    out = str(tmp_path / "dropin_demo")
    compile_demo(out)
    assert os.path.exists(out)


@pytest.mark.gpu
def test_dropin_program_runs_on_gpu(tmp_path, lib_built):
    out = str(tmp_path / "dropin_demo")
    compile_demo(out)
    r = subprocess.run([out, str(tmp_path / "g.bin")], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "beam_search agrees 1" in r.stdout


def _write_bin(path, a):
    with open(path, "wb") as f:
        np.array(a.shape, dtype=np.uint32).tofile(f)
        a.tofile(f)


def _write_graph(path, rows, max_deg):
    """The reference's graph file (graph.h:210-237): n, max degree, the
    degrees, then every row's neighbours."""
    with open(path, "wb") as f:
        np.array([len(rows), max_deg], dtype=np.uint32).tofile(f)
        np.array([len(r) for r in rows], dtype=np.uint32).tofile(f)
        for r in rows:
            np.asarray(r, dtype=np.uint32).tofile(f)


def _read_graph(path):
    a = np.fromfile(path, dtype=np.uint32)
    n, max_deg = int(a[0]), int(a[1])
    deg = a[2:2 + n]
    rows, at = [], 2 + n
    for g in deg:
        rows.append(a[at:at + g].tolist())
        at += g
    assert at == len(a)
    return n, max_deg, rows


def _f32_l2(p, q):
    """euclidian_point.h:83-90: one sequential float sum, every operation rounded."""
    r = np.float32(0)
    for a, b in zip(p, q):
        t = np.float32(b - a)
        r = np.float32(r + np.float32(t * t))
    return r


def _f32_mips(p, q):
    """mips_point.h:60-66: the negated sequential float dot product."""
    r = np.float32(0)
    for a, b in zip(p, q):
        r = np.float32(r + np.float32(b * a))
    return -r


def test_dropin_host_pieces_match_reference_formats(tmp_path, lib_built):
    rng = np.random.default_rng(5)
    bf = rng.standard_normal((12, 24)).astype(np.float32)
    bu = rng.integers(0, 256, size=(12, 32), dtype=np.uint8)
    rows = [sorted(rng.choice(12, size=int(rng.integers(0, 9)), replace=False).tolist()) for _ in range(12)]
    rows[1] = [4, 9, 2, 11]
    paths = [str(tmp_path / x) for x in ("f.bin", "u.bin", "g_in", "g_out")]
    _write_bin(paths[0], bf)
    _write_bin(paths[1], bu)
    _write_graph(paths[2], rows, 8)
    exe = str(tmp_path / "host_check")
    cmd = ["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "cpp", "host_check.cpp"), "-o", exe,
           "-L", os.path.join(ROOT, "parlayann_b200"), "-lparlayann_b200",
           "-Wl,-rpath," + os.path.join(ROOT, "parlayann_b200")]
    subprocess.run(cmd, check=True, capture_output=True)
    r = subprocess.run([exe, *paths], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    lines = r.stdout.splitlines()
    assert lines[0] == "sizes 12 24 12 32"
    seen = 0
    for ln in lines:
        if not ln.startswith("d "):
            continue
        _, i, j, fl2, fip, ul2, uip = ln.split()
        i, j = int(i), int(j)
        assert float.fromhex(fl2) == _f32_l2(bf[i], bf[j])
        assert float.fromhex(fip) == _f32_mips(bf[i], bf[j])
        a, b = bu[i].astype(np.int64), bu[j].astype(np.int64)
        assert float.fromhex(ul2) == float(np.float32(((a - b) ** 2).sum()))
        assert float.fromhex(uip) == -float(np.float32((a * b).sum()))
        seen += 1
    assert seen == 36
    # the same pairs through the oracle's distance (pinned to the reference)
    from oracle import oracle as O
    dist = O.olib().oracle_distance
    for ln in lines:
        if ln.startswith("d "):
            _, i, j, fl2, fip, ul2, uip = ln.split()
            i, j = int(i), int(j)
            for dt, mt, base, got in ((2, 0, bf, fl2), (2, 1, bf, fip), (0, 0, bu, ul2), (0, 1, bu, uip)):
                want = dist(dt, mt, base.shape[1], base[i].ctypes.data, base[j].ctypes.data)
                assert float.fromhex(got) == want
    # one-byte quantization: the oracle's parameters, translate_point restated
    slope = np.zeros(1, np.float32)
    offset = np.zeros(1, np.int32)
    O.olib().oracle_quant_params(12, 24, bf.ctypes.data, slope.ctypes.data, offset.ctypes.data)
    q = [ln for ln in lines if ln.startswith("quant ")][0].split()
    assert np.float32(float.fromhex(q[1])) == slope[0] and int(q[2]) == int(offset[0])
    for ln in lines:
        if ln.startswith("qrow "):
            parts = ln.split()
            i = int(parts[1])
            want = []
            for x in bf[i]:
                v = float(np.float32(x) * slope[0])
                r = int(math.copysign(math.floor(abs(v) + 0.5), v)) - int(offset[0])  # roundf: half away from 0
                want.append(min(255, max(0, r)))
            assert [int(t) for t in parts[2:]] == want
    assert f"graph 12 8 {len(rows[4])}" in lines
    n, max_deg, out = _read_graph(paths[3])
    assert (n, max_deg) == (12, 8)
    want = [list(x) for x in rows]
    want[0] = [7, 3, 5]
    want[1] = sorted(rows[1], reverse=True)
    want[2] = [1, 2]
    assert out == want
