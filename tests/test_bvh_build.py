"""The host BVH builder (lightpropagation_b200/csrc/lp_bvh.cpp), checked on the CPU.

The builder runs large meshes (32,768 triangles and more) on worker threads.  These
tests compile it with a small harness (tests/bvh_dump.cpp) and check, for meshes on
both sides of that size and for a mesh of coincident triangles:
  * the leaves hold every triangle exactly once, and each triangle record is the
    reference's (M, E = K - M, F = L - M) of FindTriangleInPath (.cl:1037-1093);
  * every child box contains all vertices of the triangles below it;
  * the depth fits the device traversal stack (64);
  * two builds of the same mesh give the same bytes;
  * the tree does not depend on the number of worker threads (1, 2, 8, 16 threads give
    the same bytes, whatever the test machine's own core count).
"""
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from lightpropagation_b200 import meshes  # noqa: E402

STACK_DEPTH = 64


@pytest.fixture(scope="module")
def dump_exe(tmp_path_factory):
    out = tmp_path_factory.mktemp("bvh") / "bvh_dump"
    csrc = os.path.join(ROOT, "lightpropagation_b200", "csrc")
    subprocess.check_call(["g++", "-O2", "-std=c++17", "-pthread", "-I", csrc,
                           os.path.join(ROOT, "tests", "bvh_dump.cpp"), os.path.join(csrc, "lp_bvh.cpp"),
                           "-o", str(out)])
    return str(out)


def build(exe, tri, tmp_path, tag, threads=0):
    src, dst = tmp_path / f"{tag}.f32", tmp_path / f"{tag}.bin"
    np.ascontiguousarray(tri, np.float32).tofile(src)
    subprocess.check_call([exe, str(src), str(dst)] + ([str(threads)] if threads else []))
    raw = dst.read_bytes()
    nn, nt, depth = np.frombuffer(raw[:12], np.int32)
    margin = np.frombuffer(raw[12:16], np.float32)[0]
    off = 16
    arrs = []
    for dt, cnt in ((np.float32, nn), (np.float32, nn), (np.float32, nn), (np.int32, nn),
                    (np.float32, nt), (np.float32, nt), (np.float32, nt)):
        arrs.append(np.frombuffer(raw[off:off + 16 * cnt], dt).reshape(cnt, 4))
        off += 16 * cnt
    return raw, int(depth), float(margin), arrs


def check_tree(tri, depth, margin, arrs):
    na, nb, nc, nd, ta, tb, tc = arrs
    n = tri.shape[0]
    t = tri.reshape(n, 3, 3)
    ids = tc[:, 1].view(np.int32)
    assert np.array_equal(np.sort(ids), np.arange(n)), "leaves do not hold every triangle once"
    K, L, M = t[ids, 0], t[ids, 1], t[ids, 2]
    assert np.array_equal(ta[:, :3], M)
    assert np.array_equal(np.stack([ta[:, 3], tb[:, 0], tb[:, 1]], 1), (K - M).astype(np.float32))
    assert np.array_equal(np.stack([tb[:, 2], tb[:, 3], tc[:, 0]], 1), (L - M).astype(np.float32))
    assert depth < STACK_DEPTH
    # vertex bounds of each leaf-order triangle
    vlo, vhi = t[ids].min(1), t[ids].max(1)
    nodes = na.shape[0]
    lo = np.zeros((nodes, 3), np.float32)
    hi = np.zeros((nodes, 3), np.float32)
    # breadth-first order: children have larger indices, so walk the nodes backwards
    for i in range(nodes - 1, -1, -1):
        boxes = [(np.array([na[i, 0], na[i, 2], nc[i, 0]]), np.array([na[i, 1], na[i, 3], nc[i, 1]])),
                 (np.array([nb[i, 0], nb[i, 2], nc[i, 2]]), np.array([nb[i, 1], nb[i, 3], nc[i, 3]]))]
        los, his = [], []
        for c in range(2):
            ref = int(nd[i, c])
            if ref < 0:
                e = ~ref
                first, cnt = e >> 3, (e & 7) + 1
                assert first + cnt <= n
                clo, chi = vlo[first:first + cnt].min(0), vhi[first:first + cnt].max(0)
            else:
                assert ref > i, "child precedes its parent in breadth-first order"
                clo, chi = lo[ref], hi[ref]
            blo, bhi = boxes[c]
            assert np.all(blo <= clo) and np.all(chi <= bhi), f"node {i} child {c} box misses its triangles"
            los.append(clo)
            his.append(chi)
        lo[i], hi[i] = np.minimum(*los), np.maximum(*his)


@pytest.mark.parametrize("case", ["soup_3000", "abdomen_52900", "coincident_40000"])
def test_bvh_tree_is_valid_and_deterministic(dump_exe, tmp_path, case):
    rng = np.random.default_rng(7)
    if case == "soup_3000":
        c = rng.uniform(-20, 20, (3000, 1, 3))
        tri = (c + rng.normal(scale=1.5, size=(3000, 3, 3))).reshape(-1, 9)
    elif case == "abdomen_52900":
        tri, _, _ = meshes.curved_abdomen(freq=23)     # above the size built on worker threads
    else:
        one = np.array([0, 0, 0, 1, 0, 0, 0, 1, 0], np.float32)
        tri = np.tile(one, (40000, 1))                    # every centroid equal: splits by position
    tri = np.asarray(tri, np.float32).reshape(-1, 9)
    raw1, depth, margin, arrs = build(dump_exe, tri, tmp_path, "a")
    raw2, _, _, _ = build(dump_exe, tri, tmp_path, "b")
    assert raw1 == raw2, "two builds of the same mesh differ"
    check_tree(tri, depth, margin, arrs)


@pytest.mark.parametrize("case", ["abdomen_52900", "coincident_40000"])
def test_bvh_tree_does_not_depend_on_the_thread_count(dump_exe, tmp_path, case):
    """One worker thread runs the serial build (build_from); 2, 8 and 16 run the parallel
    recursion (build_par) and the threaded binning of large nodes.  All give the same tree."""
    if case == "abdomen_52900":
        tri, _, _ = meshes.curved_abdomen(freq=23)
    else:
        one = np.array([0, 0, 0, 1, 0, 0, 0, 1, 0], np.float32)
        tri = np.tile(one, (40000, 1))
    tri = np.asarray(tri, np.float32).reshape(-1, 9)
    ref, _, _, _ = build(dump_exe, tri, tmp_path, "t1", threads=1)
    for k in (2, 8, 16):
        raw, _, _, _ = build(dump_exe, tri, tmp_path, f"t{k}", threads=k)
        assert raw == ref, f"the tree built on {k} threads differs from the one-thread tree"
