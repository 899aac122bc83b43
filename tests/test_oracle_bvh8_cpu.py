"""The oracle's restatement of the device traversal (oracle/ffo_bvh8.c) on a
hand-built 8-wide BVH, on the CPU: one node whose eight leaf slots hold one
triangle each.  Every ray fetches the root once and tests the triangles of
the slots whose quantised boxes it enters; its closest hit equals the
brute-force oracle's (the same restated triangle test, ties to the lowest
index), and its any-hit answer agrees.  (The GPU test
test_trace_gpu.py::test_traversal_pinned_by_oracle_restatement checks the
restatement against the device on device-built BVHs.)"""
import numpy as np

from tests.conftest import cpu_threads


def _one_node_bvh(tris):
    n = len(tris)
    assert 1 <= n <= 8
    lo = tris.reshape(-1, 3).min(0) - np.float32(0.01)
    node = np.zeros(80, np.uint8)
    node[0:12] = np.asarray(lo, np.float32).view(np.uint8)
    node[12:15] = 127 - 7          # 2^-7 per plane step: 255 steps cover more than the 1.02 extent
    node[15] = 0                   # no internal children
    node[16:24] = 0                # first internal child, first triangle: 0
    for s in range(8):
        node[24 + s] = (1 << 5) | s if s < n else 0          # one triangle at offset s
    # planes: lo = 0, hi = 255 on every axis (the whole node box) for used slots
    for a in range(3):
        node[32 + 8 * a: 40 + 8 * a] = 0
        node[56 + 8 * a: 64 + 8 * a] = [255 if s < n else 0 for s in range(8)]
    recs = np.zeros((n, 12), np.float32)
    v0, v1, v2 = tris[:, 0], tris[:, 1], tris[:, 2]
    recs[:, 0:3] = v0
    recs[:, 3] = np.arange(n, dtype=np.int32).view(np.float32)
    recs[:, 4:7] = v1 - v0
    recs[:, 8:11] = v2 - v0
    return node.reshape(1, 80), recs.view(np.uint8).reshape(n, 48)


def test_bvh8_restatement_on_a_hand_built_node(oracle):
    rng = np.random.default_rng(7)
    tris = rng.uniform(0, 1, (8, 3, 3)).astype(np.float32)
    nodes, recs = _one_node_bvh(tris)
    n = 20_000
    rays = np.zeros((n, 8), np.float32)
    rays[:, 0:3] = rng.uniform(-0.5, 1.5, (n, 3))
    d = rng.normal(size=(n, 3))
    rays[:, 4:7] = d / np.linalg.norm(d, axis=1, keepdims=True)
    rays[:, 7] = np.inf
    soup = tris.reshape(-1, 9)
    got, n_nodes, n_tris, errors = oracle.bvh8_trace(nodes, recs, rays, threads=cpu_threads())
    ref = oracle.trace_brute(soup, rays, threads=cpu_threads())
    assert errors == 0
    assert n_nodes == n                      # the root, once per ray
    assert 0 < n_tris <= 8 * n
    bad = got["prim"] != ref["prim"]
    for f in ("t", "u", "v"):
        bad |= (ref["prim"] >= 0) & (got[f].view(np.uint32) != ref[f].view(np.uint32))
    assert int(bad.sum()) == 0
    assert (ref["prim"] >= 0).sum() > 100
    # any hit: the same occluded / clear answers as the brute force
    rays[:, 7] = rng.uniform(0.1, 3.0, n).astype(np.float32)
    ga, _, _, errors = oracle.bvh8_trace(nodes, recs, rays, any_hit=True, threads=cpu_threads())
    ra = oracle.trace_brute(soup, rays, any_hit=True, threads=cpu_threads())
    assert errors == 0
    assert np.array_equal(ga["prim"] >= 0, ra["prim"] >= 0)
