"""Parity against the REFERENCE's own CUDA kernels (oracle/_ref/libhipref.so,
built from the reference's sources) on the same inputs (sm_100a).

Bit-exact: Morton keys, sorted keys and reference order, Karras topology,
refitted pre-collapse boxes. After the collapse, whose numbering the reference
takes from atomics, both trees are compared in a canonical depth-first form
(structure, child boxes bit for bit, each leaf's set of triangles). The SAH
cost agrees to 0.1 %. With the reference's arithmetic selected
(hp_ctx_set_arithmetic: its fast-math reciprocals), Woop rows are bit-identical
and every hit record equals the reference tracer's except on rays with two
hits at exactly the same t, where this library reports the lower triangle id;
those are counted. With the default IEEE reciprocals, hits agree by triangle
id on all but a few rays near triangle edges, and t to 1e-6 relative.
"""
import numpy as np
import pytest
import torch

import hippie_b200 as hp
import oracle
from oracle import ref_harness as R

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not R.available(), reason="reference harness not built (needs the reference sources)")]


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def canonical(nodes, tri_idx):
    """Depth-first (left first) serialisation: child boxes (bits), sizes, leaf triangle sets."""
    out = []
    stack = [0]
    while stack:
        i = stack.pop()
        c0, c1, size, _ = nodes[i, 12:16]
        if size < 0:
            out.append(("L", tuple(nodes[i, :12].tolist()), tuple(sorted(tri_idx[c0:c1].tolist()))))
        else:
            out.append(("I", tuple(nodes[i, :12].tolist()), int(size)))
            stack.append(~c1 if c1 < 0 else c1)
            stack.append(~c0 if c0 < 0 else c0)
    return out


def _mine(ctx, V, T, n, bits, method="lbvh"):
    nn = 2 * n - 1
    taps = dict(morton_keys=torch.zeros(n, dtype=torch.int64, device="cuda"),
                sorted_keys=torch.zeros(n, dtype=torch.int64, device="cuda"),
                sorted_refs=torch.zeros(n, dtype=torch.int32, device="cuda"))
    if method == "lbvh":
        taps.update(node_parent=torch.zeros(nn, dtype=torch.int32, device="cuda"),
                    node_left=torch.zeros(nn, dtype=torch.int32, device="cuda"),
                    node_right=torch.zeros(nn, dtype=torch.int32, device="cuda"),
                    node_box_min=torch.zeros((nn, 4), dtype=torch.float32, device="cuda"),
                    node_box_max=torch.zeros((nn, 4), dtype=torch.float32, device="cuda"))
    p = hp.BuildParams(method=method, morton_bits=bits, ploc_radius=16, ploc_max_radius=256)
    bvh = ctx.build(V, T, p, taps=taps)
    bvh.sync()
    ctx.check()
    return bvh, {k: x.cpu().numpy() for k, x in taps.items()}


@pytest.mark.parametrize("kind,n,bits", [("uniform", 65536, 30), ("clustered", 262144, 60)])
def test_lbvh_matches_reference_kernels(ctx, kind, n, bits):
    if kind == "uniform":
        v, t = hp.gen.uniform_mesh(0xC0FFEE + 1, n)
    else:
        v, t = hp.gen.clustered_mesh(0xC0FFEE + 2, n, clusters=1024)
    V, T = dev(v), dev(t)
    bvh, mine = _mine(ctx, V, T, n, bits)
    box = np.array(bvh.c.scene_box, np.float32)
    ref = R.build(V, T, box, method="lbvh", bits=bits, taps=True)
    np.testing.assert_array_equal(mine["morton_keys"], ref["keys"])
    np.testing.assert_array_equal(mine["sorted_keys"], ref["sorted"])
    np.testing.assert_array_equal(mine["sorted_refs"], ref["refs"])
    np.testing.assert_array_equal(mine["node_parent"], ref["parent"])
    np.testing.assert_array_equal(mine["node_left"], ref["left"])
    np.testing.assert_array_equal(mine["node_right"], ref["right"])
    np.testing.assert_array_equal(mine["node_box_min"][:, :3], ref["bmin"][:, :3])
    np.testing.assert_array_equal(mine["node_box_max"][:, :3], ref["bmax"][:, :3])
    nodes, woop, tri = bvh.download()
    assert (bvh.c.num_interior, bvh.c.num_leaf) == tuple(ref["counts"].tolist())
    assert canonical(nodes, tri) == canonical(ref["nodes"], ref["tri_idx"])
    # Woop rows per triangle: the reference inverts with a fast-math reciprocal
    mw = np.zeros_like(woop)
    rw = np.zeros_like(woop)
    mw[tri] = woop
    rw[ref["tri_idx"]] = ref["woop"]
    rel = np.abs(mw - rw) / np.maximum(np.abs(rw), 1e-3 * np.abs(rw).max(axis=1, keepdims=True))
    assert np.quantile(rel, 0.999) < 1e-5
    area = 2 * np.float32((box[3] - box[0]) * (box[4] - box[1]) + (box[4] - box[1]) * (box[5] - box[2]) +
                          (box[5] - box[2]) * (box[3] - box[0]))
    rc = R.cost(torch.from_numpy(ref["nodes"]).cuda(), ref["nodes"].shape[0], float(area))
    assert bvh.cost() == pytest.approx(rc, rel=1e-3)
    assert bvh.cost() == pytest.approx(oracle.cost(nodes, box), rel=1e-12)


def test_ploc_matches_reference_kernels(ctx):
    n = 262144
    v, t = hp.gen.clustered_mesh(0xC0FFEE + 3, n, clusters=1024)
    V, T = dev(v), dev(t)
    bvh, mine = _mine(ctx, V, T, n, 60, method="ploc")
    box = np.array(bvh.c.scene_box, np.float32)
    ref = R.build(V, T, box, method="ploc", bits=60, radius=16, max_radius=256, taps=True)
    np.testing.assert_array_equal(mine["morton_keys"], ref["keys"])
    np.testing.assert_array_equal(mine["sorted_refs"], ref["refs"])
    nodes, woop, tri = bvh.download()
    assert (bvh.c.num_interior, bvh.c.num_leaf) == tuple(ref["counts"].tolist())
    assert canonical(nodes, tri) == canonical(ref["nodes"], ref["tri_idx"])
    area = 2 * np.float32((box[3] - box[0]) * (box[4] - box[1]) + (box[4] - box[1]) * (box[5] - box[2]) +
                          (box[5] - box[2]) * (box[3] - box[0]))
    rc = R.cost(torch.from_numpy(ref["nodes"]).cuda(), ref["nodes"].shape[0], float(area))
    assert bvh.cost() == pytest.approx(rc, rel=1e-3)


def compare_hits(mine, ref):
    """Split rays into equal hit records, exact-t ties and other differences.

    A tie: both hit at the same t (bit for bit) on different triangles, and
    this library reports the lower triangle id (the reference keeps the first
    one its traversal meets). Returns (equal, ties, indices of the others)."""
    same = np.all(mine == ref, axis=1)
    both = (mine[:, 0] >= 0) & (ref[:, 0] >= 0)
    tie = ~same & both & (mine[:, 1] == ref[:, 1]) & (mine[:, 0] < ref[:, 0])
    return int(same.sum()), int(tie.sum()), np.nonzero(~same & ~tie)[0]


def test_trace_matches_reference_tracer_ieee(ctx):
    """Default (IEEE reciprocal) arithmetic against the reference tracer on the
    same nodes and Woop rows: the reciprocals differ in the last bit, so a few
    rays near a triangle edge may change triangle; t agrees to 1e-6."""
    n = 65536
    v, t = hp.gen.uniform_mesh(0xC0FFEE + 1, n)
    rays = hp.gen.rays_targeted(0xC0FFEE + 11, 1 << 20)
    V, T, Rr = dev(v), dev(t), dev(rays)
    bvh = ctx.build(V, T, hp.BuildParams(morton_bits=30))
    mine = ctx.trace(bvh, Rr, results=torch.zeros((rays.shape[0], 4), dtype=torch.int32, device="cuda")).cpu().numpy()
    nodes, woop, tri = bvh.download()
    # the reference tracer reads this library's 64-byte nodes and Woop layout directly
    ref, _ = R.trace(torch.from_numpy(nodes).cuda(), torch.from_numpy(woop).cuda(), torch.from_numpy(tri).cuda(), Rr)
    hit_m, hit_r = mine[:, 0] >= 0, ref[:, 0] >= 0
    assert np.mean(hit_m == hit_r) > 0.9999
    both = hit_m & hit_r
    same = mine[both, 0] == ref[both, 0]
    assert np.mean(same) > 0.9999
    tm = mine[both][same, 1:].view(np.float32).astype(np.float64)
    tr = ref[both][same, 1:].view(np.float32).astype(np.float64)
    err = np.abs(tm - tr) / np.maximum(1.0, np.abs(tr))
    assert np.quantile(err[:, 0], 0.999) <= 1e-6
    assert np.quantile(err[:, 1:], 0.99) <= 1e-4


def _ref_ctx():
    c = hp.Context(0)
    c.set_arithmetic("reference")
    return c


def _check_reference_hits(rctx, V, T, rays, params, method, **build_kw):
    """Build and trace in reference arithmetic; compare (1) Woop rows per
    triangle with the reference's woopify, (2) hits with the reference tracer
    on this library's BVH, (3) hits with the reference's own build + tracer.
    Every differing ray must be an exact-t tie won by the lower id."""
    Rr = dev(rays)
    bvh = rctx.build(V, T, params)
    mine = rctx.trace(bvh, Rr, results=torch.zeros((rays.shape[0], 4), dtype=torch.int32, device="cuda"))
    mine = mine.cpu().numpy()
    rctx.check()
    nodes, woop, tri = bvh.download()
    box = np.array(bvh.c.scene_box, np.float32)
    ref = R.build(V, T, box, method=method, **build_kw)
    mw = np.zeros_like(woop)
    rw = np.zeros_like(woop)
    mw[tri] = woop
    rw[ref["tri_idx"]] = ref["woop"]
    np.testing.assert_array_equal(mw.view(np.int32), rw.view(np.int32))
    on_mine, _ = R.trace(torch.from_numpy(nodes).cuda(), torch.from_numpy(woop).cuda(), torch.from_numpy(tri).cuda(),
                         Rr)
    own, _ = R.trace(torch.from_numpy(ref["nodes"]).cuda(), torch.from_numpy(ref["woop"]).cuda(),
                     torch.from_numpy(ref["tri_idx"]).cuda(), Rr)
    out = {}
    for name, r in (("same_bvh", on_mine), ("reference_build", own)):
        eq, ties, other = compare_hits(mine, r)
        assert other.size == 0, (name, other[:10], mine[other[:10]], r[other[:10]])
        out[name] = (eq, ties)
    print(f"reference-arithmetic hits: {rays.shape[0]} rays; equal / exact-t ties: {out}")
    return out


def test_trace_reference_arithmetic_bit_identical_uniform64k():
    """65,536 uniform triangles (30-bit LBVH), 1,048,576 targeted rays."""
    v, t = hp.gen.uniform_mesh(0xC0FFEE, 65536, 0.01)
    rays = hp.gen.rays_targeted(0xC0FFEE + 1, 1 << 20, -0.5, 1.5)
    rctx = _ref_ctx()
    try:
        out = _check_reference_hits(rctx, dev(v), dev(t), rays, hp.BuildParams(morton_bits=30), "lbvh", bits=30)
        assert out["same_bvh"][0] + out["same_bvh"][1] == rays.shape[0]
    finally:
        rctx.close()


def test_trace_reference_arithmetic_bit_identical_ploc4m():
    """4,194,304 clustered triangles (PLOC radius 16, 60-bit), all 16,777,216
    sphere rays: the bench workload."""
    seed = 0xC0FFEE + 1
    v, t = hp.gen.clustered_mesh(seed, 4194304, 1024, 0.02, 0.005)
    box = np.concatenate([v.min(0), v.max(0)]).astype(np.float32)
    rays = hp.gen.rays_sphere(seed + 1, 16777216, box)
    rctx = _ref_ctx()
    try:
        p = hp.BuildParams(method="ploc", morton_bits=60, ploc_radius=16, ploc_max_radius=256, ploc_adaptive=0)
        _check_reference_hits(rctx, dev(v), dev(t), rays, p, "ploc", bits=60, radius=16, max_radius=256)
    finally:
        rctx.close()


def test_reference_arithmetic_refit_woop():
    """hp_refit in reference arithmetic rewrites the Woop rows as the reference's
    woopify of the moved vertices (compared through a fresh reference build)."""
    v, t = hp.gen.heightfield(3, 64, 128)
    rctx = _ref_ctx()
    try:
        V, T = dev(v), dev(t)
        bvh = rctx.build(V, T, hp.BuildParams(morton_bits=60))
        v2 = v.copy()
        v2[:, 2] += np.random.default_rng(1).uniform(-0.01, 0.01, v.shape[0]).astype(np.float32)
        V2 = dev(v2)
        rctx.refit(bvh, V2, T)
        rctx.check()
        _, woop, tri = bvh.download()
        ref = R.build(V2, T, np.concatenate([v2.min(0), v2.max(0)]).astype(np.float32), method="lbvh", bits=60)
        mw = np.zeros_like(woop)
        rw = np.zeros_like(woop)
        mw[tri] = woop
        rw[ref["tri_idx"]] = ref["woop"]
        np.testing.assert_array_equal(mw.view(np.int32), rw.view(np.int32))
    finally:
        rctx.close()
