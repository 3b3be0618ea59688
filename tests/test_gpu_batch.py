"""Batched build + trace of many meshes (hp_batch_*) against the single-mesh
path: every mesh's BVH (nodes, triangle order, Woop rows) and every ray's hit
are bit-identical; CUDA-graph replay, direct launches, empty and tiny meshes."""
import numpy as np
import pytest
import torch

import hippie_b200 as hp

pytestmark = pytest.mark.gpu


def _mesh(seed, n):
    if n == 0:
        return np.zeros((0, 3), np.float32), np.zeros((0, 3), np.int32)
    return hp.gen.uniform_mesh(seed, n)


def _setup(sizes, seed=0, rays_per_tri=4):
    meshes, rays, counts = [], [], []
    for i, n in enumerate(sizes):
        v, t = _mesh(seed + i, n)
        meshes.append((torch.from_numpy(v).cuda(), torch.from_numpy(t).cuda()))
        k = rays_per_tri * n if n else 7
        box = np.concatenate([v.min(0), v.max(0)]) if n else np.array([0, 0, 0, 1, 1, 1], np.float32)
        rays.append(hp.gen.rays_sphere(1000 + seed + i, k, box))
        counts.append(k)
    return meshes, np.concatenate(rays), counts


@pytest.fixture(scope="module")
def case():
    rng = np.random.default_rng(5)
    sizes = [0, 1, 2, 3, 17, 256, 1000, 4096, 33333, 100000, 0, 1]
    sizes += [int(round(np.exp(x))) for x in rng.uniform(np.log(256), np.log(65536), 40)]
    return sizes, _setup(sizes)


@pytest.mark.parametrize("graph", [True, False])
def test_batch_equals_plain(ctx, case, graph):
    sizes, (meshes, rays, counts) = case
    p = hp.BuildParams(method="lbvh", morton_bits=30)
    batch = hp.Batch(ctx, meshes, counts, p)
    R = torch.from_numpy(rays).cuda()
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        res = batch.build_trace(R, results=torch.zeros((batch.num_rays, 4), dtype=torch.int32, device="cuda"),
                                graph=graph)
        if graph:  # a replay gives the same answer
            res2 = batch.build_trace(R, results=torch.zeros_like(res), graph=graph)
    s.synchronize()
    ctx.check()
    got = res.cpu().numpy()
    if graph:
        np.testing.assert_array_equal(res2.cpu().numpy(), got)
    for m, (V, T) in enumerate(meshes):
        o0, o1 = batch.ray_offset(m), batch.ray_offset(m + 1)
        assert o1 - o0 == counts[m]
        Rm = R[o0:o1].contiguous()
        n = sizes[m]
        if n == 0:
            assert np.all(got[o0:o1, 0] == -1)
            np.testing.assert_array_equal(got[o0:o1, 1], rays[o0:o1, 7].view(np.int32))
            continue
        plain = ctx.build(V, T, p)
        pn, pw, pt = plain.download()
        view = batch.bvh(m)
        bn, bw, bt = view.download()
        assert (view.c.num_interior, view.c.num_leaf) == (plain.c.num_interior, plain.c.num_leaf)
        assert list(view.c.scene_box) == list(plain.c.scene_box)
        np.testing.assert_array_equal(bn, pn)
        np.testing.assert_array_equal(bt, pt)
        np.testing.assert_array_equal(bw, pw)
        exp = ctx.trace(plain, Rm, results=torch.zeros((Rm.shape[0], 4), dtype=torch.int32, device="cuda"))
        exp = exp.cpu().numpy()
        np.testing.assert_array_equal(got[o0:o1], exp)
    batch.close()


def test_batch_flags_and_rebuild(ctx):
    sizes = [500, 3000, 12000]
    meshes, rays, counts = _setup(sizes, seed=40)
    p = hp.BuildParams(method="lbvh", morton_bits=30)
    batch = hp.Batch(ctx, meshes, counts, p)
    R = torch.from_numpy(rays).cuda()
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        batch.build(graph=True)
        st = torch.zeros((batch.num_rays, 2), dtype=torch.int32, device="cuda")
        closest = batch.trace(R, stats=st, graph=True)
        anyh = batch.trace(R, any_hit=True, graph=True)
        zeros = torch.zeros((batch.num_rays, 4), dtype=torch.int32, device="cuda")
    s.synchronize()
    ctx.check()
    c, a = closest.cpu().numpy(), anyh.cpu().numpy()
    np.testing.assert_array_equal(a[:, 0] >= 0, c[:, 0] >= 0)
    stn = st.cpu().numpy()
    assert np.all(stn[c[:, 0] >= 0] > 0)
    # move one mesh's vertices: a rebuild from the same graph follows the new geometry
    V0, T0 = meshes[1]
    V0 += 0.25
    with torch.cuda.stream(s):
        res = batch.build_trace(R, results=zeros, graph=True)
    s.synchronize()
    plain = ctx.build(V0, T0, p)
    o0, o1 = batch.ray_offset(1), batch.ray_offset(2)
    exp = ctx.trace(plain, R[o0:o1].contiguous(), results=torch.zeros((o1 - o0, 4), dtype=torch.int32, device="cuda"))
    np.testing.assert_array_equal(res.cpu().numpy()[o0:o1], exp.cpu().numpy())
    nodes, _, _ = batch.bvh(1).download()
    np.testing.assert_array_equal(nodes, plain.download()[0])


def test_batch_graph_needs_stream(ctx):
    meshes, rays, counts = _setup([300], seed=60)
    batch = hp.Batch(ctx, meshes, counts)
    with pytest.raises(ValueError):
        batch.build(graph=True, stream=0)
    batch.build(graph=False, stream=0)
    torch.cuda.synchronize()
    ctx.check()


def test_batch_rejects_bad_input(ctx):
    meshes, rays, counts = _setup([300], seed=61)
    with pytest.raises(hp.HPError):
        hp.Batch(ctx, meshes, counts, hp.BuildParams(method="ploc", morton_bits=60))
    with pytest.raises(hp.HPError):
        hp.Batch(ctx, meshes * 20, counts * 20, hp.BuildParams(method="lbvh", morton_bits=60))


def test_batch_wide_keys_equal_plain(ctx):
    """60-bit Morton codes with the mesh index above them (62-bit keys) over
    more than 2^20 triangles: the batch sorts them with the wide-key sort (three
    passes over the top 24 bits, whose digit counts its Morton kernel takes,
    then the segment sort); every mesh's BVH and hits equal the plain path's."""
    sizes = [300000, 500000, 250000, 100000]
    meshes, rays, counts = _setup(sizes, seed=77, rays_per_tri=2)
    assert sum(sizes) >= 1 << 20
    p = hp.BuildParams(method="lbvh", morton_bits=60)
    batch = hp.Batch(ctx, meshes, counts, p)
    R = torch.from_numpy(rays).cuda()
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        res = batch.build_trace(R, results=torch.zeros((batch.num_rays, 4), dtype=torch.int32, device="cuda"))
    s.synchronize()
    ctx.check()
    got = res.cpu().numpy()
    for m, (V, T) in enumerate(meshes):
        o0, o1 = batch.ray_offset(m), batch.ray_offset(m + 1)
        plain = ctx.build(V, T, p)
        pn, pw, pt = plain.download()
        bn, bw, bt = batch.bvh(m).download()
        np.testing.assert_array_equal(bn, pn)
        np.testing.assert_array_equal(bt, pt)
        np.testing.assert_array_equal(bw.view(np.int32), pw.view(np.int32))
        Rm = R[o0:o1].contiguous()
        exp = ctx.trace(plain, Rm, results=torch.zeros((Rm.shape[0], 4), dtype=torch.int32, device="cuda"))
        np.testing.assert_array_equal(got[o0:o1], exp.cpu().numpy())
    batch.close()
