"""Builds captured in a CUDA graph: every builder and layout rebuilds into an
existing BVH from a graph replay, with nothing read back to the host inside
the build, and the replayed BVH equals the eagerly built one byte for byte."""
import numpy as np
import pytest
import torch

import hippie_b200 as hp

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("method,layout", [("lbvh", 2), ("ploc", 2), ("atr", 2), ("tr", 2), ("hlbvh", 2),
                                           ("ploc", 4), ("lbvh", 8)])
def test_build_replayed_from_graph_equals_eager(ctx, method, layout):
    v, t = hp.gen.clustered_mesh(31, 150000, 128, 0.03, 0.004)
    V, T = torch.from_numpy(v).cuda(), torch.from_numpy(t).cuda()
    p = hp.BuildParams(method=method, morton_bits=60, layout=layout, ploc_radius=8)
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        bvh = ctx.build(V, T, p, stream=s)  # allocates the BVH and the scratch arena
    s.synchronize()
    ref = [np.array(a, copy=True) for a in bvh.download()]
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        ctx.build(V, T, p, bvh=bvh, stream=s)
    nodes, woop, tri = bvh.arrays()
    nodes.zero_()
    woop.zero_()
    tri.fill_(-1)
    torch.cuda.synchronize()
    for _ in range(2):
        g.replay()
    torch.cuda.synchronize()
    ctx.check()
    got = bvh.download()
    for a, b in zip(ref, got):
        np.testing.assert_array_equal(np.asarray(a).view(np.uint8), np.asarray(b).view(np.uint8))
    del g
