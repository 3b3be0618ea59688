"""Launch-choice tuning (hp_tune / hp_autotune): every result-neutral choice
gives bit-identical BVHs and hits, and the autotuner returns valid choices
(sm_100a)."""
import numpy as np
import pytest
import torch

import hippie_b200 as hp
import oracle

pytestmark = pytest.mark.gpu


def _zeros(n):
    return torch.zeros((n, 4), dtype=torch.int32, device="cuda")


@pytest.fixture(scope="module")
def scene():
    v, t = hp.gen.clustered_mesh(81, 300000, 256)
    rays = hp.gen.rays_sphere(82, 1 << 19, np.concatenate([v.min(0), v.max(0)]))
    return v, t, rays


def test_choices_do_not_change_results(ctx, scene):
    v, t, rays = scene
    V, T, R = (torch.from_numpy(x).cuda() for x in (v, t, rays))
    p = hp.BuildParams(method="ploc", morton_bits=60, ploc_radius=16, ploc_max_radius=256)
    ctx.reset_tune()
    ref_bvh = ctx.build(V, T, p)
    ref_nodes = ref_bvh.download()
    ref_hits = ctx.trace(ref_bvh, R, results=_zeros(R.shape[0])).cpu().numpy()
    try:
        for kw in [dict(sort_block=256), dict(trace_stack=8), dict(trace_stack=32), dict(trace_ctas_per_sm=4),
                   dict(trace_sorted=1), dict(sort_block=256, trace_stack=32, trace_ctas_per_sm=6, trace_sorted=1)]:
            ctx.reset_tune()
            ctx.set_tune(**kw)
            b = ctx.build(V, T, p)
            got = b.download()
            for x, y in zip(got, ref_nodes):
                np.testing.assert_array_equal(x, y)
            hits = ctx.trace(b, R, results=_zeros(R.shape[0])).cpu().numpy()
            np.testing.assert_array_equal(hits, ref_hits)
            ctx.check()
    finally:
        ctx.reset_tune()
    nodes, woop, tri = ref_nodes
    np.testing.assert_array_equal(ref_hits[:20000], oracle.trace(nodes, woop, tri, rays[:20000]))


def test_set_tune_rejects_bad_values(ctx):
    for kw in [dict(sort_block=128), dict(trace_stack=12), dict(trace_ctas_per_sm=-1), dict(trace_sorted=2)]:
        with pytest.raises(hp.HPError):
            ctx.set_tune(**kw)
    assert ctx.get_tune()["sort_block"] == 512


def test_autotune(ctx, scene):
    v, t, rays = scene
    V, T, R = (torch.from_numpy(x).cuda() for x in (v, t, rays))
    p = hp.BuildParams(method="ploc", morton_bits=60, ploc_radius=16, ploc_max_radius=256)
    try:
        got = ctx.autotune(V, T, R, p, ploc_radius=True)
        assert got["sort_block"] in (256, 512)
        assert got["trace_stack"] in (8, 16, 32)
        assert got["trace_sorted"] in (0, 1)
        assert got["ploc_radius"] in (4, 8, 16, 32)
        assert got["build_ms"] > 0 and got["trace_ms"] > 0
        applied = ctx.get_tune()
        for k in ("sort_block", "trace_stack", "trace_sorted", "trace_ctas_per_sm"):
            assert applied[k] == got[k]
        # the tuned context still gives the default results
        b = ctx.build(V, T, p)
        hits = ctx.trace(b, R, results=_zeros(R.shape[0])).cpu().numpy()
        ctx.reset_tune()
        b2 = ctx.build(V, T, p)
        np.testing.assert_array_equal(hits, ctx.trace(b2, R, results=_zeros(R.shape[0])).cpu().numpy())
    finally:
        ctx.reset_tune()
