"""The CPU oracle against outputs of the REFERENCE's own CUDA kernels (CPU only).

tests/golden/ref_fixtures.npz was produced by tests/golden/make_ref_fixtures.py
on a B200 from the reference's kernels (oracle/_ref). The meshes are
regenerated here from the same seeds; the oracle, given the scene box and the
Morton scale the reference used, must reproduce the reference bit for bit up to
the collapse, and the same trees in canonical form after it.
"""
from pathlib import Path

import numpy as np
import pytest

import hippie_b200 as hp
import oracle

FIX = Path(__file__).resolve().parent / "golden" / "ref_fixtures.npz"
CASES = {"uniform": (lambda: hp.gen.uniform_mesh(71, 3000), 30),
         "clustered": (lambda: hp.gen.clustered_mesh(72, 4000, 16), 60)}


@pytest.fixture(scope="module")
def fx():
    return np.load(FIX)


def canonical(nodes, tri_idx):
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


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_lbvh_equals_reference_kernels(fx, name):
    make, bits = CASES[name]
    v, t = make()
    box, scale = fx[f"{name}_box"], fx[f"{name}_scale"]
    bmin, bmax, obox = oracle.tri_boxes(v, t)
    np.testing.assert_array_equal(obox, box)
    keys, _ = oracle.morton(bmin, bmax, box, bits, scale=scale)
    np.testing.assert_array_equal(keys, fx[f"{name}_lbvh_keys"].view(np.uint64))
    sk, sr = oracle.sort(keys, bits)
    np.testing.assert_array_equal(sk, fx[f"{name}_lbvh_sorted"].view(np.uint64))
    np.testing.assert_array_equal(sr, fx[f"{name}_lbvh_refs"])
    parent, left, right = oracle.karras(sk)
    np.testing.assert_array_equal(parent, fx[f"{name}_lbvh_parent"])
    np.testing.assert_array_equal(left, fx[f"{name}_lbvh_left"])
    np.testing.assert_array_equal(right, fx[f"{name}_lbvh_right"])
    nbmin, nbmax, _, _, _ = oracle.refit(v, t, sr, parent, left, right)
    np.testing.assert_array_equal(nbmin[:, :3], fx[f"{name}_lbvh_bmin"][:, :3])
    np.testing.assert_array_equal(nbmax[:, :3], fx[f"{name}_lbvh_bmax"][:, :3])
    r = oracle.build_lbvh(v, t, bits=bits, scale=scale)
    np.testing.assert_array_equal(r["counts"], fx[f"{name}_lbvh_counts"])
    assert canonical(r["nodes"], r["tri_idx"]) == canonical(fx[f"{name}_lbvh_nodes"], fx[f"{name}_lbvh_tri_idx"])


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_ploc_equals_reference_kernels(fx, name):
    make, bits = CASES[name]
    v, t = make()
    r = oracle.build_ploc(v, t, bits=bits, radius=4, max_radius=64, scale=fx[f"{name}_scale"])
    np.testing.assert_array_equal(r["counts"], fx[f"{name}_ploc_counts"])
    assert canonical(r["nodes"], r["tri_idx"]) == canonical(fx[f"{name}_ploc_nodes"], fx[f"{name}_ploc_tri_idx"])


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_atr_equals_reference_kernels(fx, name):
    if f"{name}_atr_nodes" not in fx:
        pytest.skip("fixture predates the ATR vectors")
    make, bits = CASES[name]
    v, t = make()
    r = oracle.build_atr(v, t, bits=bits, treelet=9, iterations=2, scale=fx[f"{name}_scale"])
    np.testing.assert_array_equal(r["counts"], fx[f"{name}_atr_counts"])
    assert canonical(r["nodes"], r["tri_idx"]) == canonical(fx[f"{name}_atr_nodes"], fx[f"{name}_atr_tri_idx"])


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_trace_on_reference_bvh(fx, name):
    """The oracle's traversal of the reference's own BVH finds the reference tracer's hits."""
    v, t = CASES[name][0]()
    rays = hp.gen.rays_targeted(73, 2000) if name == "uniform" else \
        hp.gen.rays_sphere(74, 2000, np.concatenate([v.min(0), v.max(0)]))
    ref = fx[f"{name}_trace"]
    got = oracle.trace(fx[f"{name}_lbvh_nodes"], fx[f"{name}_lbvh_woop"], fx[f"{name}_lbvh_tri_idx"], rays)
    assert np.mean((got[:, 0] >= 0) == (ref[:, 0] >= 0)) >= 0.999
    both = (got[:, 0] >= 0) & (ref[:, 0] >= 0)
    assert np.mean(got[both, 0] == ref[both, 0]) >= 0.999
    tt = got[both, 1].view(np.float32).astype(np.float64)
    tr = ref[both, 1].view(np.float32).astype(np.float64)
    assert np.quantile(np.abs(tt - tr) / np.maximum(1.0, tr), 0.99) <= 1e-6
