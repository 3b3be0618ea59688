"""The C-ABI library: loads, exports every declared symbol, rejects bad arguments
without a GPU, and its generators are deterministic (CPU only)."""
import ctypes as C
import re
from pathlib import Path

import numpy as np

import hippie_b200 as hp
from hippie_b200 import _lib

ROOT = Path(__file__).resolve().parent.parent


def _declared():
    text = (ROOT / "include" / "hippie_b200.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(hp_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    declared = _declared()
    assert len(declared) >= 30
    for name in declared:
        assert hasattr(lib, name), name
    assert set(_lib.exported_symbols()) <= set(declared)
    assert lib.hp_abi_version() == 2


def test_bad_arguments_are_rejected():
    lib = _lib.load()
    assert lib.hp_build(None, None, None, None, None, None) == 2
    assert lib.hp_trace(None, None, None, 0, None, None, 0, None) == 2
    assert lib.hp_radix_sort(None, None, None, None, None, 10, 4, 32, None) == 2
    assert lib.hp_trace_host(None, None, None, 10, None, None, 0, 0, None) == 2
    assert b"null" in lib.hp_last_error()


def test_context_without_device_reports_error():
    import torch
    if torch.cuda.is_available():
        return
    h = C.c_void_p()
    st = _lib.load().hp_ctx_create(C.byref(h), 0)
    assert st in (1, 2)  # HP_ERR_CUDA or HP_ERR_ARG, never a crash


def test_generators_deterministic():
    v1, t1 = hp.gen.uniform_mesh(7, 1000)
    v2, t2 = hp.gen.uniform_mesh(7, 1000)
    np.testing.assert_array_equal(v1, v2)
    assert t1.tolist()[:2] == [[0, 1, 2], [3, 4, 5]]
    c = v1.reshape(-1, 3, 3).mean(1)
    assert c.min() >= -0.011 and c.max() <= 1.011
    d = np.abs(v1.reshape(-1, 3, 3) - v1.reshape(-1, 3, 3).mean(1, keepdims=True))
    assert d.max() <= 0.02
    vc, tc = hp.gen.clustered_mesh(7, 4096, clusters=16)
    assert vc.shape == (3 * 4096, 3)
    r = hp.gen.rays_targeted(3, 500)
    assert np.allclose(np.linalg.norm(r[:, 4:7], axis=1), 1, atol=1e-6)
    assert np.all(r[:, 3] == 0) and np.all(np.isinf(r[:, 7]))
    rs = hp.gen.rays_sphere(3, 500, np.array([0, 0, 0, 1, 1, 1], np.float32))
    assert np.allclose(np.linalg.norm(rs[:, 4:7], axis=1), 1, atol=1e-6)
    vh, th = hp.gen.heightfield(5, 16, 32)
    assert th.shape == (2 * 15 * 31, 3) and vh.shape == (16 * 32, 3)
    assert np.abs(vh[:, 2]).max() <= 16 * 0.05
    rg = hp.gen.rays_grid_down(1, 8, 8)
    assert np.all(rg[:, 6] == -1) and np.all(rg[:, 2] == 1)


def test_tune_defaults():
    """hp_tune_default: the launch choices every context starts from (host only)."""
    import ctypes as C
    t = _lib.hp_tune()
    _lib.load().hp_tune_default(C.byref(t))
    assert (t.sort_block, t.trace_ctas_per_sm, t.trace_stack, t.trace_sorted) == (512, 0, 16, 0)
    assert (t.ploc_radius, t.ploc_adaptive, t.ploc_max_radius) == (0, 0, 0)
    assert C.sizeof(t) == 64
