"""The allocation-free sort entry point, hp_radix_sort_noalloc, through the C ABI.

It exists for callers that cannot allocate GPU memory themselves: a plugin
inside a host application that owns the device memory budget, or a frame loop
that cannot afford the device synchronisation an allocation may imply. Its
scratch lives in a fixed device array inside the library, so two calls in a
row must each start from a clean state. Each call here is checked against the
arena-backed hp_radix_sort on the same keys (results must be identical: the
sort is an integer permutation). This file is collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from hippie_b200 import _lib

pytestmark = pytest.mark.gpu

MAX_KEYS = 262144  # HP_NOALLOC_SORT_MAX_KEYS in include/hippie_b200.h


def _keys(n, kb, bits, seed):
    rng = np.random.default_rng(seed)
    if kb == 4:
        k = rng.integers(0, 1 << bits, size=n, dtype=np.uint64).astype(np.uint32)
        k[: n // 4] = k[0]
        return torch.from_numpy(k.view(np.int32)).cuda()
    k = rng.integers(0, 1 << min(bits, 63), size=n, dtype=np.uint64)
    k[: n // 4] = k[0]
    return torch.from_numpy(k.view(np.int64)).cuda()


def test_noalloc_sort_matches_arena_sort_on_consecutive_calls():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import hippie_b200 as hp
    lib = _lib.load()
    ctx = hp.Context(0)
    stream = torch.cuda.current_stream()
    # One int32 of status, as the header documents; it starts with a stale
    # nonzero value because every call overwrites it with its own code.
    status = torch.full((1,), 7, dtype=torch.int32, device="cuda")
    cases = [  # (n, key bytes, bits, caller values, status word)
        (200003, 8, 60, False, True),
        (MAX_KEYS, 4, 30, True, True),   # caller-supplied values: a permutation
        (4099, 8, 64, False, False),     # no status word
        (70001, 4, 8, True, True),       # one pass, written straight to the output
        (MAX_KEYS, 8, 60, True, False),
    ]
    for call, (n, kb, bits, with_vals, with_status) in enumerate(cases):
        K = _keys(n, kb, bits, seed=call)
        V = None
        if with_vals:
            V = torch.from_numpy(np.random.default_rng(100 + call).permutation(n).astype(np.int32)).cuda()
        ref_k, ref_v = ctx.radix_sort(K, vals=V, bits=bits)
        ctx.check()
        out_k = torch.full_like(K, -1)
        out_v = torch.full((n,), -1, dtype=torch.int32, device="cuda")
        st = lib.hp_radix_sort_noalloc(C.c_void_p(K.data_ptr()), None if V is None else C.c_void_p(V.data_ptr()),
                                       C.c_void_p(out_k.data_ptr()), C.c_void_p(out_v.data_ptr()), n, kb, bits,
                                       C.c_void_p(status.data_ptr()) if with_status else None,
                                       C.c_void_p(stream.cuda_stream))
        assert st == 0, lib.hp_last_error()
        torch.cuda.synchronize()
        if with_status:
            assert int(status.item()) == 0
        assert torch.equal(out_v, ref_v), f"call {call}: values differ"
        assert torch.equal(out_k, ref_k), f"call {call}: keys differ"
    ctx.close()


def test_noalloc_sort_rejects_sizes_beyond_its_scratch():
    lib = _lib.load()
    dummy = C.c_void_p(16)  # never dereferenced: the size check comes first
    st = lib.hp_radix_sort_noalloc(dummy, None, dummy, dummy, MAX_KEYS + 1, 4, 32, None, None)
    assert st == 2
    assert b"exceeds the fixed scratch capacity" in lib.hp_last_error()
