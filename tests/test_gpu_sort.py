"""GPU radix sort: equals a stable sort by the low `bits` of each key (sm_100a)."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [1, 2, 100, 4095, 4096, 4097, 6143, 6144, 6145, 100000, 1 << 20])
@pytest.mark.parametrize("kb,bits", [(4, 32), (4, 30), (4, 13), (8, 60), (8, 64), (8, 41)])
def test_radix_sort_stable(ctx, n, kb, bits):
    rng = np.random.default_rng(n * 131 + bits)
    if kb == 4:
        keys = rng.integers(0, 1 << 32, size=n, dtype=np.uint64).astype(np.uint32)
        keys[: n // 3] = keys[0]  # a long run of duplicates
        K = torch.from_numpy(keys.view(np.int32)).cuda()
        mask = np.uint32((1 << bits) - 1) if bits < 32 else np.uint32(0xffffffff)
        sk = keys & mask
    else:
        keys = rng.integers(0, 1 << 63, size=n, dtype=np.uint64) * np.uint64(2) + rng.integers(0, 2, size=n,
                                                                                             dtype=np.uint64)
        keys[: n // 3] = keys[0]
        K = torch.from_numpy(keys.view(np.int64)).cuda()
        mask = np.uint64((1 << bits) - 1) if bits < 64 else np.uint64(0xffffffffffffffff)
        sk = keys & mask
    ko, vo = ctx.radix_sort(K, bits=bits)
    ctx.check()
    order = np.argsort(sk, kind="stable")
    np.testing.assert_array_equal(vo.cpu().numpy(), order.astype(np.int32))
    got = ko.cpu().numpy().view(keys.dtype)
    np.testing.assert_array_equal(got, keys[order])


def test_radix_sort_with_values(ctx):
    rng = np.random.default_rng(1)
    keys = rng.integers(0, 1 << 20, size=300000).astype(np.uint32)
    vals = rng.integers(-5, 5, size=300000).astype(np.int32)
    ko, vo = ctx.radix_sort(torch.from_numpy(keys.view(np.int32)).cuda(), torch.from_numpy(vals).cuda(), bits=20)
    order = np.argsort(keys, kind="stable")
    np.testing.assert_array_equal(vo.cpu().numpy(), vals[order])


def _wide_case(kind, n, bits, rng):
    """Keys for the wide-key path (bits > 48, n >= 2^20): the array is first
    ordered by its top 16 sorted bits, then every run of equal top bits is
    sorted by the rest, in shared memory, or by the large-segment kernel when
    a run exceeds 4096 keys."""
    low = rng.integers(0, 1 << (bits - 16), size=n, dtype=np.uint64)
    if kind == "uniform":
        top = rng.integers(0, 1 << 16, size=n, dtype=np.uint64)
    elif kind == "skewed":
        # one prefix with 30 % of the keys, 40 prefixes of 3,000-6,000 keys
        # around the shared-memory capacity, the rest spread out
        top = rng.integers(0, 1 << 16, size=n, dtype=np.uint64)
        top[: int(0.3 * n)] = 777
        sizes = rng.integers(3000, 6000, size=40)
        pos = int(0.3 * n)
        for k, m in enumerate(sizes):
            top[pos:pos + m] = 1000 + k
            pos += m
        rng.shuffle(top)
    else:  # one prefix only
        top = np.full(n, 4242, np.uint64)
    keys = (top << np.uint64(bits - 16)) | low
    keys[: n // 50] = keys[0]  # duplicates
    if bits < 64:  # bits above the sorted width are carried, not sorted
        keys |= rng.integers(0, 2, size=n, dtype=np.uint64) << np.uint64(63)
    return keys


@pytest.mark.parametrize("kind,n,bits", [("uniform", (1 << 20) + 123, 60), ("uniform", 3 << 20, 64),
                                         ("uniform", 1 << 21, 49), ("skewed", 1 << 21, 60),
                                         ("skewed", (1 << 20) + 7, 56), ("single", 1 << 20, 60)])
@pytest.mark.parametrize("with_vals", [False, True])
def test_radix_sort_wide_keys_by_segments(ctx, kind, n, bits, with_vals):
    rng = np.random.default_rng(n + bits + (7 if with_vals else 0))
    keys = _wide_case(kind, n, bits, rng)
    mask = np.uint64((1 << bits) - 1) if bits < 64 else np.uint64(0xffffffffffffffff)
    K = torch.from_numpy(keys.view(np.int64)).cuda()
    vals = rng.permutation(n).astype(np.int32) if with_vals else None
    ko, vo = ctx.radix_sort(K, None if vals is None else torch.from_numpy(vals).cuda(), bits=bits)
    ctx.check()
    order = np.argsort(keys & mask, kind="stable")
    np.testing.assert_array_equal(vo.cpu().numpy(), (vals[order] if with_vals else order.astype(np.int32)))
    np.testing.assert_array_equal(ko.cpu().numpy().view(np.uint64), keys[order])
