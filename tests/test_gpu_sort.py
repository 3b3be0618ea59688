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
