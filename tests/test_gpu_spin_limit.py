"""Bounded waits give up cleanly: a radix sort whose look-back spin limit is
set to one spin reports HP_ERR_DEVICE_STATUS (a bounded wait gave up) through
hp_ctx_check instead of hanging, and the context stays usable: the next sort
with the default limit is exact.

With one spin allowed, any tile that finds an earlier tile's digit counts not
yet published gives up at once; the sort then scatters with the partial prefix
it has, which can only lower a key's output position, so every write stays
inside the output buffer (the output is discarded). Over 16 M keys and eight
passes (26,000 look-backs) some wait meets an unpublished word.
"""
import numpy as np
import pytest
import torch

import hippie_b200 as hp

pytestmark = pytest.mark.gpu


def test_sort_spin_limit_gives_up_with_device_status(ctx):
    n = 1 << 24
    rng = np.random.default_rng(5)
    keys = torch.from_numpy(rng.integers(0, 1 << 60, size=n, dtype=np.uint64).view(np.int64)).cuda()
    ctx.check()
    ctx.set_sort_spin_limit(1)
    try:
        ctx.radix_sort(keys, bits=60)
        with pytest.raises(hp.HPError) as e:
            ctx.check()
        assert e.value.status == 5  # HP_ERR_DEVICE_STATUS
        assert "bounded wait gave up" in str(e.value)
    finally:
        ctx.set_sort_spin_limit(0)
    ctx.check()  # the error word was cleared by the failing check
    ko, vo = ctx.radix_sort(keys, bits=60)
    ctx.check()
    order = np.argsort(keys.cpu().numpy().view(np.uint64), kind="stable")
    np.testing.assert_array_equal(vo.cpu().numpy(), order.astype(np.int32))
