"""The radix sort entry point that allocates no device memory.

mc_radix_sort_pairs_static sorts through a fixed scratch array inside the
library instead of context scratch. It must give exactly the keys and values
mc_radix_sort_pairs gives (both are stable sorts of integers), on consecutive
calls that reuse the scratch, and must not change the device's free memory.
This file is collected last so that it also runs after every other test in one
process; it passes alone as well.
"""
import ctypes as C

import numpy as np
import pytest

import mcpt

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _pairs(rng, n):
    keys = rng.integers(0, 1 << 30, n, dtype=np.uint32)
    keys[::5] = keys[3]  # long runs of equal keys: the value order shows stability
    vals = np.arange(n, dtype=np.int32)[::-1].copy()
    return keys, vals


def _device(keys, vals):
    return torch.from_numpy(keys.view(np.int32)).cuda(), torch.from_numpy(vals).cuda()


def _host(k, v):
    return k.cpu().numpy().view(np.uint32), v.cpu().numpy()


def test_static_sort_equals_allocating_sort_on_consecutive_calls():
    ctx = mcpt.Context(0)
    lib = ctx.lib
    try:
        # set-up call: no pairs, no pointers
        mcpt.check(lib.mc_radix_sort_pairs_static(ctx.handle, None, None, 0, 30))
        rng = np.random.default_rng(2024)
        # two calls in a row on the same scratch: 30-bit keys (4 passes), then
        # 24-bit keys (3 passes, result copied back) at the maximum size
        for n, bits in ((300_001, 30), (mcpt.SORT_STATIC_MAX_PAIRS, 24)):
            keys, vals = _pairs(rng, n)
            keys &= np.uint32((1 << bits) - 1)
            ks, vs = _device(keys, vals)
            kr, vr = _device(keys, vals)
            torch.cuda.synchronize()
            free_before = torch.cuda.mem_get_info()[0]
            mcpt.check(lib.mc_radix_sort_pairs_static(ctx.handle, ks.data_ptr(), vs.data_ptr(), n, bits))
            torch.cuda.synchronize()
            free_after = torch.cuda.mem_get_info()[0]
            assert free_after == free_before, "the static sort changed free device memory"
            mcpt.check(lib.mc_radix_sort_pairs(ctx.handle, kr.data_ptr(), vr.data_ptr(), n, bits))
            got_k, got_v = _host(ks, vs)
            ref_k, ref_v = _host(kr, vr)
            assert np.array_equal(got_k, ref_k)
            assert np.array_equal(got_v, ref_v)
            order = np.argsort(keys, kind="stable")
            assert np.array_equal(got_k, keys[order])
            assert np.array_equal(got_v, vals[order])
    finally:
        ctx.close()


def test_static_sort_rejects_sizes_beyond_its_scratch():
    ctx = mcpt.Context(0)
    try:
        k = torch.zeros(8, dtype=torch.int32, device="cuda")
        st = ctx.lib.mc_radix_sort_pairs_static(ctx.handle, k.data_ptr(), k.data_ptr(), mcpt.SORT_STATIC_MAX_PAIRS + 1, 30)
        assert st == 1  # MC_ERR_INVALID, before any launch
        assert b"exceeds" in ctx.lib.mc_last_error()
        assert ctx.lib.mc_radix_sort_pairs_static(ctx.handle, k.data_ptr(), k.data_ptr(), 8, 0) == 1
    finally:
        ctx.close()
