"""ath_sort_pairs_static: the radix sort for callers that cannot allocate device
memory while they sort (a plugin whose host application owns the device memory
and holds it to a fixed budget mid-frame). Its working memory is a fixed array in
the library, so the test checks that its results equal the allocating
ath_sorter_sort's on two calls in a row (the second must not see the first's
leftovers), that it rejects counts past its limit, and that a call takes no
device memory. Collected last, so that a run stopping at its first failure has
run everything else first; it passes alone in a fresh process too. A call reads
nothing back: its status is asked for separately (ath_sort_pairs_static_status).
"""
import ctypes as C

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

LIMIT = 1 << 20


def _keys(count: int, key_bits: int, seed: int):
    rng = np.random.default_rng(seed)
    keys = rng.integers(0, 1 << min(key_bits, 63), size=count, dtype=np.uint64)
    keys[::7] = keys[0]   # ties, which the sort must keep in input order
    return keys, np.arange(count, dtype=np.uint32)


def _sort(N, fn, keys, vals, key_bits, handle=None):
    k = torch.from_numpy(keys.view(np.int64).copy()).cuda()
    v = torch.from_numpy(vals.view(np.int32).copy()).cuda()
    sk, sv = torch.empty_like(k), torch.empty_like(v)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    args = [C.c_void_p(k.data_ptr()), C.c_void_p(v.data_ptr()), C.c_void_p(sk.data_ptr()),
            C.c_void_p(sv.data_ptr()), keys.shape[0], key_bits, stream]
    N.check(fn(handle, *args) if handle is not None else fn(*args))
    torch.cuda.synchronize()
    return k.cpu().numpy().view(np.uint64), v.cpu().numpy().view(np.uint32)


# (LIMIT, 64) sorts in eight 8-bit passes, 63 bits in seven 9-bit passes (the most look-back words);
# 48 bits is an even pass count (6) at the limit, whose result needs no copy back.
@pytest.mark.parametrize("count,key_bits", [(65537, 40), (LIMIT, 37), (LIMIT, 64), (LIMIT, 63), (LIMIT, 48)])
def test_static_sort_equals_the_allocating_sort_twice_in_a_row(native, count, key_bits):
    N = native
    lib = N.lib()
    h = C.c_void_p()
    N.check(lib.ath_sorter_create(C.byref(h)))
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    try:
        for call, seed in enumerate((1, 2)):
            keys, vals = _keys(count, key_bits, seed + count)
            want = _sort(N, lib.ath_sorter_sort, keys, vals, key_bits, handle=h)
            got = _sort(N, lib.ath_sort_pairs_static, keys, vals, key_bits)
            np.testing.assert_array_equal(got[0], want[0], err_msg=f"keys, call {call}")
            np.testing.assert_array_equal(got[1], want[1], err_msg=f"values, call {call}")
        # neither call raised anything: the status, asked for once both are done
        N.check(lib.ath_sort_pairs_static_status(stream))
        N.check(lib.ath_sorter_check(h))
    finally:
        lib.ath_sorter_destroy(h)


def test_static_sort_rejects_counts_past_its_limit(native):
    N = native
    status = N.lib().ath_sort_pairs_static(None, None, None, None, LIMIT + 1, 32, None)
    assert status == 3   # InvalidArgument
    assert b"limit" in N.lib().ath_last_error_message()


def test_static_sort_takes_no_device_memory(native):
    N = native
    keys, vals = _keys(200_000, 32, 7)
    _sort(N, N.lib().ath_sort_pairs_static, keys, vals, 32)   # the first call on a device sets up
    k = torch.from_numpy(keys.view(np.int64).copy()).cuda()
    v = torch.from_numpy(vals.view(np.int32).copy()).cuda()
    sk, sv = torch.empty_like(k), torch.empty_like(v)
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    for _ in range(3):
        N.check(N.lib().ath_sort_pairs_static(C.c_void_p(k.data_ptr()), C.c_void_p(v.data_ptr()),
                                              C.c_void_p(sk.data_ptr()), C.c_void_p(sv.data_ptr()), keys.shape[0],
                                              32, stream))
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free_before
    order = np.argsort(keys, kind="stable")
    np.testing.assert_array_equal(v.cpu().numpy().view(np.uint32), vals[order])
