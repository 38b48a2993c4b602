"""The allocation-free sort entry point (ar_radix_sort_pairs_u32_noalloc).

It exists for callers that cannot allocate device memory -- a frame loop that must not stall
on cudaMalloc's implicit synchronisation, or code running while another component owns the
memory pool -- and keeps its workspace in a static array inside libarsim.so.  This file is
collected last, so a failure here comes after every other test has run.

Checks, through the C ABI: two calls in a row (the second one reuses whatever the first left
in the shared array) each give exactly the output of the regular ar_radix_sort_pairs_u32
and of numpy's stable argsort (integer keys and indices, so the tolerance is zero), over
plans with 8-bit digits only (21, 32 bits) and with a 9-bit digit (25 bits at 2^20 pairs),
the copy path (begin_bit == end_bit) and n = 0; the device's free memory is the same before
and after a call; the status word stays clear; sizes beyond the stated limit and outputs that
overlap their inputs are rejected before anything is launched."""
import numpy as np
import pytest
import torch

from gpu_util import P, S, dev, empty, host

pytestmark = pytest.mark.gpu

LIMIT = 1 << 20


def _regular(ctx, keys, vals, bits):
    from diploma_thesis_b200._lib import call
    n = len(keys)
    ko, vo = empty(n, torch.int32), empty(n, torch.int32)
    call("ar_radix_sort_pairs_u32", ctx.handle, P(dev(keys)), P(dev(vals)) if vals is not None else None,
         P(ko), P(vo), n, 0, bits, S())
    return host(ko, np.uint32), host(vo, np.uint32)


def _noalloc(keys, vals, bits, status):
    from diploma_thesis_b200._lib import call
    n = len(keys)
    ko, vo = empty(n, torch.int32), empty(n, torch.int32)
    call("ar_radix_sort_pairs_u32_noalloc", P(dev(keys)),
         P(dev(vals)) if vals is not None else None, P(ko), P(vo), n, 0, bits,
         P(status) if status is not None else None, S())
    return host(ko, np.uint32), host(vo, np.uint32)


def test_noalloc_sort_matches_regular_sort_twice_in_a_row(ctx):
    rng = np.random.default_rng(2024)
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    cases = [(300_001, 21, True), (LIMIT, 32, False), (LIMIT, 25, True)]
    for n, bits, with_vals in cases:
        keys = rng.integers(0, 1 << bits, n, dtype=np.uint64).astype(np.uint32)
        keys[: n // 4] = keys[n // 4: 2 * (n // 4)]  # ties: stability matters
        vals = rng.integers(0, 1 << 31, n).astype(np.uint32) if with_vals else None
        k_ref, v_ref = _regular(ctx, keys, vals, bits)
        order = np.argsort(keys, kind="stable")
        v_np = (vals[order] if vals is not None else order.astype(np.uint32))
        for _ in range(2):  # the second call starts from what the first left in the array
            k, v = _noalloc(keys, vals, bits, status)
            assert np.array_equal(k, k_ref) and np.array_equal(v, v_ref)
            assert np.array_equal(k, keys[order]) and np.array_equal(v, v_np)
    assert int(host(status)[0]) == 0
    assert ctx.status() == 0


def test_noalloc_sort_copy_path_and_empty_input(ctx):
    from diploma_thesis_b200._lib import call, lib
    rng = np.random.default_rng(7)
    n = 1000
    keys = rng.integers(0, 1 << 20, n, dtype=np.uint64).astype(np.uint32)
    for _ in range(2):
        k, v = _noalloc(keys, None, 0, None)  # begin_bit == end_bit == 0: keys as given, iota
        assert np.array_equal(k, keys) and np.array_equal(v, np.arange(n, dtype=np.uint32))
    ko, vo = empty(4, torch.int32), empty(4, torch.int32)
    call("ar_radix_sort_pairs_u32_noalloc", None, None, None, None, 0, 0, 32, None, S())
    call("ar_radix_sort_pairs_u32_noalloc", P(ko), None, P(ko), P(vo), 0, 0, 32, None, S())
    assert lib.ar_radix_sort_pairs_u32_noalloc(P(ko), None, P(ko), P(vo), 4, 0, 32, None,
                                               S()) == 1  # n > 0: aliasing is an error
    assert ctx.status() == 0


def test_noalloc_sort_allocates_no_device_memory(ctx):
    from diploma_thesis_b200._lib import call
    rng = np.random.default_rng(11)
    n = 500_000
    keys = dev(rng.integers(0, 1 << 30, n, dtype=np.uint64).astype(np.uint32))
    ko, vo = empty(n, torch.int32), empty(n, torch.int32)
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    call("ar_radix_sort_pairs_u32_noalloc", P(keys), None, P(ko), P(vo), n, 0, 30, P(status), S())
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    call("ar_radix_sort_pairs_u32_noalloc", P(keys), None, P(ko), P(vo), n, 0, 30, P(status), S())
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free_before
    order = np.argsort(host(keys, np.uint32), kind="stable").astype(np.uint32)
    assert np.array_equal(host(vo, np.uint32), order)
    assert int(host(status)[0]) == 0


def test_noalloc_sort_rejects_sizes_beyond_its_limit():
    from diploma_thesis_b200._lib import lib
    k = empty(4, torch.int32)
    st = lib.ar_radix_sort_pairs_u32_noalloc(P(k), None, P(empty(4, torch.int32)),
                                             P(empty(4, torch.int32)), LIMIT + 1, 0, 32, None, S())
    assert st == 1  # AR_ERR_INVALID_ARG
    assert b"limit" in lib.ar_last_error()
