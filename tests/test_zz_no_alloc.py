"""The allocation-free sort entry point (ar_radix_sort_pairs_u32_noalloc).

It exists for callers that cannot allocate device memory -- a frame loop that must not stall
on cudaMalloc's implicit synchronisation, or code running while another component owns the
memory pool -- and keeps its workspace in a static array inside libarsim.so.  This file is
collected last, so a failure here comes after every other test has run.

Checks, through the C ABI: two calls in a row (the second one reuses whatever the first left
in the shared array) each give exactly the output of the regular ar_radix_sort_pairs_u32
(integer keys and indices, so the tolerance is zero); the status word stays clear; sizes
beyond the stated limit are rejected before anything is launched."""
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
         P(dev(vals)) if vals is not None else None, P(ko), P(vo), n, 0, bits, P(status), S())
    return host(ko, np.uint32), host(vo, np.uint32)


def test_noalloc_sort_matches_regular_sort_twice_in_a_row(ctx):
    rng = np.random.default_rng(2024)
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    cases = [(300_001, 21, True), (LIMIT, 32, False)]
    for n, bits, with_vals in cases:
        keys = rng.integers(0, 1 << bits, n, dtype=np.uint64).astype(np.uint32)
        keys[: n // 4] = keys[n // 4: 2 * (n // 4)]  # ties: stability matters
        vals = rng.integers(0, 1 << 31, n).astype(np.uint32) if with_vals else None
        k_ref, v_ref = _regular(ctx, keys, vals, bits)
        k, v = _noalloc(keys, vals, bits, status)
        assert np.array_equal(k, k_ref) and np.array_equal(v, v_ref)
    assert int(host(status)[0]) == 0
    assert ctx.status() == 0


def test_noalloc_sort_rejects_sizes_beyond_its_limit():
    from diploma_thesis_b200._lib import lib
    k = empty(4, torch.int32)
    st = lib.ar_radix_sort_pairs_u32_noalloc(P(k), None, P(empty(4, torch.int32)),
                                             P(empty(4, torch.int32)), LIMIT + 1, 0, 32, None, S())
    assert st == 1  # AR_ERR_INVALID_ARG
    assert b"limit" in lib.ar_last_error()
