"""Sort paths that the small sort tests do not reach, through the C ABI:

* match.any ranking (AR_SORT_RANK_MATCH) on 512-thread tiles, which the fused grid step uses
  from 2^19 keys on: n = 2^19 + 3 and 2^21 + 3 with 24- and 25-bit keys (the 25-bit plan
  adds a 9-bit pass, ranked by ballots), keys laid out like cell keys in particle order (runs
  of nearby values) and uniformly random, checked against numpy's stable argsort and the
  oracle;
* the look-back's bounded wait: with AR_SORT_TEST_MUTE_FIRST_TILE, tile 0 never publishes its
  status, so every later tile's look-back runs out of polls; the context then reports
  AR_ERR_TIMEOUT, and guard words on both sides of every output stay untouched."""
import numpy as np
import pytest
import torch

from gpu_util import P, S, dev, empty, host
from oracle import cpu

pytestmark = pytest.mark.gpu

AR_SORT_RANK_MATCH = 1
AR_SORT_TEST_MUTE_FIRST_TILE = 0x80000000
AR_ERR_TIMEOUT = 3


def _cell_like_keys(rng, n, bits):
    """Runs of 64 keys near one another (a body's particles fall in neighbouring cells)."""
    base = rng.integers(0, 1 << bits, (n + 63) // 64, dtype=np.int64)
    off = rng.integers(-300, 300, ((n + 63) // 64, 64))
    return np.clip(base[:, None] + off, 0, (1 << bits) - 1).reshape(-1)[:n].astype(np.uint32)


def _sort_ex(ctx, keys, vals, bits, flags):
    from diploma_thesis_b200._lib import call
    n = len(keys)
    ko, vo = empty(n, torch.int32), empty(n, torch.int32)
    call("ar_radix_sort_pairs_u32_ex", ctx.handle, P(dev(keys)),
         P(dev(vals)) if vals is not None else None, P(ko), P(vo), n, 0, bits, flags, S())
    return host(ko, np.uint32), host(vo, np.uint32)


@pytest.mark.parametrize("n,bits,layout", [((1 << 19) + 3, 24, "cells"),
                                           ((1 << 21) + 3, 25, "cells"),
                                           ((1 << 21) + 3, 24, "random")])
def test_match_rank_on_512_thread_tiles(ctx, n, bits, layout):
    rng = np.random.default_rng(n + bits)
    if layout == "cells":
        keys = _cell_like_keys(rng, n, bits)
    else:
        keys = rng.integers(0, 1 << bits, n, dtype=np.uint64).astype(np.uint32)
    keys[: n // 8] = keys[n // 8: 2 * (n // 8)]  # exact ties: stability matters
    order = np.argsort(keys, kind="stable").astype(np.uint32)
    for flags in (AR_SORT_RANK_MATCH, 0):
        k, v = _sort_ex(ctx, keys, None, bits, flags)
        assert np.array_equal(v, order), f"permutation differs (flags {flags})"
        assert np.array_equal(k, keys[order])
    vals = rng.integers(0, 1 << 31, n).astype(np.uint32)
    k, v = _sort_ex(ctx, keys, vals, bits, AR_SORT_RANK_MATCH)
    k_ref, v_ref = cpu.sort_pairs(keys, vals, 0, bits)
    assert np.array_equal(k, k_ref) and np.array_equal(v, v_ref)
    assert ctx.status() == 0


def test_lookback_timeout_is_reported_and_writes_stay_in_range(ctx):
    from diploma_thesis_b200._lib import lib
    rng = np.random.default_rng(5)
    n = 3 * 8192 + 17  # four 512-thread tiles per pass
    bits = 24
    keys = rng.integers(0, 1 << bits, n, dtype=np.uint64).astype(np.uint32)
    guard = 4096
    sentinel = np.int32(0x5A5A5A5A)
    ko = torch.full((n + 2 * guard,), int(sentinel), dtype=torch.int32, device="cuda")
    vo = torch.full((n + 2 * guard,), int(sentinel), dtype=torch.int32, device="cuda")
    kin = dev(keys)
    st = lib.ar_radix_sort_pairs_u32_ex(ctx.handle, P(kin), None, P(ko[guard:guard + n]),
                                        P(vo[guard:guard + n]), n, 0, bits,
                                        AR_SORT_TEST_MUTE_FIRST_TILE, S())
    assert st == 0  # launched; the failure is reported by the device
    assert ctx.status() == AR_ERR_TIMEOUT
    assert ctx.status() == 0  # reading the status clears it
    for buf in (ko, vo):
        h = host(buf)
        assert (h[:guard] == sentinel).all() and (h[guard + n:] == sentinel).all()
    assert np.array_equal(host(kin, np.uint32), keys)  # the input is left intact
    # the context stays usable: a normal sort right after is exact
    k, v = _sort_ex(ctx, keys, None, bits, 0)
    assert np.array_equal(v, np.argsort(keys, kind="stable").astype(np.uint32))
    assert ctx.status() == 0
