"""The C ABI library loads, exports exactly what include/arsim.h declares, and reports
argument errors without touching a GPU."""
import ctypes as C
import re
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "arsim.h"
LIB = ROOT / "diploma_thesis_b200" / "libarsim.so"


def declared_symbols() -> set[str]:
    text = HEADER.read_text()
    return set(re.findall(r"AR_API\s+[\w\s\*]+?\b(ar_\w+)\s*\(", text))


def test_library_exports_every_declared_symbol():
    assert LIB.exists(), "build with `python -m diploma_thesis_b200.build`"
    out = subprocess.run(["nm", "-D", "--defined-only", str(LIB)], capture_output=True,
                         text=True, check=True).stdout
    exported = set(re.findall(r"\bT (ar_\w+)", out))
    declared = declared_symbols()
    assert len(declared) >= 40
    assert declared <= exported, sorted(declared - exported)
    # nothing undeclared leaks out under the ar_ prefix
    assert exported <= declared, sorted(exported - declared)


def test_sim_params_layout_matches_reference():
    from diploma_thesis_b200._lib import SimParams
    assert C.sizeof(SimParams) == 128  # sizeof(SimParams), Kernels/particleSystem.cuh:27-55
    from oracle import ref
    if ref.available():
        assert ref.lib().refcpu_sizeof_simparams() == 128


def test_argument_errors_need_no_gpu():
    from diploma_thesis_b200 import _lib
    L = _lib.lib
    assert L.ar_ctx_create(0, None) == 1  # INVALID_ARG
    assert L.ar_scene_destroy(None) == 1
    assert L.ar_batch_destroy(None) == 1
    assert L.ar_radix_sort_pairs_u32(None, None, None, None, None, 0, 0, 32, None) == 1
    assert L.ar_step(None, None, 1, 1, None) == 1
    assert L.ar_scene_footprint(None) == 0
    assert L.ar_version().startswith(b"arsim-b200")


def test_context_without_gpu_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from diploma_thesis_b200 import _lib
    h = C.c_void_p()
    st = _lib.lib.ar_ctx_create(0, C.byref(h))
    assert st == 5  # AR_ERR_CUDA, not a crash
    assert b"cudaSetDevice" in _lib.lib.ar_last_error()


def test_scene_footprint_scales_with_size():
    from diploma_thesis_b200 import _lib, api, scenes
    s = scenes.small_scene(0, nb_side=4)
    for bp, factor in ((0, 2), (1, 5)):  # grid: the cell table grows slower than N
        d = api.make_desc(s, bp)
        f1 = _lib.lib.ar_scene_footprint(C.byref(d))
        d.num_particles *= 10
        d.num_bodies *= 10
        assert _lib.lib.ar_scene_footprint(C.byref(d)) > factor * f1 > 0
        assert (_lib.lib.ar_scene_cells(C.byref(d)) > 0) == (bp == 0)


def test_sort_rejects_overlapping_outputs_without_a_gpu():
    """The allocation-free sort checks its arguments before any CUDA call: outputs that
    overlap an input (or each other) anywhere, not only at the same start address."""
    from diploma_thesis_b200 import _lib
    L = _lib.lib
    f = L.ar_radix_sort_pairs_u32_noalloc
    a, b, c = 0x100000, 0x200000, 0x300000  # never dereferenced: rejected first
    n = 1024
    assert f(C.c_void_p(a), None, C.c_void_p(a + 4), C.c_void_p(b), n, 0, 32, None, None) == 1
    assert b"overlap" in L.ar_last_error()
    assert f(C.c_void_p(a), C.c_void_p(b), C.c_void_p(c), C.c_void_p(b + 4 * n - 4), n, 0, 32,
             None, None) == 1
    assert f(C.c_void_p(a), None, C.c_void_p(b), C.c_void_p(b + 4 * n - 4), n, 0, 32, None,
             None) == 1
    assert f(C.c_void_p(a), None, C.c_void_p(c), C.c_void_p(a), n, 0, 32, None, None) == 1
    assert L.ar_radix_sort_pairs_u32_ex(None, None, None, None, None, 0, 0, 32, 0, None) == 1
