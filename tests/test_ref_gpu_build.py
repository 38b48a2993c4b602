"""The reference-GPU baseline library (oracle/_ref/libref_gpu.so, built from the reference's
CUDA sources by oracle/ref_gpu_build.py) loads without a GPU and exports the entry points
oracle/ref_gpu.py binds.  No compute call is made here; tests/test_gpu_ref_gpu.py runs it."""
import ctypes as C

import pytest

from oracle import ref_gpu


@pytest.mark.skipif(not ref_gpu.available(), reason="the reference GPU build is not present")
def test_reference_gpu_library_loads_and_exports_its_entry_points():
    lib = C.CDLL(str(ref_gpu._SO))
    for name in ("ref_gpu_create", "ref_gpu_step", "ref_gpu_download", "ref_gpu_destroy",
                 "ref_gpu_last_error", "ref_gpu_stages"):
        assert hasattr(lib, name), name
    assert lib.ref_gpu_stages() == len(ref_gpu.STAGES)
