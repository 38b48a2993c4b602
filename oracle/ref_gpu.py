"""ctypes wrapper of oracle/_ref/libref_gpu.so -- the reference's own GPU step
(updateUniformGridDEM) on this GPU, built from the reference's CUDA sources by
oracle/ref_gpu_build.py.

BASELINE / TEST INFRASTRUCTURE ONLY: bench.py's reference-GPU workload times it beside this
repository's step, and a GPU test checks it against the reference's CPU build; the product
never loads it.  ``available()`` is False where it was not built (no reference checkout).
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

_SO = Path(__file__).resolve().parent / "_ref" / "libref_gpu.so"
# integrate (with its allocations and copies) | reset impulses | hash | sort | reorder (with the
# full-grid cellStart clear) | collide | reduce (scans, host prefix, combine)
STAGES = ["integrate", "reset", "hash", "sort", "reorder", "collide", "reduce"]


def available() -> bool:
    return _SO.exists()


def _f(a: np.ndarray):
    return np.ascontiguousarray(a, np.float32).ctypes.data_as(C.c_void_p)


class RefGpuStep:
    """One scene stepped by the reference's GPU code (one at a time per process: the library
    keeps a single scene)."""

    def __init__(self, scene, grid):
        from oracle.ref_step import reference_layout
        self.lib = C.CDLL(str(_SO))
        self.lib.ref_gpu_last_error.restype = C.c_char_p
        L = reference_layout(scene, grid)
        self.nb, self.n = scene.num_bodies, scene.num_particles
        keep = [np.ascontiguousarray(L[k], np.float32) for k in
                ("cms", "vel", "ang", "cum", "ib", "mass", "rel")]
        rb = np.ascontiguousarray(L["rb"], np.int32)
        counts = np.ascontiguousarray(L["counts"], np.int32)
        st = self.lib.ref_gpu_create(
            self.n, self.nb, *[k.ctypes.data_as(C.c_void_p) for k in keep],
            rb.ctypes.data_as(C.c_void_p), counts.ctypes.data_as(C.c_void_p),
            C.byref(L["prm"]), C.c_float(L["dt"]))
        if st != 0:
            raise RuntimeError(f"ref_gpu_create: {self.lib.ref_gpu_last_error().decode()}")

    def step(self) -> tuple[np.ndarray, float]:
        """One step; (per-stage GPU milliseconds, host wall milliseconds)."""
        ms = np.zeros(len(STAGES), np.float32)
        host = C.c_float(0)
        if self.lib.ref_gpu_step(ms.ctypes.data_as(C.c_void_p), C.byref(host)) != 0:
            raise RuntimeError(f"ref_gpu_step: {self.lib.ref_gpu_last_error().decode()}")
        return ms, host.value

    def bodies(self) -> tuple[np.ndarray, np.ndarray]:
        pos = np.zeros((self.nb, 4), np.float32)
        vel = np.zeros((self.nb, 4), np.float32)
        if self.lib.ref_gpu_download(pos.ctypes.data_as(C.c_void_p),
                                     vel.ctypes.data_as(C.c_void_p)) != 0:
            raise RuntimeError(f"ref_gpu_download: {self.lib.ref_gpu_last_error().decode()}")
        return pos, vel

    def close(self):
        self.lib.ref_gpu_destroy()
