"""The reference's own kernels on the GPU, behind the same Python interface as the oracle (HandleSolver).

TEST AND BASELINE INFRASTRUCTURE ONLY: used by the GPU parity tests as a checker and by the benchmark's reference
arm as the reference-kernel timing.  The cubins and the driver are built from the reference's sources by
``ref_gpu_build`` where those sources exist, and travel prebuilt under ``oracle/_ref/`` to machines where they do
not.
"""
from __future__ import annotations

import ctypes as C
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
for p in (os.path.join(ROOT, "dem-engine-sbel_b200"), HERE):
    if p not in sys.path:
        sys.path.insert(0, p)

import ref_gpu_build  # noqa: E402
from deme_b200 import capi  # noqa: E402
from deme_b200.solver import DemeError, HandleSolver  # noqa: E402


def prebuilt(built, fmad: bool = True) -> bool:
    return (os.path.exists(os.path.join(ref_gpu_build.cubin_dir(built, fmad), "kernels.txt"))
            and os.path.exists(ref_gpu_build.HARNESS_LIB))


class RefGPU(HandleSolver):
    """Runs a built scene with the reference's kernels (one stream; see ref_gpu_harness.cu)."""

    def __init__(self, built, fmad: bool = True, sync_each: bool = False):
        self._cubins = ref_gpu_build.build_cubins(built, fmad)
        self._sync_each = 1 if sync_each else 0
        lib = capi.load_library(ref_gpu_build.build_harness())
        lib.refg_get_error.restype = C.c_char_p
        lib.refg_get_error.argtypes = [C.c_void_p]
        lib.refg_time_steps.restype = C.c_int32
        lib.refg_time_steps.argtypes = [C.c_void_p, C.c_int32, C.POINTER(C.c_float)]
        lib.refg_sync.restype = C.c_int32
        lib.refg_sync.argtypes = [C.c_void_p]
        super().__init__(lib, "refg_", built)

    def _create(self, scene):
        fn = self.lib.refg_create
        fn.restype = C.c_int32
        fn.argtypes = [C.c_char_p, C.POINTER(capi.SimParams), C.POINTER(capi.Scene), C.c_int32,
                       C.POINTER(C.c_void_p)]
        h = C.c_void_p()
        st = fn(self._cubins.encode(), C.byref(self._params), C.byref(scene), self._sync_each, C.byref(h))
        if st != capi.DEME_OK:
            msg = self.lib.refg_get_error(h).decode() if h else ""
            if h:
                self.lib.refg_destroy(h)
            raise DemeError(f"refg_create: {capi.STATUS_NAMES.get(st, st)}: {msg}")
        return h

    def _check(self, st, what):
        if st != capi.DEME_OK:
            raise DemeError(f"refg_{what}: {capi.STATUS_NAMES.get(st, st)}: {self.lib.refg_get_error(self.h).decode()}")

    def sync(self):
        self._check(self.lib.refg_sync(self.h), "sync")

    def set_sync_each(self, on: bool):
        self.lib.refg_set_sync_each.argtypes = [C.c_void_p, C.c_int32]
        self.lib.refg_set_sync_each.restype = None
        self.lib.refg_set_sync_each(self.h, 1 if on else 0)

    def set_one_bin_per_thread(self, on: bool):
        """The reference's thread-per-bin contact kernels instead of its default block-per-bin ones."""
        self.lib.refg_set_one_bin_per_thread.argtypes = [C.c_void_p, C.c_int32]
        self.lib.refg_set_one_bin_per_thread.restype = None
        self.lib.refg_set_one_bin_per_thread(self.h, 1 if on else 0)

    PHASES = ("bins", "bin_sort", "active_bins", "pair_kernels", "contact_sort", "history_map", "handover_remap",
              "force_kernel", "force_collection", "integration")

    def profile_steps(self, n: int) -> dict:
        """Runs n steps with events at the phase boundaries; milliseconds per step of each phase."""
        out = (C.c_float * len(self.PHASES))()
        self.lib.refg_profile_steps.argtypes = [C.c_void_p, C.c_int32, C.POINTER(C.c_float)]
        self.lib.refg_profile_steps.restype = C.c_int32
        self._check(self.lib.refg_profile_steps(self.h, n, out), "profile_steps")
        return {k: float(v) / max(n, 1) for k, v in zip(self.PHASES, out)}

    def time_steps(self, n: int) -> float:
        """Device milliseconds of n steps (CUDA events on the driver's stream)."""
        ms = C.c_float()
        self._check(self.lib.refg_time_steps(self.h, n, C.byref(ms)), "time_steps")
        return float(ms.value)
