"""Host side of the reference-kernel GPU build (oracle/ref_gpu_build.py, oracle/ref_gpu_harness.cu), no GPU needed:
the cubin key, the prebuilt cubins of the parity scenes and the driver's exported entry points."""
import ctypes as C
import os

import numpy as np
import pytest

from _util import workloads

from oracle import ref_gpu_build  # noqa: E402

REF = ref_gpu_build.available()


def test_scene_key_reads_only_what_the_substitution_reads():
    a = workloads.settling_box(n=300, seed=1)
    b = workloads.settling_box(n=300, seed=2)  # other positions, same world and materials
    assert ref_gpu_build.scene_key(a) == ref_gpu_build.scene_key(b)
    assert ref_gpu_build.scene_key(a, fmad=True) != ref_gpu_build.scene_key(a, fmad=False)
    c = workloads.settling_box(n=300, seed=1)
    c.arrays["mat_E"] = np.asarray(c.arrays["mat_E"]) * 2
    assert ref_gpu_build.scene_key(c) != ref_gpu_build.scene_key(a)


@pytest.mark.skipif(not REF, reason="reference sources not mounted")
def test_parity_scene_cubins_hold_every_kernel():
    for name in ref_gpu_build.PARITY_SCENES:
        d = ref_gpu_build.build_cubins(ref_gpu_build.parity_scene(name), fmad=False)
        with open(os.path.join(d, "kernels.txt")) as f:
            rows = [line.split() for line in f if line.strip()]
        have = {(r[0], r[1]) for r in rows}
        for prog, kernels in ref_gpu_build.PROGRAMS.items():
            assert os.path.getsize(os.path.join(d, prog + ".cubin")) > 0
            for k in kernels:
                assert (prog, k) in have, (name, prog, k)


@pytest.mark.skipif(not (REF or os.path.exists(ref_gpu_build.HARNESS_LIB)), reason="driver not built")
def test_driver_loads_and_exports_its_entry_points():
    lib = C.CDLL(ref_gpu_build.build_harness())
    for sym in ("refg_create", "refg_destroy", "refg_get_error", "refg_detect_contacts", "refg_compute_forces",
                "refg_integrate", "refg_step", "refg_time_steps", "refg_profile_steps", "refg_sync",
                "refg_num_contacts", "refg_download_contacts", "refg_download_contact_forces", "refg_download_state",
                "refg_upload_state", "refg_set_sync_each", "refg_set_one_bin_per_thread"):
        assert hasattr(lib, sym), sym
