"""The C oracle against the reference's kernel sources compiled for the CPU (oracle/_ref), on fresh seeded scenes.

Runs only where the reference sources are mounted (skipped elsewhere); the golden fixtures carry the same check to
machines without them.
"""
import numpy as np
import pytest

from _util import oracle, reference, reference_available, workloads

pytestmark = pytest.mark.skipif(not reference_available(), reason="reference sources not mounted")

SCENES = {
    "clumps_dense": lambda: workloads.packed_clumps(n_clumps=300, seed=21, spacing=1.3),
    "spheres_masks": lambda: workloads.packed_clumps(n_clumps=500, seed=22, three=False, families=True, beta=5e-4),
    "settle": lambda: workloads.settling_box(n=600, r=5e-3, box=(0.08, 0.08, 0.12), spacing=1.99, jitter=0.03,
                                             seed=23, vel_scale=0.3, ang_scale=30.0),
}


@pytest.mark.parametrize("name", list(SCENES))
def test_oracle_bit_exact_vs_reference_cpu_build(name):
    built = SCENES[name]()
    ref, orc = reference(built), oracle(built)
    for step in range(5):
        for s in (ref, orc):
            s.detect_contacts()
        cr, co = ref.contacts(), orc.contacts()
        for k in cr:
            np.testing.assert_array_equal(cr[k], co[k], err_msg=f"{name} step {step} contacts {k}")
        if step == 0:
            br, bo = ref.bin_assignment(), orc.bin_assignment()
            for k in br:
                np.testing.assert_array_equal(br[k], bo[k], err_msg=f"{name} bins {k}")
        for s in (ref, orc):
            s.compute_forces()
        fr, fo = ref.contact_forces(), orc.contact_forces()
        for k in fr:
            np.testing.assert_array_equal(fr[k], fo[k], err_msg=f"{name} step {step} {k}")
        for s in (ref, orc):
            s.integrate()
        sr, so = ref.state(), orc.state()
        for k in sr:
            np.testing.assert_array_equal(sr[k], so[k], err_msg=f"{name} step {step} state {k}")
