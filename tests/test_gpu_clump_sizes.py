"""ChangeClumpSizes on a running solver (deme_change_clump_sizes; the reference scales the component spheres'
relative positions and radii of the listed clumps, DEMMiscKernels.cu:4-52): the CUDA path and the C oracle resize
the same clumps of a dense three-sphere clump pack between steps and then find the same contact lists, bit for bit,
step after step.  Growing some clumps raises the largest radius (coarser search cells); shrinking all of them by 0.85
lowers it below its value at creation, so the search grid gets more cells than its arrays were sized for and they
grow."""
import numpy as np
import pytest

from _util import canonical, contact_key, oracle, workloads
from test_gpu_parity import gpu_solver

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.mark.parametrize("case", ["grow_some", "shrink_all"])
def test_gpu_resized_clumps_match_oracle(case):
    built = workloads.packed_clumps(n_clumps=300, seed=7, spacing=1.35)
    g, o = gpu_solver(built, keep=False), oracle(built)
    g.step(2)
    o.step(2)
    if case == "grow_some":
        owners = np.arange(0, 300, 3, dtype=np.uint32)
        factors = np.linspace(0.8, 1.3, len(owners)).astype(np.float32)
    else:
        owners = np.arange(300, dtype=np.uint32)
        factors = np.full(300, 0.85, np.float32)
    g.change_clump_sizes(owners, factors)
    o.change_clump_sizes(owners, factors)
    for step in range(4):
        g.step(1)
        o.step(1)
        np.testing.assert_array_equal(contact_key(g.contacts()), contact_key(canonical(o.contacts())),
                                      err_msg=f"{case} step {step}")
    ke_g, ke_o = g.kinetic_energy(), o.kinetic_energy()
    assert abs(ke_g - ke_o) <= 1e-4 * abs(ke_o), (ke_g, ke_o)
    g.close()
    o.close()
