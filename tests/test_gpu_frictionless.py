"""The frictionless Hertzian model on the GPU (UseFrictionlessHertzianModel: the built-in model with no contact
wildcards runs its normal part only), against the C oracle's frictionless model in lockstep: contact lists and
partners bit-exact, per-contact forces within 1e-5 relative, one-step states as in test_gpu_walls.  The adjoint
refuses the model (it differentiates the full one)."""
import numpy as np
import pytest

from _util import capi, workloads
from test_gpu_walls import lockstep

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def test_gpu_frictionless_model_matches_oracle_lockstep():
    built = workloads.sphere_pile(n=400, seed=5, frictionless=True)
    assert built.params.n_contact_wildcards == 0
    n_type = lockstep(built, 6, "frictionless_pile")
    assert n_type[capi.SPHERE_SPHERE_CONTACT] > 20 and n_type[capi.SPHERE_PLANE_CONTACT] > 20, n_type


def test_gpu_frictionless_forces_have_no_tangential_part():
    from test_gpu_parity import gpu_solver
    built = workloads.sphere_pile(n=400, seed=5, frictionless=True)
    g = gpu_solver(built)
    g.step(5)
    g.detect_contacts()
    g.compute_forces()
    f = g.contact_forces()
    assert np.abs(f["torque_only_force"]).max() == 0.0 and np.abs(f["force"]).max() > 0.0
    g.close()


def test_gpu_frictionless_model_is_refused_by_the_adjoint():
    from deme_b200 import Solver, adjoint
    from deme_b200.solver import DemeError
    g = Solver(workloads.sphere_pile(n=60, seed=3, frictionless=True))
    with pytest.raises(DemeError, match="INVALID.*frictionless"):
        adjoint.record(g, 2, 1)
    g.close()
