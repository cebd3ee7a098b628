"""The frictionless Hertzian model (UseFrictionlessHertzianModel; the reference's FrictionlessHertzianForceModel.cu):
the normal spring and damper of the full model, no rolling resistance, no tangential force, no contact wildcards.
Pinned on the CPU through the oracle:

* a pile of spheres with friction and rolling resistance in its materials steps under the frictionless model exactly
  as the same pile under the full model with both coefficients zero (the full model's normal part is the
  frictionless model), bit for bit over 30 steps; with the coefficients kept, the full model differs;
* the scene carries no contact wildcards, and the per-contact forces are along the contact normals.
"""
import numpy as np

from _util import oracle, workloads
from oracle import fp64_model as M

KEYS = ("voxel", "locX", "locY", "locZ", "oriQw", "oriQx", "oriQy", "oriQz", "vX", "vY", "vZ", "omgX", "omgY", "omgZ")


def _run(built, steps=30):
    o = oracle(built, threads=1)
    o.step(steps)
    st, c = o.state(), o.contacts()
    o.close()
    return st, c


def test_frictionless_equals_full_model_without_friction_and_rolling():
    fl = workloads.sphere_pile(n=60, seed=3, frictionless=True)
    assert fl.params.n_contact_wildcards == 0
    nofr = workloads.sphere_pile(n=60, seed=3)
    nofr.arrays["mat_mu"][:] = 0.0
    nofr.arrays["mat_Crr"][:] = 0.0
    full = workloads.sphere_pile(n=60, seed=3)
    a, ca = _run(fl)
    b, cb = _run(nofr)
    d, _ = _run(full)
    for k in KEYS:
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)
    np.testing.assert_array_equal(ca["idA"], cb["idA"])
    assert any(not np.array_equal(a[k], d[k]) for k in ("omgX", "omgY", "omgZ"))


def test_frictionless_forces_are_normal():
    built = workloads.sphere_pile(n=60, seed=3, frictionless=True)
    o = oracle(built, threads=1)
    o.step(10)
    o.detect_contacts()
    o.compute_forces()
    c, f, st = o.contacts(), o.contact_forces(), o.state()
    o.close()
    assert len(c["idA"]) > 20 and c["wildcards"].shape[0] == 0
    F = f["force"].astype(np.float64)
    T = f["torque_only_force"].astype(np.float64)
    assert np.abs(T).max() == 0.0
    # a normal force applied at the contact point passes through sphere A's centre: no torque about it (the contact
    # point is given in A's frame; single spheres, so A's centre is its owner's)
    oA = built.arrays["sphere_owner"][c["idA"]]
    q = np.stack([st[k][oA] for k in ("oriQw", "oriQx", "oriQy", "oriQz")], 1).astype(np.float64)
    P = M.rot(q, f["cpA"].astype(np.float64))
    act = np.linalg.norm(F, axis=1) > 0
    cross = np.linalg.norm(np.cross(P[act], F[act]), axis=1)
    assert cross.max() <= 1e-5 * (np.linalg.norm(P[act], axis=1) * np.linalg.norm(F[act], axis=1)).max()
