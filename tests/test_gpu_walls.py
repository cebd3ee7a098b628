"""Analytical cylinder and cone walls (no reference counterpart) and contact detection every few steps with a contact
margin, CUDA path against the C oracle.

The oracle's cylinder and cone follow the reference's plane conventions (contact when the signed gap is at most the
expanded radius plus the margin, overlap depth half the penetration, contact point mid-penetration), so these scenes
are pinned to the oracle only.  Bars as in test_gpu_parity: contact lists, partners and remapped history bit-exact;
per-contact forces within 1e-5 relative (floor 1e-6 of the largest); owner accelerations within 1e-5 of the sum of
contribution magnitudes; one-step velocities within 1e-5 relative, positions within 1e-9 m, quaternions within 1e-6.
"""
import numpy as np
import pytest

from _util import canonical, contact_key, oracle, partner_keys, workloads
from test_gpu_parity import gpu_solver, owner_scale

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

STATE_KEYS = ("voxel", "locX", "locY", "locZ", "oriQw", "oriQx", "oriQy", "oriQz", "vX", "vY", "vZ", "omgX", "omgY",
              "omgZ", "family")


def wall_scenes():
    return {
        # outer clumps start pressed into the rotating cylinder and the end planes
        "drum_walls": lambda: workloads.drum(n_clumps=700, seed=21, wall_clearance=0.7, spacing=0.8),
        # outer spheres start pressed into the cone; margin 0.15 mm
        "hopper_walls": lambda: workloads.hopper(n=1500, seed=22, wall_clearance=0.4),
    }


def lockstep(built, steps, name):
    """Each step: CD, forces, integration on both; compare; then give the GPU the oracle's state and history.
    Returns the contacts seen, counted by type."""
    g = gpu_solver(built)
    o = oracle(built)
    prev = None
    n_type = np.zeros(8, np.int64)
    for step in range(steps):
        g.detect_contacts()
        o.detect_contacts()
        oc = o.contacts()
        rc = canonical(oc)
        gc = g.contacts()
        for k in ("idA", "idB", "type"):
            np.testing.assert_array_equal(gc[k], rc[k], err_msg=f"{name} step {step} {k}")
        n_type += np.bincount(rc["type"], minlength=8)
        if prev is not None:
            np.testing.assert_array_equal(partner_keys(gc, prev), partner_keys(oc, prev_o)[rc["perm"]],
                                          err_msg=f"{name} step {step} partners")
        np.testing.assert_array_equal(gc["wildcards"], rc["wildcards"], err_msg=f"{name} step {step} history")
        g.compute_forces()
        o.compute_forces()
        gf, of = g.contact_forces(), o.contact_forces()
        of = {k: v[rc["perm"]] for k, v in of.items()}
        active = np.any(of["force"] != 0, axis=1)
        for k in ("force", "torque_only_force", "cpA", "cpB"):
            a, b = gf[k][active].astype(np.float64), of[k][active].astype(np.float64)
            floor = 1e-6 * max(np.abs(b).max(initial=0), 1e-30)
            err = np.abs(a - b) / (np.abs(b) + floor)
            assert err.max(initial=0) <= 1e-5, f"{name} step {step} {k} rel err {err.max()}"
        gs, os_ = g.state(), o.state()
        scale = owner_scale(built, {k: rc[k] for k in ("idA", "idB", "type")}, of)
        for k in ("aX", "aY", "aZ"):
            d = np.abs(gs[k].astype(np.float64) - os_[k].astype(np.float64))
            assert np.all(d <= 1e-5 * scale + 1e-30), f"{name} step {step} {k}"
        g.integrate()
        o.integrate()
        gs, os_ = g.state(), o.state()
        for k in ("vX", "vY", "vZ", "omgX", "omgY", "omgZ"):
            a, b = gs[k].astype(np.float64), os_[k].astype(np.float64)
            assert np.all(np.abs(a - b) <= 1e-5 * np.abs(b) + 1e-5 * np.abs(b).max() + 1e-12), f"{name} {k}"
        pg, po = built.decode_positions(gs), built.decode_positions(os_)
        assert np.abs(pg - po).max() <= 1e-9, f"{name} step {step} position diff {np.abs(pg - po).max()}"
        for k in ("oriQw", "oriQx", "oriQy", "oriQz"):
            assert np.abs(gs[k] - os_[k]).max() <= 1e-6, f"{name} step {step} {k}"
        # same input for the next step
        oc_post = o.contacts()
        g.set_state({k: os_[k] for k in STATE_KEYS})
        g.set_contacts({"idA": oc_post["idA"], "idB": oc_post["idB"], "type": oc_post["type"],
                        "wildcards": oc_post["wildcards"]})
        prev = {k: rc[k] for k in ("idA", "idB", "type")}
        prev_o = {k: oc[k] for k in ("idA", "idB", "type")}
    return n_type


@pytest.mark.parametrize("name", sorted(wall_scenes()))
def test_gpu_curved_walls_match_oracle_lockstep(name):
    built = wall_scenes()[name]()
    n_type = lockstep(built, 4, name)
    assert n_type[5:7].sum() > 0, "the scene must exercise cylinder or cone contacts"


def test_gpu_contact_margin_every_5_steps_matches_oracle():
    """Free-running hopper with contact detection every 5 steps and a 0.15 mm margin: the lists (computed on steps
    0, 5, 10) stay bit-identical and the kinetic energy agrees to 1e-4."""
    built = workloads.hopper(n=1500, seed=23, wall_clearance=0.4)
    assert built.params.cd_update_freq == 5 and built.params.beta > 0
    g = gpu_solver(built, keep=False)
    o = oracle(built)
    for step in range(12):
        g.step(1)
        o.step(1)
        if step < 6:
            np.testing.assert_array_equal(contact_key(g.contacts()), contact_key(canonical(o.contacts())),
                                          err_msg=f"step {step}")
    ke_g, ke_o = g.kinetic_energy(), o.kinetic_energy()
    assert abs(ke_g - ke_o) <= 1e-4 * abs(ke_o), (ke_g, ke_o)
