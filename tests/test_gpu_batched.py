"""Many independent scenes packed into one run (no reference counterpart): per-scene walls (each scene's spheres meet
only its own six planes), per-scene materials beyond 256 when needed, one launch per kernel for all scenes.

* The packed run against the C oracle on the same packed scene: contact lists bit-exact for several steps.
* The packed run against each scene run alone in the packed run's domain and slot (so positions encode on the same
  voxel grid and the search uses the same cells): the same contacts per scene after 30 steps and displacements
  within 1e-5 of the scene's largest displacement (the two runs differ only in the order of float sums).  A scene
  run in its own smaller box encodes positions on a finer grid; in these pressed lattices, contacts hovering at
  zero overlap then switch in one run and not the other, and the damping term (which grows as the fourth root of
  the overlap) makes such switches visible in the motion, so that comparison is not bitwise meaningful.
"""
import numpy as np
import pytest

from _util import canonical, capi, contact_key, oracle, workloads

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def small_specs(n=6):
    """Six small scenes whose spheres start in contact (pitch 1.98 r, bottom layer pressed into the floor)."""
    specs = workloads.batch_scene_specs(n, seed=9, n_range=(200, 800), r_range=(2e-3, 4e-3), side_range=(0.03, 0.06))
    for sp in specs:
        sp.update(pitch=1.98, lift=0.98)
    return specs


def test_packed_scenes_match_oracle_contact_lists():
    from deme_b200 import Solver
    built = workloads.batched_settling(small_specs())
    assert "owner_anal_first" in built.arrays and built.counts["a"] == 36
    g = Solver(built)
    o = oracle(built)
    for step in range(8):
        g.step(1)
        o.step(1)
        np.testing.assert_array_equal(contact_key(g.contacts()), contact_key(canonical(o.contacts())),
                                      err_msg=f"step {step}")
    assert g.num_contacts() > 100


def test_packed_run_equals_scenes_run_alone():
    from deme_b200 import Solver
    specs = small_specs()
    built = workloads.batched_settling(specs)
    g = Solver(built)
    p0 = built.decode_positions(built.initial_state(), kernel_literals=False)
    steps = 30
    g.step(steps)
    st = g.state()
    p1 = built.decode_positions(st, kernel_literals=False)
    c = g.contacts()
    for i, sp in enumerate(specs):
        first, n = built.info["scenes"][i]
        b1 = workloads.single_settling(sp, packed=built, index=i)
        s1 = Solver(b1)
        q0 = b1.decode_positions(b1.initial_state(), kernel_literals=False)
        s1.step(steps)
        q1 = b1.decode_positions(s1.state(), kernel_literals=False)
        d_packed = p1[first:first + n] - p0[first:first + n]
        d_alone = q1[:n] - q0[:n]
        bar = 1e-5 * np.abs(d_alone).max() + 1e-12
        assert np.abs(d_packed - d_alone).max() <= bar, (i, np.abs(d_packed - d_alone).max(), bar)
        c1 = s1.contacts()
        in_scene = (c["idA"] >= first) & (c["idA"] < first + n)
        assert in_scene.sum() == len(c1["idA"]), (i, in_scene.sum(), len(c1["idA"]))
        # the same list: packed ids shifted by the scene's first sphere, and by 6 planes per earlier scene
        ss = c["type"][in_scene] == capi.SPHERE_SPHERE_CONTACT
        np.testing.assert_array_equal(c["idA"][in_scene] - first, c1["idA"], err_msg=f"scene {i} idA")
        np.testing.assert_array_equal(np.where(ss, c["idB"][in_scene] - first, c["idB"][in_scene] - 6 * i), c1["idB"],
                                      err_msg=f"scene {i} idB")
        np.testing.assert_array_equal(c["type"][in_scene], c1["type"], err_msg=f"scene {i} type")
        s1.close()
