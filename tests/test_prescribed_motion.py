"""Prescribed motions written as expressions of the time (SetFamilyPrescribedLinVel / AngVel / Position with strings
that are not constants, src/DEM/APIPublic.cpp:210-273), on the CPU.

* SceneBuilder keeps families whose strings are plain numbers in the constant table and hands every other family,
  with its strings and flags, to deme_set_prescribed_motion;
* the C oracle, given before each step the values the expressions take at that step's float time (tests/_util.py,
  shaker_motion), runs bit for bit with the reference's own integration kernel compiled for the CPU with the
  expression strings pasted in (oracle/_ref): this pins the evaluation the GPU tests use as their checker.
"""
import numpy as np
import pytest

from _util import oracle, reference, reference_available, set_oracle_motion, shaker_motion, workloads
from deme_b200 import SceneBuilder


def test_expression_families_leave_the_constant_table():
    built = workloads.shaker_box()
    motion = {m["family"]: m for m in built.info["motion_expressions"]}
    assert sorted(motion) == [1, 2, 3]
    assert motion[1]["lin_vel"] == ["0", "0", workloads.PISTON_VZ]
    assert motion[1]["lin_vel_prescribed"] and motion[1]["rot_vel_prescribed"]
    assert not motion[1]["lin_pos_prescribed"]
    assert motion[2]["lin_pos"] == [workloads.SLIDER_X, "none", "none"]
    assert motion[2]["lin_pos_prescribed"] and motion[2]["rot_pos_prescribed"]
    assert motion[3]["ang_vel"] == ["0", "0", workloads.SPINNER_WZ]
    assert not motion[3]["rot_vel_prescribed"]
    for fam in (1, 2, 3):
        assert built.prescriptions[fam].used == 0
    # the walls' fixed family stays a constant entry
    from deme_b200 import capi
    assert built.prescriptions[capi.RESERVED_FAMILY].used == 1


def test_constant_strings_stay_in_the_table():
    s = SceneBuilder()
    s.InstructBoxDomainDimension(0.1, 0.1, 0.1)
    mat = s.LoadMaterial({"E": 1e7, "nu": 0.3, "CoR": 0.5, "mu": 0.5, "Crr": 0.0})
    t = s.LoadSphereType(1e-3, 4e-3, mat)
    b = s.AddClumps(t, np.array([[0.0, 0.0, 0.0], [0.02, 0.0, 0.0]], np.float32))
    b.SetFamilies([4, 5])
    s.SetFamilyPrescribedLinVel(4, "0.5", "none", "-1e-2")
    s.SetFamilyPrescribedAngVel(5, "0", "0", "3.0 * t")
    s.SetInitTimeStep(1e-5)
    built = s.Initialize()
    assert [m["family"] for m in built.info["motion_expressions"]] == [5]
    e = built.prescriptions[4]
    assert e.used == 1 and list(e.has_vel) == [1, 0, 1]
    assert e.vel[0] == np.float32(0.5) and e.vel[2] == np.float32(-1e-2)
    assert built.prescriptions[5].used == 0


@pytest.mark.skipif(not reference_available(), reason="reference sources not mounted")
def test_stepwise_values_match_the_reference_expressions_bit_for_bit():
    built = workloads.shaker_box()
    ref, orc = reference(built), oracle(built)
    h = np.float32(built.params.h)
    t = np.float32(0.0)
    moved = {1: False, 2: False, 3: False}
    slider0 = None
    for step in range(40):
        set_oracle_motion(orc, shaker_motion(t))
        for s in (ref, orc):
            s.detect_contacts()
        cr, co = ref.contacts(), orc.contacts()
        for k in cr:
            np.testing.assert_array_equal(cr[k], co[k], err_msg=f"step {step} contacts {k}")
        for s in (ref, orc):
            s.compute_forces()
            s.integrate()
        sr, so = ref.state(), orc.state()
        for k in sr:
            np.testing.assert_array_equal(sr[k], so[k], err_msg=f"step {step} state {k}")
        fam = sr["family"]
        moved[1] |= bool(np.any(sr["vZ"][fam == 1] != 0))
        moved[3] |= bool(np.any(sr["omgZ"][fam == 3] != 0))
        slider = (sr["voxel"][fam == 2].copy(), sr["locX"][fam == 2].copy())
        if slider0 is None:
            slider0 = slider
        else:
            moved[2] |= bool(np.any(slider[0] != slider0[0]) or np.any(slider[1] != slider0[1]))
        t = np.float32(t + h)
    assert all(moved.values()), moved
    ref.close()
    orc.close()
