"""AddPlate (DEMExternObj, src/DEM/BdrsAndObjs.h:152-170): the plate is flattened as a component of type
ANAL_OBJ_TYPE_PLATE with its half sizes, and, as in the reference (checkSphereEntityOverlap returns no contact for a
plate, src/kernel/DEMHelperKernels.cu:385-387, 439-441), it meets no sphere: a sphere pressed into it has no contact
in the oracle (the CUDA path shares the component test)."""
import numpy as np

from _util import oracle, capi
from deme_b200.scene import SceneBuilder


def test_plate_is_flattened_and_meets_no_sphere():
    s = SceneBuilder()
    s.InstructBoxDomainDimension(0.2, 0.2, 0.2)
    s.SetCoordSysOrigin("center")
    m = s.LoadMaterial({"E": 1e7, "nu": 0.3, "CoR": 0.5, "mu": 0.3, "Crr": 0.0})
    t = s.LoadSphereType(1e-4, 2e-3, m)
    s.AddClumps([t], np.array([[0.0, 0.0, 0.0015]], np.float32))
    w = s.AddExternalObject()
    w.AddPlate((0, 0, 0), (0, 0, 2), 0.04, 0.03, m)
    s.SetInitTimeStep(1e-5)
    s.SetExpandFactor(0.0)
    built = s.Initialize()
    a = built.arrays
    assert list(a["anal_type"]) == [capi.ANAL_PLATE]
    assert a["anal_size1"][0] == np.float32(0.02) and a["anal_size2"][0] == np.float32(0.015)
    assert a["anal_rotZ"][0] == np.float32(1.0)
    o = oracle(built, threads=1)
    o.detect_contacts()
    assert o.num_contacts() == 0
    o.close()
