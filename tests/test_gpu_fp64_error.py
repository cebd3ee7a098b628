"""The CUDA path's error against an FP64 evaluation of the reference's arithmetic (oracle/fp64_model.py): per-contact
forces and one-step state updates, measured on the golden scenes, the 20k-clump shell drum, the 20k-clump drum with
its analytical cylinder and a 20k-sphere hopper with its cone.

From one state (after a few free steps, so that contacts carry history), the CUDA path detects contacts, computes
forces and integrates one step; the FP64 model takes the same state and the same contact list with its history.

* Forces: over the whole list (norm of all differences over the norm of all forces) within 1e-5; per contact
  (vector difference over the contact's own force) the distribution is printed and 99 % of the contacts are
  within 1e-4.  Where the normal spring and damper nearly cancel (contacts about to separate) FP32 arithmetic
  loses most digits of the small remainder, so single contacts can differ by far more.
* One-step updates: over all owners (norm of the differences over the norm of the FP64 values) within 1e-6 for
  velocities and 5e-3 for angular velocities, which collect the torques of those cancelling contacts and the
  rolling-resistance torque, whose direction is that of the relative rolling velocity and turns freely where that
  velocity is near zero; quaternions within 1e-6; the position change of the step within 1e-3 over all owners
  (the CUDA path encodes positions on the reference's voxel grid, truncating to the sub-voxel step, and an owner's
  acceleration error enters its position as h^2 / 2 times that error).  The largest owner's errors are printed.

The CUDA path's forces are bit-identical to the reference's kernels built with FMA contraction off (see
test_gpu_reference_kernels.py), so these numbers are also the reference's own FP32 error against FP64.
"""
import numpy as np
import pytest

from _util import load_golden, workloads
from oracle import fp64_model as M

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

SCENES = {
    "golden_clumps_planes": lambda: load_golden("clumps_planes")[0],
    "golden_spheres_families": lambda: load_golden("spheres_families")[0],
    "golden_settle_small": lambda: load_golden("settle_small")[0],
    "drum_shell_20k": lambda: workloads.drum(20000, shell=True, spacing=0.745),
    "drum_cylinder_20k": lambda: workloads.drum(20000, spacing=0.745, wall_clearance=0.6),
    "hopper_cone_20k": lambda: workloads.hopper(n=20000, seed=5, cd_freq=1, wall_clearance=0.7),
}


def _rel_vec(a, b, floor):
    return np.linalg.norm(a - b, axis=1) / (np.linalg.norm(b, axis=1) + floor)


@pytest.mark.parametrize("name", sorted(SCENES))
def test_cuda_step_against_fp64(name):
    from deme_b200 import Solver
    built = SCENES[name]()
    g = Solver(built)
    g.keep_contact_forces(True)
    g.step(5)
    st0 = g.state()
    g.detect_contacts()
    c = g.contacts()
    g.compute_forces()
    f = g.contact_forces()
    g.integrate()
    st1 = g.state()
    r = M.step(built, st0, c)
    act = r["active"]
    np.testing.assert_array_equal(np.any(f["force"] != 0, axis=1), act, err_msg="contacts carrying a force")
    a, b = f["force"][act].astype(np.float64), r["force"][act]
    whole = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)
    floor = 1e-6 * max(np.linalg.norm(b, axis=1).max(initial=0), 1e-300)
    per = _rel_vec(a, b, floor)
    assert whole <= 1e-5, whole
    q99 = float(np.quantile(per, 0.99)) if per.size else 0.0
    q999 = float(np.quantile(per, 0.999)) if per.size else 0.0
    assert q99 <= 1e-4, q99
    # one-step updates
    def vec(st, keys):
        return np.stack([st[k] for k in keys], 1).astype(np.float64)
    v1, w1 = vec(st1, ("vX", "vY", "vZ")), vec(st1, ("omgX", "omgY", "omgZ"))
    q1 = vec(st1, ("oriQw", "oriQx", "oriQy", "oriQz"))
    errs = {}
    for key, got, want, bar in (("vel", v1, r["vel"], 1e-6), ("angvel", w1, r["angvel"], 5e-3)):
        fl = 1e-6 * max(np.linalg.norm(want, axis=1).max(initial=0), 1e-300)
        errs[key] = float(_rel_vec(got, want, fl).max(initial=0))
        errs[key + "_all"] = float(np.linalg.norm(got - want) / max(np.linalg.norm(want), 1e-300))
        assert errs[key + "_all"] <= bar, (key, errs[key + "_all"])
    errs["quat"] = float(np.abs(q1 - r["quat"]).max(initial=0))
    assert errs["quat"] <= 1e-6, errs["quat"]
    p1 = built.decode_positions(st1)
    dpos = np.abs(p1 - r["pos"]).max(initial=0)
    l = float(built.params.l_kernel)
    moved = np.linalg.norm(r["pos"] - r["pos0"])
    errs["pos_all"] = float(np.linalg.norm(p1 - r["pos"]) / max(moved, 1e-300))
    assert errs["pos_all"] <= 1e-3, (errs["pos_all"], dpos, l)
    print(f"{name}: {len(c['idA'])} contacts ({int(act.sum())} touching); forces against FP64: {whole:.1e} over the "
          f"list, per contact median {np.median(per) if per.size else 0:.1e}, 99 % {q99:.1e}, 99.9 % {q999:.1e}, "
          f"largest {per.max(initial=0):.1e}; one step over all owners / largest owner: velocity {errs['vel_all']:.1e}"
          f" / {errs['vel']:.1e}, angular velocity {errs['angvel_all']:.1e} / {errs['angvel']:.1e}, quaternion "
          f"{errs['quat']:.1e}, position change {errs['pos_all']:.1e} / {dpos:.1e} m (sub-voxel step {l:.1e} m)")
    g.close()
