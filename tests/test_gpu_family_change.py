"""Family changes on the GPU (deme_change_family, deme_set_family_change_rules) against the C oracle, whose steps
apply the same rules on the host between the forces and the integration (where the reference's routineChecks
applies them, src/DEM/dT.cpp:1434-1444).

* ChangeFamily moves every owner of a family at once; a fixed target family stops them.
* A position rule (spheres that fall below a height freeze) and a time rule, step by step and replayed from CUDA
  graphs: the families owner by owner, the contact lists and the positions equal the oracle's run.
* A rule that does not compile is refused with the compiler's log.
Like the reference, which replaces every `return` of a condition by an assignment, a condition should end in a
single `return <bool>;` (a second return would overwrite the first decision).
"""
import numpy as np
import pytest

from _util import canonical, capi, oracle, workloads
from deme_b200 import SceneBuilder

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

Z_FREEZE = 0.03  # from the domain's lower corner
T_SWITCH = 2.0e-4


def scene():
    """Spheres falling in a box; family 2 is fixed, family 3 moves at a prescribed velocity."""
    s = SceneBuilder()
    s.InstructBoxDomainDimension(0.1, 0.1, 0.2)
    s.SetCoordSysOrigin("center")
    mat = s.LoadMaterial({"E": 1e7, "nu": 0.3, "CoR": 0.5, "mu": 0.5, "Crr": 0.0})
    s.InstructBoxDomainBoundingBC("all", mat)
    r = 4e-3
    t = s.LoadSphereType(2600 * 4.18879 * r ** 3, r, mat)
    rng = np.random.default_rng(3)
    g = np.arange(6) * 2.3 * r - 5 * 1.15 * r
    X, Y, Z = np.meshgrid(g, g, np.arange(10) * 2.3 * r, indexing="ij")
    P = np.stack([X.ravel(), Y.ravel(), Z.ravel() - 0.1 + 1.2 * r], 1)
    P += rng.uniform(-0.1 * r, 0.1 * r, P.shape)
    b = s.AddClumps(t, P.astype(np.float32))
    b.SetVel(np.tile(np.array([[0.0, 0.0, -0.5]], np.float32), (len(P), 1)))
    s.SetFamilyFixed(2)
    s.SetFamilyPrescribedLinVel(3, "0", "0", "0.2")
    s.SetInitTimeStep(2e-5)
    s.SetGravitationalAcceleration((0, 0, -9.81))
    return s.Initialize()


RULES = [(0, 2, f"return pos.z < {Z_FREEZE};"),
         (0, 3, f"float z = (float)pos.z; return (t > {T_SWITCH}f) && (z > 0.07f);")]


def oracle_rules(built, st, t):
    """The rules in numpy, as the kernel evaluates them (pos from the kernel's voxel literals)."""
    pos = built.decode_positions(st, kernel_literals=True)
    fam = st["family"].copy()
    code = st["family"]
    n = built.info["n_clumps"]
    new = fam.copy()
    new[:n][(code[:n] == 0) & (pos[:n, 2] < Z_FREEZE)] = 2
    hit = (code[:n] == 0) & (np.float32(t) > np.float32(T_SWITCH)) & (pos[:n, 2].astype(np.float32) > np.float32(0.07))
    new[:n][hit] = 3
    return new


@pytest.mark.parametrize("graph", [False, True], ids=["step_by_step", "graph"])
def test_rules_match_the_oracle(graph):
    from deme_b200 import Solver
    built = scene()
    g = Solver(built)
    g.set_family_change_rules(RULES)
    if graph:
        g.set_graph(True)
    o = oracle(built)
    steps, t = 40, np.float32(0.0)
    h = np.float32(built.params.h)
    for chunk in range(4):
        g.step(steps // 4)
        for _ in range(steps // 4):
            o.detect_contacts()
            o.compute_forces()
            st = o.state()
            st["family"] = oracle_rules(built, st, t)
            o.set_state(st)
            o.integrate()
            t = np.float32(t + h)  # the reference's dT keeps the time as a float
        sg, so = g.state(), o.state()
        np.testing.assert_array_equal(sg["family"], so["family"], err_msg=f"chunk {chunk} families")
        cg, co = g.contacts(), canonical(o.contacts())
        for k in ("idA", "idB", "type"):
            np.testing.assert_array_equal(cg[k], co[k], err_msg=f"chunk {chunk} {k}")
        pg = built.decode_positions(sg, kernel_literals=False)
        po = built.decode_positions(so, kernel_literals=False)
        assert np.abs(pg - po).max() <= 1e-8, np.abs(pg - po).max()
    fam = g.state()["family"]
    assert (fam == 2).sum() > 0 and (fam == 3).sum() > 0 and (fam == 0).sum() > 0
    g.close()


def test_change_family_moves_a_whole_family():
    from deme_b200 import Solver
    built = scene()
    g = Solver(built)
    g.step(5)
    g.change_family(0, 2)
    fam = g.state()["family"]
    n = built.info["n_clumps"]
    assert np.all(fam[:n] == 2)
    p0 = built.decode_positions(g.state(), kernel_literals=False)[:n]
    g.step(10)
    p1 = built.decode_positions(g.state(), kernel_literals=False)[:n]
    # family 2 is fixed: positions only drift by the rounding of the voxel re-encoding each step (a few sub-voxel
    # units over 10 steps, as in the reference's integrator)
    assert np.abs(p1 - p0).max() <= 1e-9, np.abs(p1 - p0).max()
    g.close()


def test_rule_that_does_not_compile_is_refused():
    from deme_b200 import Solver
    from deme_b200.solver import DemeError
    g = Solver(scene())
    with pytest.raises(DemeError):
        g.set_family_change_rules([(0, 2, "return pos.q < 1;")])
    g.close()


def test_contact_between_families_toggled_on_a_running_solver():
    """DisableContactBetweenFamilies / EnableContactBetweenFamilies after Initialize (deme_set_family_contact): the
    next detection drops the pile's floor contacts and keeps its sphere pairs; enabled again, it finds the first
    list again, bit for bit (the state does not move in between)."""
    from deme_b200 import Solver
    built = workloads.sphere_pile(n=400, seed=5)
    fam_s, fam_w = int(built.arrays["family"][0]), int(built.arrays["family"][-1])
    g = Solver(built)
    g.step(3)
    g.detect_contacts()
    c0 = g.contacts()
    floor = c0["type"] == capi.SPHERE_PLANE_CONTACT
    assert floor.sum() > 20 and (~floor).sum() > 20
    g.DisableContactBetweenFamilies(fam_w, fam_s)
    g.detect_contacts()
    c1 = g.contacts()
    assert not np.any(c1["type"] == capi.SPHERE_PLANE_CONTACT)
    for k in ("idA", "idB", "type"):
        np.testing.assert_array_equal(c1[k], c0[k][~floor], err_msg=k)
    g.EnableContactBetweenFamilies(fam_s, fam_w)
    g.detect_contacts()
    c2 = g.contacts()
    for k in ("idA", "idB", "type"):
        np.testing.assert_array_equal(c2[k], c0[k], err_msg=k)
    g.close()
