"""Sphere--mesh contacts (triangle facets of mesh-represented owners), CUDA path against the C oracle.

The reference loads mesh bodies (DEMMeshConnected) and declares the sphere--mesh contact type but detects no such
contact, so these scenes are pinned to the oracle's restatement only (closest point on the facet by Ericson's region
tests; the plane's conventions for depth, normal and contact point).  Bars as in test_gpu_walls: contact lists,
partners and remapped history bit-exact; per-contact forces within 1e-5 relative; owner accelerations within 1e-5
of the sum of contribution magnitudes; one-step velocities within 1e-5 relative, positions within 1e-9 m.

* a square funnel of 160 facets (walls and floor on 4 x 4 grids of split quads) with 1500 spheres pressed into it:
  contacts on facet interiors, edges and corners, a fixed mesh owner;
* a free icosphere of 1280 facets driven into a bed of 2000 spheres inside analytical planes: a moving, rotating
  mesh owner whose reactions are collected and integrated;
* the drum of 700 clumps with its cylinder as 1664 facets turning at 20 rpm: a mesh owner with prescribed rotation;
* the conical hopper of 1500 log-normal spheres with its cone as 2304 facets;
* a floor of two large facets against the same floor as an analytical plane: the same contacts, forces equal to
  float rounding;
* 1,600 spheres in one layer on a two-facet floor: more sphere--mesh pairs than the mesh pool first holds, so the
  search grows the pool and runs again; the list equals the oracle's;
* detection on the kT stream (two streams, lag 2): the adopted list is the oracle's detection on the snapshot;
* scope: packed scenes and the adjoint refuse meshes; graph replay falls back to plain steps.
"""
import numpy as np
import pytest

from _util import canonical, contact_key, oracle, workloads, capi
from test_gpu_parity import gpu_solver
from test_gpu_walls import lockstep

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def mesh_scenes():
    return {
        "funnel_fixed_mesh": lambda: workloads.mesh_funnel(n=1500, seed=31, wall_clearance=0.8),
        "ball_drop_free_mesh": lambda: workloads.mesh_ball_drop(n=2000, seed=32, press=0.2),
        # the drum's cylinder as 1664 facets turning with the end planes (prescribed rotation); outer clumps pressed in
        "drum_turning_mesh_cylinder": lambda: workloads.drum(n_clumps=700, seed=21, wall_clearance=0.7, spacing=0.8,
                                                             mesh=True),
        # the conical hopper's cone as 2304 fixed facets, polydisperse spheres pressed into it
        "hopper_mesh_cone": lambda: workloads.hopper(n=1500, seed=22, wall_clearance=0.4, mesh=True),
    }


@pytest.mark.parametrize("name", sorted(mesh_scenes()))
def test_gpu_mesh_contacts_match_oracle_lockstep(name):
    built = mesh_scenes()[name]()
    n_type = lockstep(built, 4, name)
    assert n_type[capi.SPHERE_MESH_CONTACT] > 20, n_type


def test_gpu_free_running_ball_drop_matches_oracle():
    """200 free steps of the ball drop (detection every step): the lists of the first 20 steps stay bit-identical,
    the ball's velocity and the kinetic energy agree to 1e-4 at the end."""
    built = workloads.mesh_ball_drop(n=2000, seed=33, press=0.1)
    g = gpu_solver(built, keep=False)
    o = oracle(built)
    for step in range(200):
        g.step(1)
        o.step(1)
        if step < 20:
            np.testing.assert_array_equal(contact_key(g.contacts()), contact_key(canonical(o.contacts())),
                                          err_msg=f"step {step}")
    gs, os_ = g.state(), o.state()
    vb_g = np.array([gs[k][-1] for k in ("vX", "vY", "vZ")], np.float64)
    vb_o = np.array([os_[k][-1] for k in ("vX", "vY", "vZ")], np.float64)
    assert np.abs(vb_g - vb_o).max() <= 1e-4 * np.abs(vb_o).max(), (vb_g, vb_o)
    ke_g, ke_o = g.kinetic_energy(), o.kinetic_energy()
    assert abs(ke_g - ke_o) <= 1e-4 * abs(ke_o), (ke_g, ke_o)
    assert np.any(g.contacts()["type"] == capi.SPHERE_MESH_CONTACT)
    g.close()
    o.close()


def _pile(mesh_floor: bool):
    """sphere_pile's 400 spheres on its floor, an analytical plane or two facets 0.19 m wide in the same plane."""
    return workloads.sphere_pile(n=400, seed=5, mesh_floor=mesh_floor)


def test_gpu_mesh_floor_equals_analytical_plane():
    plane, mesh = _pile(False), _pile(True)
    gp, gm = gpu_solver(plane), gpu_solver(mesh)
    ever_double = np.zeros(0, np.int64)
    for step in range(3):
        gp.detect_contacts()
        gm.detect_contacts()
        cp, cm = gp.contacts(), gm.contacts()
        wall_p = cp["type"] == capi.SPHERE_PLANE_CONTACT
        wall_m = cm["type"] == capi.SPHERE_MESH_CONTACT
        assert wall_p.sum() > 20
        # a sphere over the shared diagonal touches both facets: compare the spheres that touch one
        idA_m, cnt = np.unique(cm["idA"][wall_m], return_counts=True)
        ever_double = np.union1d(ever_double, idA_m[cnt > 1])
        single = np.setdiff1d(idA_m[cnt == 1], ever_double)
        assert len(single) > 20
        np.testing.assert_array_equal(np.unique(cp["idA"][wall_p]), idA_m)
        np.testing.assert_array_equal(cp["idA"][~wall_p], cm["idA"][~wall_m])
        np.testing.assert_array_equal(cp["idB"][~wall_p], cm["idB"][~wall_m])
        gp.compute_forces()
        gm.compute_forces()
        fp, fm = gp.contact_forces(), gm.contact_forces()
        ip = np.nonzero(wall_p & np.isin(cp["idA"], single))[0]
        im = np.nonzero(wall_m & np.isin(cm["idA"], single))[0]
        for k in ("force", "torque_only_force", "cpA"):
            a, b = fm[k][im].astype(np.float64), fp[k][ip].astype(np.float64)
            scale = np.abs(b).max() + 1e-30
            assert np.abs(a - b).max() <= 1e-5 * scale, (step, k, np.abs(a - b).max(), scale)
        gp.integrate()
        gm.integrate()
        sm = gm.state()
        gp.set_state({k: sm[k][:plane.counts["o"]] for k in ("voxel", "locX", "locY", "locZ", "oriQw", "oriQx",
                                                               "oriQy", "oriQz", "vX", "vY", "vZ", "omgX", "omgY",
                                                               "omgZ")})
    gp.close()
    gm.close()


def test_gpu_mesh_detection_on_the_kt_stream_is_the_detection_on_the_snapshot():
    """kT and dT on two streams (deme_set_async_cd, lag 2, detection every 4 steps, margin 0.1 mm): the list dT
    adopts is the oracle's detection on the poses of the detection step, mesh facets placed from kT's snapshot."""
    from deme_b200 import Solver
    built = workloads.mesh_ball_drop(n=2000, seed=35, press=0.2, cd_freq=4, margin=1e-4)
    f, lag = 4, 2
    g = Solver(built)
    g.set_async_cd(lag)
    snaps, checked, n_mesh = {}, 0, 0
    for s in range(3 * f + lag + 1):
        if s % f == 0:
            snaps[s] = g.state()
        g.step(1)
        src = 0 if s == 0 else (s - lag if s - lag >= f and (s - lag) % f == 0 else None)
        if src is None:
            continue
        o = oracle(built)
        o.set_state(snaps[src])
        o.detect_contacts()
        oc = canonical(o.contacts())
        gc = g.contacts()
        np.testing.assert_array_equal(contact_key(gc), contact_key(oc), err_msg=f"step {s} (poses of step {src})")
        n_mesh += int(np.sum(gc["type"] == capi.SPHERE_MESH_CONTACT))
        checked += 1
        o.close()
    assert checked >= 3 and n_mesh > 0
    g.close()


def test_gpu_mesh_pool_grows():
    from deme_b200.scene import SceneBuilder
    r = 2e-3
    s = SceneBuilder()
    s.InstructBoxDomainDimension(0.4, 0.4, 0.4)
    s.SetCoordSysOrigin("center")
    m = s.LoadMaterial({"E": 1e7, "nu": 0.3, "CoR": 0.5, "mu": 0.3, "Crr": 0.0})
    t = s.LoadSphereType(1e-4, r, m)
    g = (np.arange(40) - 19.5) * 2.1 * r
    X, Y = np.meshgrid(g, g, indexing="ij")
    z0 = -0.05
    xyz = np.stack([X.ravel(), Y.ravel(), np.full(X.size, z0 + 0.95 * r)], 1).astype(np.float32)
    s.AddClumps([t] * len(xyz), xyz)
    w = 0.15
    v = np.array([[-w, -w, z0], [w, -w, z0], [w, w, z0], [-w, w, z0]], np.float32)
    s.AddWavefrontMeshObject((v, np.array([[0, 1, 2], [0, 2, 3]])), m)
    s.SetInitTimeStep(1e-5)
    s.SetCDUpdateFreq(1)
    s.SetExpandFactor(0.0)
    built = s.Initialize()
    gs, o = gpu_solver(built, keep=False), oracle(built)
    gs.detect_contacts()
    o.detect_contacts()
    gc = gs.contacts()
    assert np.sum(gc["type"] == capi.SPHERE_MESH_CONTACT) >= 1600
    np.testing.assert_array_equal(contact_key(gc), contact_key(canonical(o.contacts())))
    gs.close()
    o.close()


def test_gpu_mesh_scope():
    from deme_b200 import Solver, adjoint
    from deme_b200.scene import SceneBuilder
    from deme_b200.solver import DemeError
    # packed scenes (per-batch search grids) and meshes do not mix
    s = SceneBuilder()
    s.InstructBoxDomainDimension(0.2, 0.2, 0.2)
    s.SetCoordSysOrigin("center")
    m = s.LoadMaterial({"E": 1e7, "nu": 0.3, "CoR": 0.5, "mu": 0.3, "Crr": 0.0})
    t = s.LoadSphereType(1e-4, 2.5e-3, m)
    s.AddClumps([t] * 8, np.random.default_rng(0).uniform(-0.02, 0.02, (8, 3)).astype(np.float32)).SetSceneBox(
        (-0.05, -0.05, -0.05), (0.05, 0.05, 0.05))
    s.AddWavefrontMeshObject((np.eye(3, dtype=np.float32) * 0.01, np.array([[0, 1, 2]])), m)
    s.SetInitTimeStep(1e-5)
    with pytest.raises(DemeError, match="mesh facets are not supported together with packed scenes"):
        Solver(s.Initialize())
    built = workloads.mesh_funnel(n=300, seed=34, wall_clearance=0.9)
    g = Solver(built)
    with pytest.raises(DemeError, match="INVALID.*mesh"):
        adjoint.record(g, 2, 1)
    # graph replay is requested but mesh scenes step plainly: the same lists as plain steps
    h = Solver(built)
    g.set_graph(True)
    g.step(10)
    h.step(10)
    np.testing.assert_array_equal(contact_key(g.contacts()), contact_key(h.contacts()))
    assert g.graph_stats()[0] == 0
    g.close()
    h.close()
