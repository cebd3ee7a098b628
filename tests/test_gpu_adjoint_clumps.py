"""CUDA adjoint (deme_adjoint_record / deme_adjoint_backward) on clumps and analytical walls.

The loss is sum wx . position + wv . velocity + ww . world angular velocity + wq . quaternion over the free owners,
exact derivatives (floors 0).  Compared: the material gradients (E, CoR, mu, Crr) and the initial-state gradients
(position, velocity, world angular velocity, quaternion at fixed world angular velocity).

* Against the FP64 host adjoint (oracle/fp64_autograd.py) along the trajectory the CUDA run recorded: the same
  construction -- each step's derivative at the recorded state, contact list and incoming histories, the history
  map reversed -- in FP64 by torch's reverse mode.  Both evaluate the same derivatives at the same points, so the
  bars are tight: 1e-4 of the largest material gradient, 1e-4 of the largest gradient of each state group over
  all free owners.  Scenes, 24 steps with checkpoints every 10 (three recomputed segments, histories carried
  across them): a drum of 150 three-sphere clumps turning at 20 rpm (analytical cylinder and two end planes of a
  driven family, settled for 25000 steps: sliding and rolling contacts with history; the drum's quaternion has
  drifted off unit length, so its walls' directions are not quite unit, as in the forward step), a conical hopper
  of 300 spheres (cone, gate and floor planes, 25000 steps into the fill) and a dense pack of 100 clumps (fresh
  contacts).
* Against central differences of the FP64 forward (tests/_adjoint_fd.py) over windows of 15 steps, where the CUDA
  adjoint runs on the FP32 trajectory and the differences on the FP64 one.  Coulomb sliding at the cap and
  rolling-resistance directions are non-smooth, and where contacts sit at those points the two trajectories pick
  different sides within a few steps, so these windows are frictionless: the turning clump drum and a loose clump
  pack; the drum is settled on the C oracle (25,500 steps), so the window is the same in every run.  Central
  differences at two step sizes are compared where they agree.  Bars: 5e-3 of the largest material
  gradient, 1e-2 of the largest gradient of each state group.
* Scope: a clump family with only its linear velocity prescribed, and a wall whose family has no prescription (it
  would move under the contact forces), are refused with DEME_ERR_INVALID and the reason.
"""
import numpy as np
import pytest

import _adjoint_fd as F
from _util import oracle, workloads
from oracle import fp64_autograd as AG
from oracle import fp64_model as M

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _drum(**kw):
    return workloads.drum(n_clumps=150, fill=0.2, wall_clearance=0.8, **kw)


def _hopper():
    return workloads.hopper(n=300, seed=5, cd_freq=1, wall_clearance=0.7)


def _frictionless(built):
    built.arrays["mat_mu"][:] = 0.0
    built.arrays["mat_Crr"][:] = 0.0
    return built


HOST = {
    "drum_clumps_cylinder_turning": (_drum, 25000),
    "hopper_spheres_cone": (_hopper, 25000),
    "packed_clumps_fresh": (lambda: workloads.packed_clumps(n_clumps=100, seed=7, spacing=1.35), 0),
}
T_HOST, K_HOST = 24, 10
# settled on the C oracle, so that the window is the same in every run (a contact whose overlap passes through zero
# inside the window makes the damping term's derivative unbounded there, and the FP32 and FP64 trajectories then
# differ in the derivative they see; a settle on the GPU would give a different window each run)
WINDOW = {
    "drum_clumps_cylinder_turning_frictionless": (lambda: _frictionless(_drum()), 25500),
    "packed_clumps_frictionless": (lambda: _frictionless(workloads.packed_clumps(
        n_clumps=100, seed=7, spacing=1.45, vel_scale=0.02, ang_scale=2.0)), 0),
}
T_WINDOW, K_WINDOW = 15, 6


def _run(make, settle, T, K, settle_on_oracle=False):
    """Settles (on the GPU, or on the C oracle and then uploaded), runs the CUDA adjoint over T steps, then the same
    T steps again keeping each step's contact list and state."""
    from deme_b200 import Solver, adjoint
    built = make()
    g = Solver(built)
    adjoint.set_floors(g, 0.0, 0.0, 0.0)
    if settle and settle_on_oracle:
        o = oracle(built, threads=4)
        o.step(settle)
        so, co = o.state(), o.contacts()
        o.close()
        g.set_state({k: v for k, v in so.items() if not k.startswith("a")})
        g.set_contacts({k: co[k] for k in ("idA", "idB", "type", "wildcards")})
    elif settle:
        g.step(settle)
    st0 = {k: v for k, v in g.state().items() if not k.startswith("a")}
    c0 = {k: np.array(v, copy=True) for k, v in g.contacts().items() if k in ("idA", "idB", "type", "wildcards")}
    nO = built.counts["o"]
    free = AG.free_owners(built, st0["family"])
    wts = F.weights(nO, free)
    g.set_contacts(c0)
    adjoint.record(g, T, K)
    st_rec = g.state()
    out = adjoint.backward(g, d_pos=wts[0], d_vel=wts[1], d_angvel=wts[2], d_quat=wts[3])
    g.set_state(st0)
    g.set_contacts(c0)
    lists, states = F.record_lists(g, T, built)
    st1 = g.state()
    g.close()
    # the same window twice: equal up to the order of the float atomics that collect the forces on B sides
    for k in ("vX", "vY", "vZ", "omgX", "omgY", "omgZ", "oriQw", "oriQx", "oriQy", "oriQz"):
        a, b = st_rec[k].astype(np.float64), st1[k].astype(np.float64)
        assert np.abs(a - b).max() <= 1e-5 * max(np.abs(b).max(), 1e-30), k
    mats = {k: v.astype(np.float32).astype(np.float64) for k, v in F.materials(built).items()}
    return dict(built=built, out=out, states=states, lists=lists, wts=wts, free=free, mats=mats)


def _report(name, r, ref, mat_bar, state_bar, owners=None, converged=None):
    out, free = r["out"], r["free"]
    sel = np.nonzero(free)[0] if owners is None else owners
    res = {}
    for k in ("pos", "vel", "angvel", "quat"):
        a, b = out["d_" + k + "0"][sel], ref[k]
        ok = np.ones(b.shape, bool) if converged is None else converged[k]
        res[k] = float((np.abs(a - b) * ok).max() / max(np.abs(b).max(), 1e-300))
    gm, fm = out["d_material"], ref["material"]
    okm = np.ones(fm.shape, bool) if converged is None else converged["material"]
    res["material"] = float((np.abs(gm - fm) * okm).max() / max(np.abs(fm).max(), 1e-300))
    types = np.unique(np.concatenate([l["type"] for l in r["lists"]]))
    print(f"{name}: {len(r['lists'])} steps, {np.mean([len(l['idA']) for l in r['lists']]):.0f} contacts per step "
          f"(types {types}); material gradients CUDA {gm.ravel()} / reference {fm.ravel()}; largest difference over "
          f"the group's largest gradient: {', '.join(f'{k} {v:.1e}' for k, v in res.items())}")
    for k, v in res.items():
        assert v <= (mat_bar if k == "material" else state_bar), (k, res)
    drv = ~free
    assert np.all(out["d_pos0"][drv] == 0) and np.all(out["d_quat0"][drv] == 0)


@pytest.mark.parametrize("name", sorted(HOST))
def test_matches_fp64_host_adjoint_on_the_recorded_trajectory(name):
    make, settle = HOST[name]
    r = _run(make, settle, T_HOST, K_HOST)
    h = AG.adjoint(r["built"], r["states"], r["lists"], r["wts"], r["mats"])
    free = np.nonzero(r["free"])[0]
    ref = {k: h["d_" + k + "0"][free] for k in ("pos", "vel", "angvel", "quat")}
    ref["material"] = h["d_material"]
    _report(name, r, ref, 1e-4, 1e-4)


@pytest.mark.parametrize("name", sorted(WINDOW))
def test_frictionless_window_matches_fd_of_fp64_forward(name):
    make, settle = WINDOW[name]
    r = _run(make, settle, T_WINDOW, K_WINDOW, settle_on_oracle=True)
    built, S0 = r["built"], r["states"][0]
    S, _ = M.rollout_fixed(built, S0, r["lists"])
    d = np.abs(r["states"][-1]["pos"] - S["pos"])[r["free"]].max()
    assert d <= 1e-7, d
    nO = built.counts["o"]
    oA = built.arrays["sphere_owner"][r["lists"][0]["idA"]]
    owners = [int(o) for o in np.argsort(-(np.bincount(oA, minlength=nO) * r["free"]), kind="stable")[:4]]
    args = (built, S0, r["lists"], r["wts"])
    fm = [F.fd_materials(*args, rel=rel, base=r["mats"]) for rel in (1e-6, 2.5e-7)]
    eps = (1e-9, 1e-7, 1e-5, 1e-8)
    fs = [F.fd_state(*args, owners, eps=tuple(e * sc for e in eps), mats=r["mats"]) for sc in (1.0, 0.25)]
    ref = {k: fs[1][k] for k in ("pos", "vel", "angvel", "quat")}
    ref["material"] = fm[1]
    # components where the two step sizes agree within a tenth of the bar; at least three quarters of each group
    conv = {}
    for k, (a, b, bar) in {**{k: (fs[0][k], fs[1][k], 1e-2) for k in ("pos", "vel", "angvel", "quat")},
                           "material": (fm[0], fm[1], 5e-3)}.items():
        conv[k] = np.abs(a - b) <= 0.1 * bar * max(np.abs(b).max(), 1e-300)
        assert conv[k].mean() >= 0.75, (k, conv[k].mean())
    _report(name, r, ref, 5e-3, 1e-2, owners=owners, converged=conv)


def _pile_with(edit):
    """A sphere pile scene edited before Initialize (partial prescription, free wall)."""
    from deme_b200.scene import SceneBuilder, _Prescription
    rng = np.random.default_rng(1)
    s = SceneBuilder()
    s.InstructBoxDomainDimension(0.2, 0.2, 0.2)
    s.SetCoordSysOrigin("center")
    m = s.LoadMaterial({"E": 1e7, "nu": 0.3, "CoR": 0.5, "mu": 0.3, "Crr": 0.01})
    t = s.LoadSphereType(1e-4, 2.5e-3, m)
    b = s.AddClumps([t] * 27, (rng.uniform(-0.02, 0.02, (27, 3))).astype(np.float32))
    s.AddBCPlane((0, 0, -0.05), (0, 0, 1), m)
    edit(s, b, m, _Prescription)
    s.SetInitTimeStep(1e-5)
    s.SetCDUpdateFreq(1)
    return s.Initialize()


@pytest.mark.parametrize("case", ["partial_clump_prescription", "free_wall"])
def test_scope_is_checked(case):
    from deme_b200 import Solver, adjoint
    from deme_b200.solver import DemeError

    def partial(s, b, m, P):
        b.SetFamily(3)
        s.prescriptions.append(P(3, linVel=["0", "0", "0"], linVelPrescribed=True, rotVelPrescribed=False))

    def free_wall(s, b, m, P):
        w = s.AddExternalObject()
        w.AddPlane((0, 0, 0.05), (0, 0, -1), m)
        w.SetFamily(5)

    built = _pile_with(partial if case == "partial_clump_prescription" else free_wall)
    g = Solver(built)
    with pytest.raises(DemeError, match="INVALID.*(partly prescribed|prescribed motion)"):
        adjoint.record(g, 2, 1)
    g.close()

