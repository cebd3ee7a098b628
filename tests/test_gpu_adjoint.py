"""CUDA adjoint (deme_adjoint_record / deme_adjoint_backward) against the FP64 host adjoint and central finite
differences of the FP64 forward model (oracle/adjoint_fp64.py) on piles of spheres on a floor plane, over a window
longer than one checkpoint segment.

Two piles: a gentle one (light overlaps, slow spins), where the CUDA forward (FP32 state, orientation integrated
in the owner frame) stays within 1e-10 m of the FP64 model, and a lively one (deeper overlaps, faster spins), where
the two trajectories separate by ~1e-8 m over the window and contact chaos amplifies that separation in the
gradients.  Bars: material gradients within 1e-3 relative (gentle) / 3e-3 (lively) of the FP64 host adjoint and
of central finite differences of the FP64 forward; initial-state gradients within 1e-3 of their largest
magnitude."""
import numpy as np
import pytest

from _util import workloads
from oracle import adjoint_fp64 as A

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

STEPS, K = 30, 8


def weights(nO, n, seed=7):
    rng = np.random.default_rng(seed)
    wx = np.zeros((nO, 3))
    wv = np.zeros((nO, 3))
    wx[:n] = rng.normal(size=(n, 3))
    wv[:n] = rng.normal(size=(n, 3)) * 1e-2
    return wx, wv


PILES = {
    "gentle": (dict(noise=1e-4, vel_scale=0.02, spin_scale=5.0, spread=5.8e-3, lift=2.9e-3), 1e-3),
    "lively": (dict(noise=1e-4, vel_scale=0.05, spin_scale=10.0, spread=5.5e-3, lift=2.95e-3), 3e-3),
}


@pytest.fixture(scope="module", params=sorted(PILES))
def run(request):
    """Exact derivatives (floors 0) on both sides: the piles are compared with the derivative of the model."""
    from deme_b200 import Solver, adjoint
    kw, bar = PILES[request.param]
    built = workloads.sphere_pile(n=60, seed=3, **kw)
    g = Solver(built)
    adjoint.set_floors(g, 0.0, 0.0, 0.0)
    saved = dict(A.REG)
    A.REG.update(delta_rel=0.0, roll_speed=0.0, ft=0.0)
    n = built.counts["s"]
    wx, wv = weights(built.counts["o"], n)
    adjoint.record(g, STEPS, K)
    pos, vel, _ = adjoint.final_state(g)
    out = adjoint.backward(g, d_pos=wx, d_vel=wv)
    sc, x0, v0, w0 = A.from_built(built)
    (xf, vf, wf), rec = A.rollout(sc, x0, v0, w0, STEPS)
    gx, gv, gw, gmat = A.adjoint(sc, rec, wx[:n], wv[:n], np.zeros((n, 3)))
    A.REG.update(saved)
    return dict(built=built, out=out, pos=pos, xf=xf, sc=sc, x0=x0, v0=v0, w0=w0, host=(gx, gv, gw, gmat), wx=wx,
                wv=wv, n=n, rec=rec, bar=bar)


def test_forward_windows_agree(run):
    # the CUDA forward (mixed precision, orientation in the owner frame) and the FP64 model stay within 1e-7 m
    d = np.abs(run["pos"][:run["n"]] - run["xf"]).max()
    assert d <= 1e-7, d
    assert sum(len(s.ss) for s in run["rec"]) > 40 and sum(len(s.sp) for s in run["rec"]) > 10


def test_material_gradients_match_host_adjoint(run):
    g, (_, _, _, gm) = run["out"]["d_material"], run["host"]
    assert g.shape == gm.shape == (2, 4)
    err = np.abs(g - gm) / np.maximum(np.abs(gm), 1e-30)
    assert np.all(err <= run["bar"]), (g, gm, err)


def test_state_gradients_match_host_adjoint(run):
    out, (gx, gv, gw, _), n = run["out"], run["host"], run["n"]
    for name, a, b in (("pos", out["d_pos0"][:n], gx), ("vel", out["d_vel0"][:n], gv), ("angvel", out["d_angvel0"][:n], gw)):
        assert np.abs(a - b).max() <= 1e-3 * np.abs(b).max(), (name, np.abs(a - b).max(), np.abs(b).max())


def test_material_gradients_match_fd_of_fp64_forward(run):
    sc, n = run["sc"], run["n"]
    wx, wv = run["wx"][:n], run["wv"][:n]

    def loss():
        (xf, vf, _), _ = A.rollout(sc, run["x0"], run["v0"], run["w0"], STEPS)  # the forward has no floors
        return float(np.sum(wx * xf) + np.sum(wv * vf))

    g = run["out"]["d_material"]
    for mi in range(2):
        for j, name in enumerate(("E", "CoR", "mu", "Crr")):
            arr = getattr(sc, name)
            base = arr[mi]
            eps = 1e-5 * base
            arr[mi] = base + eps
            lp = loss()
            arr[mi] = base - eps
            lm = loss()
            arr[mi] = base
            fd = (lp - lm) / (2 * eps)
            assert abs(g[mi, j] - fd) <= run["bar"] * abs(fd), (mi, name, g[mi, j], fd)


def test_torch_autograd_function_gives_the_adjoint_gradients():
    """The torch.autograd.Function binding: parameters -> final positions and velocities; loss.backward() returns
    the material gradients of the C ABI adjoint (and hence of the FP64 host adjoint)."""
    from deme_b200 import Solver, adjoint
    kw, bar = PILES["gentle"]
    built = workloads.sphere_pile(n=60, seed=3, **kw)
    g = Solver(built)
    adjoint.set_floors(g, 0.0, 0.0, 0.0)
    init = {k: v for k, v in g.state().items() if not k.startswith("a")}
    a = built.arrays
    params = torch.tensor(np.stack([a["mat_E"], a["mat_CoR"], a["mat_mu"], a["mat_Crr"]], 1).astype(np.float64),
                          requires_grad=True)
    Rollout = adjoint.make_rollout_function()
    pos, vel = Rollout.apply(params, g, init, a["mat_nu"].astype(np.float64), STEPS, K)
    n = built.counts["s"]
    wx, wv = weights(built.counts["o"], n)
    loss = (torch.from_numpy(wx) * pos).sum() + (torch.from_numpy(wv) * vel).sum()
    loss.backward()
    sc, x0, v0, w0 = A.from_built(built)
    _, rec = A.rollout(sc, x0, v0, w0, STEPS)
    saved = dict(A.REG)
    A.REG.update(delta_rel=0.0, roll_speed=0.0, ft=0.0)
    _, _, _, gm = A.adjoint(sc, rec, wx[:n], wv[:n], np.zeros((n, 3)))
    A.REG.update(saved)
    err = np.abs(params.grad.numpy() - gm) / np.maximum(np.abs(gm), 1e-30)
    assert np.all(err <= bar), (params.grad, gm)


def _host_contacts(c):
    """A GPU contact list with its updated histories, split as the host model keeps it (sphere pairs, sphere-plane
    pairs, each with its history)."""
    from deme_b200 import capi
    ss = c["type"] == capi.SPHERE_SPHERE_CONTACT
    pairs = np.stack([c["idA"], c["idB"]], 1).astype(np.int64)
    h = c["wildcards"].T.astype(np.float64)
    return pairs[ss], pairs[~ss], h[ss], h[~ss]


def test_column_collapse_windows_match_host_adjoint_on_the_gpu_trajectory():
    """A column of 300 spheres released over a floor, 2000 steps, default derivative floors on both sides.  Over so
    many steps the FP32 CUDA trajectory and an FP64 rollout of the same start separate chaotically, and so do their
    gradients (central differences of the FP64 forward themselves spread by 40 % over 0.3-3 % steps), so the run is
    checked window by window on the CUDA trajectory itself: from the state and contact histories the CUDA run had
    at the start of each 100-step window, the CUDA adjoint of the window (seeded with the gradient the later windows
    returned) and the FP64 host adjoint of an FP64 rollout of that window agree on the E, CoR and mu gradients within
    2 % of the window's largest material gradient and on the gradient with respect to the window's initial positions
    within 2 % of its largest.  The Crr gradient comes from rolling contacts whose torque direction flips where the
    relative rolling speed crosses zero, which the FP32 and FP64 rollouts reach at slightly different steps, so
    single windows can disagree even in sign: summed over the windows, its differences stay within half of the
    summed host gradients."""
    from deme_b200 import Solver, adjoint
    built = workloads.column_collapse(n=300)
    g = Solver(built)
    n = built.counts["s"]
    T, W = 2000, 100
    init = built.decode_positions(built.initial_state(), kernel_literals=False)[:n]
    starts = []
    for w in range(T // W):
        starts.append((g.state(), g.contacts() if w else None))
        g.step(W)
    pos, _, _ = adjoint.final_state(g)
    axis, z0 = init[:, :2].mean(0), float(init[:, 2].min())
    _, gpos = workloads.collapse_loss(pos[:n], axis, z0)
    nO = built.counts["o"]
    seed = [np.zeros((nO, 3)) for _ in range(3)] + [np.zeros((nO, 4))]
    seed[0][:n] = gpos
    worst = np.zeros(4)
    worst_x = 0.0
    ratio_crr = []
    crr_diff = crr_host = 0.0
    for w in range(T // W - 1, -1, -1):
        st, c = starts[w]
        g.set_state({k: v for k, v in st.items() if not k.startswith("a")})
        if c is not None:
            g.set_contacts({k: c[k] for k in ("idA", "idB", "type", "wildcards")})
        adjoint.record(g, W, W)
        out = adjoint.backward(g, d_pos=seed[0], d_vel=seed[1], d_angvel=seed[2], d_quat=seed[3])
        sc, x0, v0, _ = A.from_built(built, state=st)
        w0 = adjoint.world_angular_velocity(st)[:n]
        hc = _host_contacts(c) if c is not None else None
        _, rec = A.rollout(sc, x0, v0, w0, W, init=hc)
        hx, hv, hw, hm = A.adjoint(sc, rec, seed[0][:n], seed[1][:n], seed[2][:n])
        gm = out["d_material"][0]
        scale = np.abs(hm[0]).max()
        err = np.abs(gm - hm[0]) / max(scale, 1e-300)
        worst = np.maximum(worst, err)
        assert np.all(err[:3] <= 2e-2), (w, gm, hm[0])
        crr_diff += abs(gm[3] - hm[0][3])
        crr_host += abs(hm[0][3])
        if abs(hm[0][3]) > 1e-3 * scale:
            ratio_crr.append(gm[3] / hm[0][3])
        ex = np.abs(out["d_pos0"][:n] - hx).max() / max(np.abs(hx).max(), 1e-300)
        worst_x = max(worst_x, ex)
        assert ex <= 2e-2, (w, ex)
        seed = [out["d_pos0"], out["d_vel0"], out["d_angvel0"], out["d_quat0"]]
    r = np.array(ratio_crr)
    assert crr_diff <= 0.5 * crr_host, (crr_diff, crr_host, r)
    print(f"column collapse, 20 windows of 100 steps: largest material-gradient difference (E, CoR, mu, Crr) "
          f"{worst.round(5)} of the window's largest, position gradient {worst_x:.2e}; Crr summed difference "
          f"{crr_diff / max(crr_host, 1e-300):.3f} of the summed host gradients, ratios {r.round(3)}")


def _fd_material(sc, x0, v0, w0, T, loss_of, rel=1e-3):
    """Central differences of the FP64 forward at relative step `rel` for material 0's E, CoR, mu, Crr."""
    out = np.zeros(4)
    for j, field in enumerate(("E", "CoR", "mu", "Crr")):
        base = float(getattr(sc, field)[0])
        if base == 0.0:
            continue
        vals = []
        for sgn in (1.0, -1.0):
            sc2 = A.SphereScene(**{k: getattr(sc, k) for k in sc.__dataclass_fields__})
            arr = getattr(sc2, field).copy()
            arr[0] = base * (1.0 + sgn * rel)
            setattr(sc2, field, arr)
            (xf, _, _), _ = A.rollout(sc2, x0, v0, w0, T)
            vals.append(loss_of(xf))
        out[j] = (vals[0] - vals[1]) / (2.0 * rel * base)
    return out


@pytest.mark.parametrize("T,bars", [(300, {"E": 1e-3, "CoR": 1e-3}), (1000, {"CoR": 2e-3})])
def test_reduced_column_collapse_against_fd_of_fp64_forward(T, bars):
    """The column-collapse loss (mean squared runout plus the heap-angle proxy) of a reduced collapse, 60 spheres of
    2-3 mm released onto the floor, checkpoints every 100 steps, exact derivatives (floors 0) on both sides: the
    CUDA adjoint's material gradients against central differences of the FP64 forward at relative step 1e-3.
    Over the first 300 steps (fall and first impact) the E and CoR gradients agree within 1e-3; over 1000 steps
    (the heap forms) the CoR gradient still does, while E and Crr come from contacts that open and close and from
    rolling torques that flip direction, where the loss is not smooth at the scale of a 1e-3 parameter step (the
    differences at 1e-3 and 1e-4 disagree with each other); those are printed.  Friction is not yet loaded over
    these windows (its gradient is 0 on both sides)."""
    from deme_b200 import Solver, adjoint
    built = workloads.column_collapse(n=60)
    n = built.counts["s"]
    g = Solver(built)
    adjoint.set_floors(g, 0.0, 0.0, 0.0)
    saved = dict(A.REG)
    A.REG.update(delta_rel=0.0, roll_speed=0.0, ft=0.0)
    try:
        sc, x0, v0, w0 = A.from_built(built)
        axis, z0 = x0[:, :2].mean(0), float(x0[:, 2].min())
        adjoint.record(g, T, 100)
        st = g.state()
        xf = built.decode_positions(st)[:n]
        _, gpos = workloads.collapse_loss(xf, axis, z0)
        seed = np.zeros((built.counts["o"], 3))
        seed[:n] = gpos
        gg = adjoint.backward(g, d_pos=seed)["d_material"][0]
        fd = _fd_material(sc, x0, v0, w0, T, lambda x: workloads.collapse_loss(x, axis, z0)[0])
    finally:
        A.REG.update(saved)
    names = ("E", "CoR", "mu", "Crr")
    err = {nm: abs(gg[j] - fd[j]) / max(abs(fd[j]), 1e-300) for j, nm in enumerate(names)}
    print(f"reduced collapse, {T} steps: CUDA adjoint {gg}, FD of the FP64 forward {fd}, relative differences "
          f"{ {k: round(v, 6) for k, v in err.items()} }")
    for nm, bar in bars.items():
        assert err[nm] <= bar, (nm, err[nm], gg, fd)
    if fd[2] == 0.0:  # no contact reached its Coulomb cap
        assert abs(gg[2]) <= 1e-9 * np.abs(gg).max(), gg
