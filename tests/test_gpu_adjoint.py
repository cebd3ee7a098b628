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


def test_column_collapse_with_default_floors_matches_host():
    """A column of 300 spheres released over a floor for 2000 steps (contact onsets at near-zero rolling speed: the
    exact derivative is unbounded there) with the default derivative floors on both sides: the CUDA and FP64 host
    adjoints agree on the E, CoR and mu gradients within 5e-2 relative (the trajectories separate chaotically over
    2000 steps) and on the Crr gradient in sign and within a factor 2: it comes from rolling contacts at near-zero
    relative spin, where the CUDA forward (orientation integrated in the owner frame) and the FP64 model differ most,
    and central differences of the FP64 forward themselves spread by 40 % over 0.3-3 % steps."""
    from deme_b200 import Solver, adjoint
    built = workloads.column_collapse(n=300)
    g = Solver(built)
    n = built.counts["s"]
    T = 2000
    init = built.decode_positions(built.initial_state(), kernel_literals=False)[:n]
    adjoint.record(g, T, 100)
    pos, _, _ = adjoint.final_state(g)
    axis, z0 = init[:, :2].mean(0), float(init[:, 2].min())
    _, gpos = workloads.collapse_loss(pos[:n], axis, z0)
    seed = np.zeros((built.counts["o"], 3))
    seed[:n] = gpos
    out = adjoint.backward(g, d_pos=seed)
    sc, x0, v0, w0 = A.from_built(built)
    (xf, _, _), rec = A.rollout(sc, x0, v0, w0, T)
    _, gh = workloads.collapse_loss(xf, axis, z0)
    gm = A.adjoint(sc, rec, gh, np.zeros((n, 3)), np.zeros((n, 3)))[3][0]
    gg = out["d_material"][0]
    for j, name in enumerate(("E", "CoR", "mu")):
        assert abs(gg[j] - gm[j]) <= 5e-2 * abs(gm[j]), (name, gg[j], gm[j])
    assert gg[3] * gm[3] > 0 and 0.5 <= gg[3] / gm[3] <= 2.0, (gg[3], gm[3])
    assert np.all(np.isfinite(gg)) and abs(gg[1]) < 1.0 and abs(gg[3]) < 1.0
