"""The FP64 host adjoint (oracle/adjoint_fp64.py) against central finite differences of the FP64 forward model:
gradients of a linear loss of the final state with respect to the material parameters (E, CoR, mu, Crr) and to
initial positions, velocities and angular velocities, on a small pile of spheres on a floor plane (sphere-sphere
and sphere-plane contacts, Coulomb cap and rolling resistance active).  Bar: 1e-5 relative.  The derivative floors
are set to zero here (exact derivative of the discrete model)."""
import numpy as np
import pytest

from oracle import adjoint_fp64 as A


@pytest.fixture(autouse=True)
def exact_derivatives():
    """These tests check the exact derivative of the discrete model: no floors at the non-smooth points."""
    saved = dict(A.REG)
    A.REG.update(delta_rel=0.0, roll_speed=0.0, ft=0.0)
    yield
    A.REG.update(saved)


def pile(seed=1, n=40):
    rng = np.random.default_rng(seed)
    r = rng.uniform(2e-3, 3e-3, n)
    rho = 2500.0
    m = 4 / 3 * np.pi * r ** 3 * rho
    inertia = 0.4 * m * r * r
    # spheres on a loose lattice just touching a floor at z = 0, a little interpenetrated
    side = int(np.ceil(n ** (1 / 3)))
    idx = np.arange(n)
    a = 5.2e-3
    x = np.stack([(idx % side) * a, ((idx // side) % side) * a, (idx // side // side) * a + 2.2e-3], 1).astype(float)
    x += rng.normal(0, 4e-4, x.shape)
    v = rng.normal(0, 0.05, (n, 3))
    w = rng.normal(0, 20.0, (n, 3))
    planes = [(np.zeros(3), np.array([0.0, 0.0, 1.0]), 1, np.zeros(3))]
    sc = A.SphereScene(r=r, m=m, inertia=inertia, mat=(idx % 2).astype(np.int64), planes=planes,
                       E=np.array([1e7, 5e7]), nu=np.array([0.3, 0.25]), CoR=np.array([0.5, 0.4]),
                       mu=np.array([0.3, 0.5]), Crr=np.array([0.01, 0.03]), h=2e-5, g=np.array([0, 0, -9.81]))
    return sc, x, v, w


def loss_weights(n, seed=7):
    rng = np.random.default_rng(seed)
    return rng.normal(size=(n, 3)), rng.normal(size=(n, 3)) * 1e-2, rng.normal(size=(n, 3)) * 1e-4


def loss(sc, x, v, w, steps, W):
    (xf, vf, wf), _ = A.rollout(sc, x, v, w, steps)
    return float(np.sum(W[0] * xf) + np.sum(W[1] * vf) + np.sum(W[2] * wf))


@pytest.mark.parametrize("steps", [1, 25])
def test_host_adjoint_matches_fd_of_fp64_forward(steps):
    sc, x, v, w = pile()
    W = loss_weights(len(sc.r))
    (_, _, _), rec = A.rollout(sc, x, v, w, steps)
    nss = sum(len(s.ss) for s in rec)
    nsp = sum(len(s.sp) for s in rec)
    assert nss > 10 and nsp > 5
    if steps > 1:  # the Coulomb cap and rolling resistance are both active somewhere in the window
        ncap = nroll = 0
        for st in rec:
            _, _, out = A.forces(sc, st.x, st.v, st.w, st.ss, st.sp, st.hist_ss, st.hist_sp, keep=True)
            for kind in out:
                ncap += int(out[kind][2]["cap"].sum())
                nroll += int(out[kind][2]["roll"].sum())
        assert ncap > 0 and nroll > 0
    gx, gv, gw, gmat = A.adjoint(sc, rec, W[0], W[1], W[2])
    # material parameters
    for mi in range(2):
        for j, name in enumerate(("E", "CoR", "mu", "Crr")):
            arr = getattr(sc, name)
            base = arr[mi]
            eps = 1e-6 * base
            arr[mi] = base + eps
            lp = loss(sc, x, v, w, steps, W)
            arr[mi] = base - eps
            lm = loss(sc, x, v, w, steps, W)
            arr[mi] = base
            fd = (lp - lm) / (2 * eps)
            assert abs(gmat[mi, j] - fd) <= 1e-5 * max(abs(fd), 1e-30) + 1e-12, (mi, name, gmat[mi, j], fd)
    # initial state (a few components)
    rng = np.random.default_rng(3)
    for arr, g, scale in ((x, gx, 1e-8), (v, gv, 1e-6), (w, gw, 1e-4)):
        for _ in range(6):
            i, c = int(rng.integers(len(sc.r))), int(rng.integers(3))
            base = arr[i, c]
            arr[i, c] = base + scale
            lp = loss(sc, x, v, w, steps, W)
            arr[i, c] = base - scale
            lm = loss(sc, x, v, w, steps, W)
            arr[i, c] = base
            fd = (lp - lm) / (2 * scale)
            assert abs(g[i, c] - fd) <= 1e-5 * max(abs(fd), abs(g[i, c])) + 1e-9, (i, c, g[i, c], fd)
