"""The FP64 host adjoint (oracle/fp64_autograd.py) that the CUDA adjoint is checked against, pinned on the CPU:
its forward step equals the FP64 model (oracle/fp64_model.step_state with the CUDA path's float32 placement) to
rounding, and its one-step gradients equal central differences of that model.  The scene is a drum of 150
three-sphere clumps turning at 20 rpm (analytical cylinder and two end planes), settled on the C oracle, so that
clump--clump, clump--plane and clump--cylinder contacts carry history, slide and roll."""
import numpy as np
import pytest

import _adjoint_fd as F
from _util import oracle, workloads
from oracle import fp64_model as M

torch = pytest.importorskip("torch")
from oracle import fp64_autograd as AG  # noqa: E402


@pytest.fixture(scope="module")
def drum():
    built = workloads.drum(n_clumps=150, fill=0.2, wall_clearance=0.8)
    orc = oracle(built, threads=4)
    orc.step(25000)
    lists, states = F.record_lists(orc, 1, built)
    orc.close()
    mats = {k: v.astype(np.float32).astype(np.float64) for k, v in F.materials(built).items()}
    return built, lists, states, mats


def test_forward_equals_fp64_model(drum):
    built, lists, states, mats = drum
    S0 = states[0]
    r = M.step_state(built, S0, lists[0], mats=mats, f32=True, q_anchor=S0["q"])
    mt = {k: AG._t(v) for k, v in mats.items()}
    (pn, qn, vn, wn), hout = AG.step(built, S0, lists[0], *(AG._t(S0[k]) for k in ("pos", "q", "v", "w")),
                                     AG._t(lists[0]["wildcards"].T.copy()), mt)
    free = AG.free_owners(built, S0["family"])
    for got, want in ((pn, r["pos"]), (vn, r["vel"]), (wn, r["angvel"]), (qn, r["quat"])):
        g, w_ = got.detach().numpy()[free], want[free]
        assert np.abs(g - w_).max() <= 1e-12 * max(np.abs(w_).max(), 1e-30)
    assert np.abs(hout.detach().numpy() - r["hist"]).max() <= 1e-12 * np.abs(r["hist"]).max()
    assert len(np.unique(lists[0]["type"])) == 3


def test_one_step_gradients_equal_central_differences(drum):
    built, lists, states, mats = drum
    S0 = states[0]
    free = AG.free_owners(built, S0["family"])
    wts = F.weights(built.counts["o"], free)
    h = AG.adjoint(built, states, lists, wts, mats)
    fm = F.fd_materials(built, S0, lists, wts, base=mats, f32=True)
    err = np.abs(h["d_material"] - fm).max() / np.abs(fm).max()
    assert err <= 1e-4, (h["d_material"], fm)
    owners = list(np.nonzero(free)[0][:4])
    fs = F.fd_state(built, S0, lists, wts, owners, eps=(1e-11, 1e-9, 1e-7, 1e-10), mats=mats, f32=True)
    for k in ("pos", "vel", "angvel", "quat"):
        e = np.abs(h["d_" + k + "0"][owners] - fs[k]).max() / np.abs(fs[k]).max()
        assert e <= 1e-3, (k, e)
