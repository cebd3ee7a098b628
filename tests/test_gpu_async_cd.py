"""kT and dT as two streams (deme_set_async_cd): a detection due at step k runs on the kT stream from the poses of step
k while dT keeps stepping, and dT adopts it at step k + lag.

* The list dT adopts is exactly the detection on the poses of step k: the oracle run on the state downloaded at step
  k gives the same contact list (canonical order, bit-exact).
* Two streams give the same run as one: kT and dT on two streams and on a single stream (the same work in program
  order) end in the same states and contact lists, up to the order of the float atomics that sum owner forces.
* A lag above the detection period, or above 1 with detection every step, is refused.
"""
import numpy as np
import pytest

from _util import canonical, oracle, workloads

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def scene(cd_freq=4):
    return workloads.hopper(n=20000, seed=5, cd_freq=cd_freq, wall_clearance=0.95)


@pytest.mark.parametrize("lag", [1, 4])
def test_adopted_list_is_the_detection_on_the_snapshot(lag):
    from deme_b200 import Solver
    built = scene()
    f = int(built.params.cd_update_freq)
    g = Solver(built)
    g.set_async_cd(lag)
    snaps = {}
    checked = 0
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
        for k in ("idA", "idB", "type"):
            np.testing.assert_array_equal(gc[k], oc[k], err_msg=f"lag {lag} step {s} (poses of step {src}) {k}")
        checked += 1
    assert checked >= 3
    g.close()


@pytest.mark.parametrize("lag", [1, 4])
def test_two_streams_equal_one_stream(lag):
    """The owner sums of a step go through float atomics, whose order the GPU does not fix, so the two runs agree to
    float-sum-order bounds, not bit for bit: positions within 1e-7 m, velocities within 1e-3 of the largest speed,
    and contact lists equal up to a few pairs at the overlap threshold."""
    from deme_b200 import Solver
    built = scene()
    two = Solver(built)
    two.set_async_cd(lag)
    one = Solver(built)
    st = torch.cuda.Stream()
    one.set_streams(st.cuda_stream, st.cuda_stream)
    one.set_async_cd(lag)
    for _ in range(6):
        two.step(7)
        one.step(7)
    a, b = two.state(), one.state()
    pa, pb = built.decode_positions(a), built.decode_positions(b)
    assert np.abs(pa - pb).max() <= 1e-7
    for k in ("vX", "vY", "vZ", "omgX", "omgY", "omgZ"):
        x, y = a[k].astype(np.float64), b[k].astype(np.float64)
        assert np.abs(x - y).max() <= 1e-3 * max(np.abs(y).max(), 1e-6), k
    np.testing.assert_array_equal(a["family"], b["family"])
    ca, cb = two.contacts(), one.contacts()
    ka = {(int(i), int(j), int(t)) for i, j, t in zip(ca["idA"], ca["idB"], ca["type"])}
    kb = {(int(i), int(j), int(t)) for i, j, t in zip(cb["idA"], cb["idB"], cb["type"])}
    assert len(ka) > 0
    assert len(ka ^ kb) <= max(2, len(ka) // 10000), len(ka ^ kb)
    two.close()
    one.close()


def test_lag_outside_range_is_refused():
    from deme_b200 import Solver
    from deme_b200.solver import DemeError
    g = Solver(scene(cd_freq=4))
    with pytest.raises(DemeError):
        g.set_async_cd(5)
    with pytest.raises(DemeError):
        g.set_async_cd(-1)
    g.set_async_cd(4)
    g.close()
    every = Solver(workloads.packed_clumps(n_clumps=64, seed=1))
    with pytest.raises(DemeError):
        every.set_async_cd(2)
    every.set_async_cd(1)
    every.close()
