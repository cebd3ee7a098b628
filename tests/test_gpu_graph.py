"""Whole steps replayed from CUDA graphs (deme_set_graph) against the same steps launched one by one.

* A settling scene: a run in graph mode and a run in the plain mode end with the same contact list and the same
  state (positions within 1e-9 m, velocities within 1e-6 of their scale), the graph windows were replayed and none
  rolled back.
* Detection every 4 steps: the same, with windows of 4 steps and steps before and after the whole windows.
* A dense lattice whose first detection finds more pairs than the pair pool holds: the replayed batch is rolled back
  and redone step by step, and the run still equals the plain run.
* The kinetic energy read without a wait (deme_kinetic_energy_enqueue / _collect), one step behind the stepping
  as a pipelined caller reads it, equals the blocking read after each step; a ticket whose slot was reused is
  refused.
"""
import numpy as np
import pytest

from _util import workloads

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def run(built, steps, graph, chunks=1):
    from deme_b200 import Solver
    s = Solver(built)
    if graph:
        s.set_graph(True)
    for _ in range(chunks):
        s.step(steps // chunks)
    st, c = s.state(), s.contacts()
    stats = s.graph_stats()
    s.close()
    return st, c, stats


def compare(built, a, b):
    (sa, ca, _), (sb, cb, _) = a, b
    for k in ("idA", "idB", "type"):
        np.testing.assert_array_equal(ca[k], cb[k], err_msg=k)
    pa = built.decode_positions(sa, kernel_literals=False)
    pb = built.decode_positions(sb, kernel_literals=False)
    assert np.abs(pa - pb).max() <= 1e-9, np.abs(pa - pb).max()
    for k in ("vX", "vY", "vZ", "omgX", "omgY", "omgZ"):
        scale = np.abs(sb[k]).max() + 1e-12
        assert np.abs(sa[k].astype(np.float64) - sb[k]).max() <= 1e-6 * scale, k


def test_graph_replay_equals_step_by_step():
    built = workloads.settling_box(n=3000, spacing=2.05, jitter=0.05, seed=4, vel_scale=0.3)
    g = run(built, 60, True, chunks=3)
    p = run(built, 60, False, chunks=3)
    compare(built, g, p)
    replays, rollbacks = g[2]
    assert replays == 60 and rollbacks == 0, g[2]
    assert len(g[1]["idA"]) > 0


def test_replayed_kernels_are_counted():
    import ctypes as C
    from deme_b200 import Solver
    built = workloads.packed_clumps(n_clumps=300, seed=7, spacing=1.35)  # contacts from the first step on
    counts = {}
    for graph in (False, True):
        s = Solver(built)
        s.lib.deme_launch_count.restype = C.c_int64
        if graph:
            s.set_graph(True)
        s.step(2)
        n0 = s.lib.deme_launch_count()
        s.step(10)
        s.sync()
        counts[graph] = s.lib.deme_launch_count() - n0
        s.close()
    # a replayed window runs the kernels the step-by-step path launches, plus the one that counts the window
    assert counts[True] == counts[False] + 10, counts


def test_graph_windows_with_detection_every_four_steps():
    built = workloads.hopper(n=20000, seed=5, cd_freq=4, wall_clearance=0.95)
    g = run(built, 42, True, chunks=2)  # 21 steps per call: windows of 4 plus steps outside them
    p = run(built, 42, False, chunks=2)
    compare(built, g, p)
    assert g[2][0] >= 8 and g[2][1] == 0, g[2]


def test_pool_overflow_inside_a_window_rolls_back():
    # pitch 1.9 r: every sphere overlaps its face neighbours, about three contacts per sphere at the first
    # detection, more than the pair pool (twice the sphere count) holds before it has grown
    built = workloads.settling_box(n=8000, spacing=1.9, jitter=0.0)
    g = run(built, 10, True)
    p = run(built, 10, False)
    compare(built, g, p)
    assert g[2][1] >= 1, g[2]


def test_kinetic_energy_enqueue_collect_matches_the_blocking_read():
    from deme_b200 import Solver
    from deme_b200.solver import DemeError
    built = workloads.settling_box(n=3000, spacing=2.05, jitter=0.05, seed=4, vel_scale=0.3)
    ref = Solver(built)
    want = []
    for _ in range(6):
        ref.step(3)
        want.append(ref.kinetic_energy())
    ref.close()
    s = Solver(built)
    s.set_graph(True)
    got, prev = [], None
    for _ in range(6):
        s.step(3)
        t = s.kinetic_energy_enqueue()
        if prev is not None:
            got.append(s.kinetic_energy_collect(prev))
        prev = t
    got.append(s.kinetic_energy_collect(prev))
    np.testing.assert_allclose(got, want, rtol=1e-6)
    # five enqueues reuse the first ticket's slot
    first = s.kinetic_energy_enqueue()
    for _ in range(4):
        s.kinetic_energy_enqueue()
    with pytest.raises(DemeError):
        s.kinetic_energy_collect(first)
    s.close()

