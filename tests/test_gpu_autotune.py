"""Search shapes and the autotuner (deme_set_search_shape, deme_autotune).

* Every pooled-search block shape and search-cell factor finds the same contact list, bit for bit, on a dense clump
  scene and on a polydisperse hopper (one detection from the same state).
* The autotuner times every shape, keeps one of them, and leaves the state (positions, orientations, velocities)
  and contact history as they were: the run after it equals a run that never called it.
"""
import numpy as np
import pytest

from _util import workloads

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

SCENES = {
    "clumps": lambda: workloads.packed_clumps(n_clumps=3000, seed=41, spacing=1.3),
    "hopper": lambda: workloads.hopper(n=30000, seed=7, cd_freq=1, wall_clearance=0.95),
}


@pytest.mark.parametrize("name", list(SCENES))
def test_every_search_shape_finds_the_same_list(name):
    from deme_b200 import Solver
    built = SCENES[name]()
    ref = None
    s = Solver(built)
    count = s.lib.deme_search_shape_count()
    assert count >= 4
    st0 = s.state()
    for shape in range(count):
        for factor in (1.0, 1.25, 1.5, 2.0):
            s.set_search_shape(shape, factor)
            s.set_state(st0)
            s.detect_contacts()
            c = s.contacts()
            got = np.stack([c["idA"], c["idB"], c["type"]], 1)
            if ref is None:
                ref = got
                assert len(ref) > 0
            else:
                np.testing.assert_array_equal(got, ref, err_msg=f"{name} shape {shape} factor {factor}")
    s.close()


def test_autotune_keeps_the_state_and_the_run():
    from deme_b200 import Solver
    built = SCENES["clumps"]()
    a = Solver(built)
    a.step(3)
    before, cb = a.state(), a.contacts()
    t = a.autotune(steps_per_trial=3)
    assert 0 <= t["shape"] < a.lib.deme_search_shape_count() and t["trials"] >= 12
    assert t["ms_per_step"] <= t["ms_per_step_default"] + 1e-6
    after, ca = a.state(), a.contacts()
    for k in before:
        if k.startswith("a"):  # accelerations are outputs of the last step, recomputed by the next
            continue
        np.testing.assert_array_equal(before[k], after[k], err_msg=k)
    for k in ("idA", "idB", "type", "wildcards"):
        np.testing.assert_array_equal(cb[k], ca[k], err_msg=k)
    b = Solver(built)
    b.step(3)
    a.step(5)
    b.step(5)
    for k in ("idA", "idB", "type"):
        np.testing.assert_array_equal(a.contacts()[k], b.contacts()[k], err_msg=k)
    pa = built.decode_positions(a.state(), kernel_literals=False)
    pb = built.decode_positions(b.state(), kernel_literals=False)
    assert np.abs(pa - pb).max() <= 1e-9
    a.close()
    b.close()
