"""Search shapes and the autotuner (deme_set_search_shape, deme_autotune).

* Every pooled-search block shape and search-cell factor finds the same contact list, bit for bit, on a dense clump
  scene and on a polydisperse hopper (one detection from the same state).
* Every block shape of the force kernel, the exact pair test and the integration (deme_set_kernel_shapes) gives
  the same contact list and bit-identical per-contact forces, and owner accelerations within float-sum order.
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


def test_every_kernel_shape_gives_the_same_forces():
    from deme_b200 import Solver
    built = SCENES["clumps"]()
    s = Solver(built)
    s.keep_contact_forces(True)
    s.step(2)
    st0, c0 = s.state(), s.contacts()
    ref = None
    for force_shape in range(s.lib.deme_force_shape_count()):
        for threads in (128, 256, 512):
            s.set_kernel_shapes(force_shape, threads, threads)
            s.set_state({k: v for k, v in st0.items() if not k.startswith("a")})
            s.set_contacts({k: c0[k] for k in ("idA", "idB", "type", "wildcards")})
            s.detect_contacts()
            s.compute_forces()
            c, f, st = s.contacts(), s.contact_forces(), s.state()
            s.integrate()
            v1 = s.state()
            got = (np.stack([c["idA"], c["idB"], c["type"]], 1), f, st, v1)
            if ref is None:
                ref = got
                continue
            tag = f"force shape {force_shape}, {threads} threads"
            np.testing.assert_array_equal(got[0], ref[0], err_msg=tag)
            for k in ("force", "torque_only_force", "cpA", "cpB"):
                np.testing.assert_array_equal(got[1][k], ref[1][k], err_msg=f"{tag} {k}")
            for k in ("aX", "aY", "aZ", "alphaX", "alphaY", "alphaZ"):
                a, b = got[2][k].astype(np.float64), ref[2][k].astype(np.float64)
                assert np.abs(a - b).max() <= 1e-5 * np.abs(b).max() + 1e-30, (tag, k)
            for k in ("vX", "vY", "vZ"):
                a, b = got[3][k].astype(np.float64), ref[3][k].astype(np.float64)
                assert np.abs(a - b).max() <= 1e-5 * np.abs(b).max() + 1e-30, (tag, k)
    s.close()


def test_autotune_keeps_the_state_and_the_run():
    from deme_b200 import Solver
    built = SCENES["clumps"]()
    a = Solver(built)
    a.step(3)
    before, cb = a.state(), a.contacts()
    t = a.autotune(steps_per_trial=3)
    assert 0 <= t["shape"] < a.lib.deme_search_shape_count() and t["trials"] >= 12
    assert 0 <= t["force_shape"] < a.lib.deme_force_shape_count()
    assert t["exact_threads"] in (128, 256, 512) and t["integrate_threads"] in (128, 256, 512)
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
