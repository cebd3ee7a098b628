"""The C oracle against the golden fixtures recorded from the reference's own kernels (CPU build).

Bit-exact on every output: bin assignment, contact list (reference order), history mapping, per-contact forces,
torque-only forces, local contact points, owner accelerations and the integrated state.
"""
import numpy as np
import pytest

from _util import GOLDEN, load_golden, oracle


@pytest.mark.parametrize("name", GOLDEN)
def test_oracle_matches_reference_fixture(name):
    built, rec = load_golden(name)
    orc = oracle(built)
    orc.step(int(rec["warmup"]))
    for k, v in orc.state().items():
        np.testing.assert_array_equal(v, rec["pre_st_" + k], err_msg=f"after warm-up: {k}")
    for step in range(int(rec["steps"])):
        orc.detect_contacts()
        c = orc.contacts()
        if step == 0:
            b = orc.bin_assignment()
            for k in ("n_bins", "n_anal", "bins", "spheres"):
                np.testing.assert_array_equal(b[k], rec["bin_" + k], err_msg=k)
        for k in ("idA", "idB", "type", "mapping", "wildcards"):
            np.testing.assert_array_equal(c[k], rec[f"s{step}_c_{k}"], err_msg=f"step {step} {k}")
        orc.compute_forces()
        f = orc.contact_forces()
        for k in ("force", "torque_only_force", "cpA", "cpB"):
            np.testing.assert_array_equal(f[k], rec[f"s{step}_f_{k}"], err_msg=f"step {step} {k}")
        st = orc.state()
        for k in ("aX", "aY", "aZ", "alphaX", "alphaY", "alphaZ"):
            np.testing.assert_array_equal(st[k], rec[f"s{step}_acc_{k}"], err_msg=f"step {step} {k}")
        orc.integrate()
        st = orc.state()
        for k in st:
            np.testing.assert_array_equal(st[k], rec[f"s{step}_st_{k}"], err_msg=f"step {step} {k}")


def test_fixtures_exercise_every_branch():
    """The fixtures contain sphere-sphere and sphere-plane contacts, persistent contacts (non-null mapping),
    and rolling resistance (non-zero torque-only force)."""
    seen_plane = seen_ss = seen_persist = seen_rr = False
    for name in GOLDEN:
        _, rec = load_golden(name)
        for s in range(1, int(rec["steps"])):
            t = rec[f"s{s}_c_type"]
            seen_plane |= bool(np.any(t == 3))
            seen_ss |= bool(np.any(t == 1))
            seen_persist |= bool(np.any(rec[f"s{s}_c_mapping"] != 0xC0000000))
            seen_rr |= bool(np.any(rec[f"s{s}_f_torque_only_force"] != 0))
    assert seen_plane and seen_ss and seen_persist and seen_rr
