"""Long chaotic runs of the CUDA path against the C oracle, compared through bulk statistics.

After a few hundred steps the two runs follow different trajectories (float sums in another order, then contact
chaos), so states are not compared; the bulk behaviour is.  The oracle's statistics are the fixture
tests/golden/statistics.npz (made by tests/golden/make_statistics.py, whose scenes this test reruns):
  * settle (4,000 spheres falling into a box, 10,000 steps): kinetic-energy curve within 6 % of its peak at every
    sample, final kinetic energy below 0.1 % of the peak, packing fraction of the bed within 0.006, bed height
    within 2 %;
  * collapse (a 3,000-sphere column spreading into a heap, 50,000 steps): kinetic-energy curve within 8 % of its
    peak, angle of repose within 2.5 degrees, RMS runout within 2.5 %.
Measured on a B200: settle 1.7 % / 0.0013 / 0.5 %, collapse 2.3 % / 0.8 degrees / 0.4 %; the bounds leave room
for the run-to-run spread that float atomics give a chaotic run.
"""
import importlib.util
import os

import numpy as np
import pytest

from _util import ROOT

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _generator():
    spec = importlib.util.spec_from_file_location("make_statistics",
                                                  os.path.join(ROOT, "tests", "golden", "make_statistics.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


GEN = _generator()
GOLD = np.load(os.path.join(ROOT, "tests", "golden", "statistics.npz"))


def test_settling_statistics_match_the_oracle():
    from deme_b200 import Solver
    built = GEN.settle_scene()
    g = Solver(built)
    ke, st = GEN.run(g, built, GEN.SETTLE_STEPS, GEN.SETTLE_EVERY)
    phi, h = GEN.settle_stats(built, st)
    ref = GOLD["settle_ke"]
    peak = ref.max()
    dev = np.abs(ke - ref).max() / peak
    print(f"settle: KE curve deviation {dev:.3f} of peak; packing {phi:.4f} vs {float(GOLD['settle_packing']):.4f}; "
          f"height {h:.4f} vs {float(GOLD['settle_height']):.4f}")
    assert dev <= 0.06
    assert ke[-1] <= 1e-3 * peak
    assert abs(phi - float(GOLD["settle_packing"])) <= 0.006
    assert abs(h - float(GOLD["settle_height"])) <= 0.02 * float(GOLD["settle_height"])
    g.close()


def test_column_collapse_statistics_match_the_oracle():
    from deme_b200 import Solver
    built = GEN.collapse_scene()
    g = Solver(built)
    ke, st = GEN.run(g, built, GEN.COLLAPSE_STEPS, GEN.COLLAPSE_EVERY)
    angle, runout = GEN.collapse_stats(built, st)
    ref = GOLD["collapse_ke"]
    dev = np.abs(ke - ref).max() / ref.max()
    print(f"collapse: KE curve deviation {dev:.3f} of peak; angle {angle:.2f} vs "
          f"{float(GOLD['collapse_angle']):.2f} deg; runout {runout:.4f} vs {float(GOLD['collapse_runout']):.4f} m")
    assert dev <= 0.08
    assert abs(angle - float(GOLD["collapse_angle"])) <= 2.5
    assert abs(runout - float(GOLD["collapse_runout"])) <= 0.025 * float(GOLD["collapse_runout"])
    g.close()
