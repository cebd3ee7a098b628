"""The bulk statistics (deme_b200.statistics) on states whose answers are known, no GPU needed."""
import math

import numpy as np

from _util import workloads
from deme_b200 import SceneBuilder
from deme_b200 import statistics as stats


def test_packing_fraction_of_a_simple_cubic_lattice_is_pi_over_six():
    r = 5e-3
    built = workloads.settling_box(n=2000, r=r, spacing=2.0, jitter=0.0)  # 20 x 20 per layer fills the 0.2 m box
    st = built.initial_state()
    floor = -0.2
    phi = stats.packing_fraction(built, st, (-0.1, -0.1), (0.1, 0.1), floor, floor + 5 * 2 * r)
    assert abs(phi - math.pi / 6) < 2e-3, phi
    # a slab cutting every sphere of a layer in half holds half of each: still pi / 6
    phi_half = stats.packing_fraction(built, st, (-0.1, -0.1), (0.1, 0.1), floor + r, floor + 3 * r)
    assert abs(phi_half - math.pi / 6) < 2e-3, phi_half
    assert abs(stats.bed_height(built, st, floor, quantile=1.0) - 5 * 2 * r) < 1e-6


def test_kinetic_energy_of_a_uniform_translation():
    built = workloads.settling_box(n=500, r=5e-3)
    st = built.initial_state()
    st["vX"][:] = 2.0
    m = np.asarray(built.arrays["mass"], np.float64)[:built.info["n_clumps"]]
    assert abs(stats.kinetic_energy(built, st) - 0.5 * 4.0 * m.sum()) < 1e-9 * m.sum()


def test_heap_angle_of_a_cone_of_spheres():
    r = 1e-3
    theta = math.radians(25.0)
    H = 0.04
    pts = []
    for rho in np.arange(0.0, H / math.tan(theta), 1.5 * r):
        n = max(1, int(2 * math.pi * rho / (2.2 * r)))
        for k in range(n):
            a = 2 * math.pi * k / n
            pts.append((rho * math.cos(a), rho * math.sin(a), H - rho * math.tan(theta) - r))
    s = SceneBuilder()
    s.InstructBoxDomainDimension(0.25, 0.25, 0.25)
    s.SetCoordSysOrigin("center")
    mat = s.LoadMaterial({"E": 1e7, "nu": 0.3, "CoR": 0.5, "mu": 0.5, "Crr": 0.0})
    t = s.LoadSphereType(1e-5, r, mat)
    s.AddClumps(t, np.asarray(pts, np.float32))
    s.SetInitTimeStep(1e-5)
    built = s.Initialize()
    angle = stats.heap_angle(built, built.initial_state(), (0.0, 0.0), 0.0, 4 * r)
    assert abs(angle - 25.0) < 1.0, angle
