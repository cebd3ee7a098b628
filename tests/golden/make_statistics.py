"""Generates tests/golden/statistics.npz: bulk statistics of two long runs of the C oracle, for comparison with the CUDA
path's runs of the same scenes (tests/test_gpu_statistics.py).

Usage:
    python tests/golden/make_statistics.py

Long runs are chaotic: after a few hundred steps two correct solvers (or one solver with float sums in another
order) follow different trajectories, so these runs are compared through bulk quantities, not states:
  * settle: 4,000 spheres of 5 mm falling into a 0.2 x 0.2 x 0.4 m box of six planes (config-1 material), 10,000
    steps at dt 4e-5 (0.4 s): kinetic energy every 250 steps, then the bed's packing fraction and height;
  * collapse: a column (height:width 1) of 3,000 spheres of 2-3 mm with strong rolling resistance (Crr 0.2,
    mu 0.6, so that single spheres come to rest in a heap instead of rolling away) released onto a floor,
    50,000 steps at dt 2e-5 (1 s): kinetic energy every 1,000 steps, then the heap's angle of repose and RMS runout.
"""
from __future__ import annotations

import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
from _util import oracle, workloads  # noqa: E402
from deme_b200 import statistics as stats  # noqa: E402

SETTLE = dict(n=4000, dt=4e-5, seed=11)
SETTLE_STEPS, SETTLE_EVERY = 10000, 250
COLLAPSE = dict(n=3000, dt=2e-5, seed=6, aspect=1.0, domain_widths=8.0, mu=0.6, Crr=0.2)
COLLAPSE_STEPS, COLLAPSE_EVERY = 50000, 1000


def settle_scene():
    return workloads.settling_box(**SETTLE)


def collapse_scene():
    return workloads.column_collapse(**COLLAPSE)


def settle_stats(built, state):
    """Packing fraction of the slab from 2 radii above the floor to 60 % of the bed height, and the bed height."""
    r = SETTLE.get("r", 5e-3)
    box = (0.2, 0.2, 0.4)
    z_floor = -box[2] / 2
    h = stats.bed_height(built, state, z_floor)
    phi = stats.packing_fraction(built, state, (-box[0] / 2, -box[1] / 2), (box[0] / 2, box[1] / 2),
                                 z_floor + 2 * r, z_floor + 0.6 * h)
    return phi, h


def collapse_stats(built, state):
    """Angle of repose (degrees) and RMS horizontal runout from the column axis."""
    z_floor = built.info["z_floor"]
    ring = built.info["lattice_spacing"]
    angle = stats.heap_angle(built, state, (0.0, 0.0), z_floor, ring)
    pos = stats.world_positions(built, state)
    runout = float(np.sqrt(np.mean(pos[:, 0] ** 2 + pos[:, 1] ** 2)))
    return angle, runout


def run(solver, built, steps, every):
    ke = [stats.kinetic_energy(built, solver.state())]
    for _ in range(steps // every):
        solver.step(every)
        ke.append(stats.kinetic_energy(built, solver.state()))
    return np.asarray(ke), solver.state()


def main():
    out = {}
    t = time.time()
    b = settle_scene()
    ke, st = run(oracle(b, threads=os.cpu_count() or 4), b, SETTLE_STEPS, SETTLE_EVERY)
    phi, h = settle_stats(b, st)
    out.update(settle_ke=ke, settle_packing=phi, settle_height=h)
    print(f"settle: packing {phi:.4f}, bed height {h:.4f} m, final KE {ke[-1]:.3e} J ({time.time() - t:.0f} s)")
    t = time.time()
    c = collapse_scene()
    ke, st = run(oracle(c, threads=os.cpu_count() or 4), c, COLLAPSE_STEPS, COLLAPSE_EVERY)
    angle, runout = collapse_stats(c, st)
    out.update(collapse_ke=ke, collapse_angle=angle, collapse_runout=runout)
    print(f"collapse: angle {angle:.2f} deg, runout {runout:.4f} m, final KE {ke[-1]:.3e} J ({time.time() - t:.0f} s)")
    np.savez(os.path.join(HERE, "statistics.npz"), **out)


if __name__ == "__main__":
    main()
