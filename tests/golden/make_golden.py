"""Generates the golden fixtures in this directory from the reference's own kernel code run on the CPU.

Usage (needs the reference sources, so it runs only where they are mounted):
    python tests/golden/make_golden.py

Each fixture stores a seeded scene (every array of deme_scene plus the parameter struct), the state and contact
history the reference reached after a few warm-up steps, and what the reference produced from there over a few steps
of contact detection, force computation and integration.  Tests replay the scene
through the C oracle (bit-exact) and through the CUDA library.
"""
from __future__ import annotations

import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
from _util import reference, workloads, capi  # noqa: E402

# name: (scene, warm-up steps before recording, recorded steps)
SCENES = {
    "clumps_planes": (lambda: workloads.packed_clumps(n_clumps=150, seed=11, spacing=1.3), 25, 3),
    "spheres_families": (lambda: workloads.packed_clumps(n_clumps=300, seed=12, three=False, families=True,
                                                         beta=2e-4), 25, 3),
    "settle_small": (lambda: workloads.settling_box(n=400, r=5e-3, box=(0.06, 0.06, 0.12), spacing=1.98, jitter=0.02,
                                                    seed=13, vel_scale=0.2, ang_scale=20.0), 5, 4),
}


def params_dict(p) -> dict:
    out = {}
    for name, _ in capi.SimParams._fields_:
        v = getattr(p, name)
        out["param_" + name] = np.array(list(v) if hasattr(v, "__len__") else v)
    return out


def main():
    for name, (make, warm, steps) in SCENES.items():
        built = make()
        ref = reference(built)
        ref.step(warm)
        rec = {"presc": np.frombuffer(bytes(built.prescriptions), np.uint8).copy(), "warmup": np.array(warm)}
        for k, v in ref.state().items():
            rec["pre_st_" + k] = v
        for k, v in ref.contacts().items():
            rec["pre_c_" + k] = v
        rec.update(params_dict(built.params))
        for k, v in built.arrays.items():
            rec["scene_" + k] = v
        rec["counts"] = np.array([built.counts[k] for k in ("o", "s", "a", "m")])
        for step in range(steps):
            ref.detect_contacts()
            c = ref.contacts()
            if step == 0:
                b = ref.bin_assignment()
                for k, v in b.items():
                    rec["bin_" + k] = np.asarray(v)
            ref.compute_forces()
            rec[f"s{step}_cpost_wildcards"] = ref.contacts()["wildcards"]
            f = ref.contact_forces()
            st_forces = ref.state()
            ref.integrate()
            st = ref.state()
            for k, v in c.items():
                rec[f"s{step}_c_{k}"] = v
            for k, v in f.items():
                rec[f"s{step}_f_{k}"] = v
            for k in ("aX", "aY", "aZ", "alphaX", "alphaY", "alphaZ"):
                rec[f"s{step}_acc_{k}"] = st_forces[k]
            for k, v in st.items():
                rec[f"s{step}_st_{k}"] = v
        rec["steps"] = np.array(steps)
        path = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(path, **rec)
        print(f"{name}: {built.counts} contacts/step {[len(rec[f's{s}_c_idA']) for s in range(steps)]} -> {path}")


if __name__ == "__main__":
    main()
