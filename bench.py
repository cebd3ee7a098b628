#!/usr/bin/env python
"""Benchmark: M sphere-steps/s of the DEM hot path on the rotating-drum workload (1M three-sphere clumps, 3M
spheres, analytical cylinder + two end planes, 20 rpm), one full step = contact detection + fused Hertz-Mindlin
forces + integration.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--clumps M]

N > 1 runs under torchrun (one process per GPU); every rank advances its own independent drum (replicas only: one
scene does not shard), value = all ranks' sphere-steps / max-over-ranks device time.

Timing: W untimed steps, then K steps bracketed by a barrier and torch.cuda.synchronize(), timed with CUDA events
recorded on the stream the library launches on.  The owner/sphere/contact arrays (several hundred MB) exceed the
126 MB L2, so no explicit flush is done.  A second short pass brackets every kernel with events to get the
per-kernel durations that give the roofline of the dominant kernel; an e2e pass goes through the C ABI with a
pinned host-to-device update of the drum's prescribed rotation and a device-to-host read of the kinetic energy
every step (each step's energy read on the host once the next step is queued).

--impl reference times the reference's CPU path on a bounded sample: its own kernel code compiled for the CPU
(OpenMP on all host cores) on the shell variant of the drum, since the reference has no analytical cylinder (the C
oracle on the analytical drum where that build is absent).  The same line carries `reference_kernels_gpu`: the
reference's own kernels, NVRTC-compiled for sm_100a, on the full-size shell drum, which the main arm also runs
(`shell_drum`) for the comparison against the reference's GPU kernels.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "dem-engine-sbel_b200"))
sys.path.insert(0, ROOT)

METRIC = "M sphere-steps/s"
UNIT = "M sphere-steps/s"


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 50 ms while the timed region runs."""

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self.proc = None

    def start(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits", "-lms",
                                          "50", "-i", str(self.index)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def wait_first(self, timeout: float = 5.0):
        """Block until nvidia-smi has reported once, so that a short timed region is still sampled."""
        t0 = time.perf_counter()
        while self.proc and not self.rows and time.perf_counter() - t0 < timeout:
            time.sleep(0.01)

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.thread.join(timeout=2)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            try:
                sm.append(float(r[1]))
                smax = float(r[2])
                for nm, v in zip(names, r[5:9]):
                    if v.strip().lower() == "active":
                        reasons.add(nm)
            except Exception:
                continue
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def algorithmic_bytes(kernel: str, nS: int, nO: int, nC: int, n_cells: int) -> float:
    """Compulsory HBM bytes of one launch (every array element read or written once per use, SoA)."""
    if kernel == "force":
        # per contact: idA, idB, type (9 B) + history read and write (32 B); per sphere: relPos+radius, owner,
        # material (21 B); per owner: voxel, loc, quat, vel+mass, omega, MOI (80 B) + accumulators (32 B)
        return 41.0 * nC + 21.0 * nS + 112.0 * nO
    if kernel == "pair_find":
        # the candidate scan and the exact test of its survivors: per sphere its cell-order float position + id
        # (16 B), its exact record (position, owner, radius: 32 B), bin ranges + family (16 B), clump run (8 B) and
        # contact count (4 B); the cell table once; per survivor (about one per contact) its pool entry (8 B) and
        # the count update of a found pair (4 B)
        return 76.0 * nS + 4.0 * n_cells + 12.0 * nC
    if kernel == "pair_assemble":
        # scatter: per pair its (A, B) entry (8 B), the count (4 B) and idB written (4 B); assemble: per sphere
        # offsets and analytical count (9 B), per contact idB read and idA, idB, type written (13 B)
        return 9.0 * nS + 29.0 * nC
    if kernel == "integrate":
        return 160.0 * nO
    if kernel == "sort_onesweep":
        return 16.0 * nS
    if kernel == "sphere_prep":
        return (21.0 + 4.0) * nS + 30.0 * nO + (24 + 16 + 8 + 1) * nS
    if kernel == "history":
        return (9.0 + 16.0 + 4.0) * nC + 9.0 * nC + 16.0 * nC
    return 0.0


def build_drum(n_clumps: int, seed: int, spacing: float = 1.02):
    from deme_b200 import workloads
    return workloads.drum(n_clumps=n_clumps, seed=seed, spacing=spacing)


# CPU samples cannot settle the bed first (16,000 steps).  A lattice of pitch 0.745 x the clump diameter gives the
# settled bed's contact density (0.95 sphere-sphere contacts per sphere, measured: 2.86 M contacts on 3 M spheres).
SAMPLE_SPACING = 0.745


def shell_drum(n_clumps: int):
    """The drum as the reference can express it (cylinder replaced by a fixed shell of spheres), on the dense
    lattice that has the settled bed's contact density; both arms run this scene for the reference-kernel
    comparison."""
    from deme_b200 import workloads
    return workloads.drum(n_clumps=n_clumps, shell=True, spacing=SAMPLE_SPACING)


SHELL_WARMUP = 3
SHELL_STEPS = 40
WEDGE_WARMUP = 5
WEDGE_STEPS = 50


def reference_kernels_gpu(args):
    """The reference's own kernels (substituted and NVRTC-compiled from its sources, prebuilt under oracle/_ref) on
    the GPU, on the full-size shell drum.  Device time with CUDA events: first with only the count read-backs the
    next launch needs, then synchronising after every launch as the reference's host code does."""
    try:
        from oracle import ref_gpu
        built = shell_drum(args.clumps)
        if not ref_gpu.prebuilt(built) and not ref_gpu.ref_gpu_build.available():
            return {"unavailable": "reference kernels for this drum size were not prebuilt (needs the reference's "
                                   "sources at build time)"}
        ref = ref_gpu.RefGPU(built, fmad=True)
    except Exception as e:  # the arm must still print its CPU line
        return {"unavailable": f"{type(e).__name__}: {e}"}
    ref.step(SHELL_WARMUP)
    ms = ref.time_steps(SHELL_STEPS)
    nC = ref.num_contacts()
    ref.set_sync_each(True)
    ms_sync = ref.time_steps(SHELL_STEPS // 4)
    ref.set_sync_each(False)
    phases = ref.profile_steps(5)
    # the reference's other contact-kernel variant (SetOneBinPerThread): the better of the two is the baseline
    ref.set_one_bin_per_thread(True)
    ref.step(1)
    ms_thread = ref.time_steps(SHELL_STEPS // 4) / (SHELL_STEPS // 4)
    phases_thread = ref.profile_steps(2)
    ref.close()
    best = min(ms / SHELL_STEPS, ms_thread)
    v = built.n_spheres / (best / 1e3) / 1e6
    return {"value": v, "unit": UNIT, "ms_per_step": best,
            "block_per_bin": {"ms_per_step": ms / SHELL_STEPS, "ms_per_step_sync_each": ms_sync / (SHELL_STEPS // 4),
                              "phase_ms_per_step": phases},
            "thread_per_bin": {"ms_per_step": ms_thread, "phase_ms_per_step": phases_thread},
            "workload": f"drum shell variant: {built.info['n_clumps']} three-sphere clumps + {built.info['n_shell']} "
                        f"fixed shell spheres + 2 end planes, dense lattice (pitch {SAMPLE_SPACING}), dt 5e-6, CD "
                        f"every step",
            "n_spheres": built.n_spheres, "n_contacts": nC, "steps": SHELL_STEPS, "warmup": SHELL_WARMUP,
            "kernels": "reference src/kernel/*.cu substituted per scene, NVRTC sm_100a (FMA default), CUB "
                       "sorts/scans/reduce-by-key; value = the faster of its two contact-kernel variants"}


def reference_kernels_quick(args, which: str):
    """The reference's kernels (thread per bin) on the shell drum or the wedge hopper, for the main line's ratio."""
    try:
        from oracle import ref_gpu
        from deme_b200 import workloads
        built = shell_drum(args.clumps) if which == "shell" else workloads.hopper_wedge(n=args.hopper_spheres)
        if not ref_gpu.prebuilt(built) and not ref_gpu.ref_gpu_build.available():
            return {"unavailable": "reference kernels for this scene were not prebuilt"}
        ref = ref_gpu.RefGPU(built, fmad=True)
    except Exception as e:
        return {"unavailable": f"{type(e).__name__}: {e}"}
    try:
        warm, steps = (SHELL_WARMUP, SHELL_STEPS // 4) if which == "shell" else (WEDGE_WARMUP, WEDGE_STEPS)
        ref.set_one_bin_per_thread(True)
        ref.step(warm)
        ms = ref.time_steps(steps)
        nC = ref.num_contacts()
    except Exception as e:
        ref.close()
        return {"unavailable": f"{type(e).__name__}: {e}"}
    ref.close()
    return {"value": built.n_spheres * steps / (ms / 1e3) / 1e6, "unit": UNIT, "ms_per_step": ms / steps,
            "n_spheres": built.n_spheres, "n_contacts": nC, "steps": steps, "warmup": warm,
            "kernels": "reference src/kernel/*.cu substituted per scene, NVRTC sm_100a (FMA default), CUB; thread "
                       "per bin"}


def reference_kernels_wedge(args):
    """The reference's own kernels on the GPU on the plane-only wedge hopper (4M log-normal spheres, CD every 5
    steps), its thread-per-bin contact kernels (the faster variant on the drum), from the lattice start."""
    try:
        from oracle import ref_gpu
        from deme_b200 import workloads
        built = workloads.hopper_wedge(n=args.hopper_spheres)
        if not ref_gpu.prebuilt(built) and not ref_gpu.ref_gpu_build.available():
            return {"unavailable": "reference kernels for the wedge hopper were not prebuilt (needs the reference's "
                                   "sources at build time)"}
        ref = ref_gpu.RefGPU(built, fmad=True)
    except Exception as e:
        return {"unavailable": f"{type(e).__name__}: {e}"}
    try:
        ref.set_one_bin_per_thread(True)
        ref.step(WEDGE_WARMUP)
        ms = ref.time_steps(WEDGE_STEPS)
        nC = ref.num_contacts()
        phases = ref.profile_steps(10)
    except Exception as e:
        ref.close()
        return {"unavailable": f"{type(e).__name__}: {e}"}
    ref.close()
    return {"value": built.n_spheres * WEDGE_STEPS / (ms / 1e3) / 1e6, "unit": UNIT, "ms_per_step": ms / WEDGE_STEPS,
            "workload": wedge_workload(built), "n_spheres": built.n_spheres, "n_contacts": nC, "steps": WEDGE_STEPS,
            "warmup": WEDGE_WARMUP, "phase_ms_per_step": phases,
            "kernels": "reference src/kernel/*.cu substituted per scene, NVRTC sm_100a (FMA default), CUB; thread "
                       "per bin"}


def run_reference(args):
    """The reference's CPU path on a bounded sample: its own kernel code compiled for the CPU (oracle/_ref, OpenMP
    over the emulated blocks) on the shell variant of the drum, or, where that build is absent, the C oracle on the
    analytical drum.  Also times the reference's kernels on the GPU on the full-size shell drum."""
    from deme_b200 import HandleSolver, capi
    cores = os.cpu_count() or 1
    n_clumps = min(args.clumps, args.ref_clumps)
    built = shell_drum(n_clumps)
    try:
        from oracle import ref_build
        lib_path = ref_build.lookup(built)
    except Exception:
        lib_path = None
    if lib_path:
        kind, prefix, who = "reference", "ref_", "the reference's kernel code compiled for the CPU (oracle/_ref)"
        wl = f"drum shell variant ({n_clumps} clumps + {built.info['n_shell']} shell spheres)"
    else:
        lib_path = os.path.join(ROOT, "oracle", "_build", "libdeme_oracle.so")
        if not os.path.exists(lib_path):
            subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "oracle")])
        built = build_drum(n_clumps, seed=1, spacing=SAMPLE_SPACING)
        kind, prefix, who = "port", "orc_", "the C oracle"
        wl = f"rotating drum ({n_clumps} clumps)"
    cpu = HandleSolver(capi.load_library(lib_path), prefix, built, threads=cores)
    w = max(1, min(args.warmup, 2))
    k = max(1, min(args.steps, args.ref_steps))
    cpu.step(w)
    t0 = time.perf_counter()
    cpu.step(k)
    dt = time.perf_counter() - t0
    v = built.n_spheres * k / dt / 1e6
    sample = (f"{wl} on the dense lattice (pitch {SAMPLE_SPACING} x clump diameter, settled-bed contact density): "
              f"{built.n_spheres} spheres, {cpu.num_contacts()} contacts, {k} timed steps after {w} warm-up steps, "
              f"{who}, OpenMP {cores} threads")
    cpu.close()
    gpu = reference_kernels_gpu(args) if not args.no_reference_gpu else None
    wedge = reference_kernels_wedge(args) if not args.no_reference_gpu and not args.no_hopper else None
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": k,
            "warmup": w, "ms_per_step": dt / k * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 forces, f64 positions, integer voxels", "data": "synthetic (seeded)",
            "config": {"workload": wl + " (CPU sample)", "n_clumps": n_clumps, "n_spheres": built.n_spheres},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "reference_kernels_gpu": gpu, "reference_kernels_gpu_hopper_wedge": wedge}
    print(json.dumps(line), flush=True)


def hopper_measure(args, stream):
    """Hopper discharge: 4M log-normal spheres in an analytical cone, contact detection every 5 steps with a margin
    of 0.1 median radius.  The seeded packing settles first with the outlet gate closed (untimed, --hopper-settle
    steps at dt 6e-6); then the gate opens (its family changes to one that has no contact with the spheres, as the
    reference's ChangeFamily + DisableContactBetweenFamilies do) and the discharge runs --hopper-steps steps at
    dt 2e-6 twice from the same opened bed: with synchronous detection, and with kT and dT on two streams (a
    detection adopted 5 steps after the poses it was made from).  Device time with CUDA events; the per-kernel
    shares of the synchronous run come from deme_kernel_timing over two detection periods."""
    import numpy as np
    import torch
    from deme_b200 import Solver, workloads
    built = workloads.hopper(n=args.hopper_spheres)
    f = int(built.params.cd_update_freq)
    dt_run = float(built.params.h)
    kt = torch.cuda.Stream()
    s = Solver(built)
    s.lib.deme_set_streams(s.h, C.c_void_p(kt.cuda_stream), C.c_void_p(stream.cuda_stream))
    t0 = time.perf_counter()
    if args.hopper_settle > 0:
        s.set_time_step(6e-6)
        s.step(args.hopper_settle)
        s.set_time_step(dt_run)
    s.sync()
    prep_s = time.perf_counter() - t0
    s.change_family(2, workloads.GATE_OPEN_FAMILY)  # the gate opens
    bed_state, bed_contacts = s.state(), s.contacts()
    apex = float(built.info["apex_z"])
    u_out = float(built.info["u_out"])
    out = {"workload": f"hopper discharge: {built.n_spheres} spheres, log-normal radii (median 1.5 mm, sigma 0.25), "
                       f"30 deg cone, 40 mm outlet opened after settling, dt {dt_run:g}, CD every {f} steps, margin "
                       f"0.1 median radius",
           "initial_state": f"seeded lattice packing settled {args.hopper_settle} steps at dt 6e-6 with the gate "
                            f"closed (untimed, {prep_s:.1f} s), then the gate opened",
           "n_spheres": built.n_spheres, "steps": args.hopper_steps, "warmup": 2 * f}
    for lag in (0, f):
        s.set_state({k: v for k, v in bed_state.items() if not k.startswith("a")})
        s.set_contacts({k: bed_contacts[k] for k in ("idA", "idB", "type", "wildcards")})
        s.set_async_cd(lag)
        s.step(2 * f)
        s.sync()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        s.step(args.hopper_steps)
        s.sync()  # adopts a pending detection: its kT work is inside the timed region
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        key = "sync" if lag == 0 else "two_streams"
        z = built.decode_positions(s.state(), kernel_literals=False)[:built.n_spheres, 2]
        lbf_z = float(built.params.lbf[2])
        out[key] = {"lag": lag, "ms_per_step": ms / args.hopper_steps,
                    "value": built.n_spheres * args.hopper_steps / (ms / 1e3) / 1e6, "unit": UNIT,
                    "n_contacts": s.num_contacts(),
                    "spheres_below_outlet": int(np.sum(z + lbf_z < apex + u_out))}
        if lag == 0:
            ks = kernel_breakdown(s, 2 * f)
            tot = sum(ks.values())
            out["kernel_ms_per_step"] = ks
            out["history_share"] = ks.get("history", 0.0) / tot if tot > 0 else None
        s.set_async_cd(0)
    s.close()
    return out


def kernel_breakdown(s, steps: int) -> dict:
    """Per-kernel device milliseconds per step over `steps` steps (deme_kernel_timing brackets every launch)."""
    lib = s.lib
    lib.deme_kernel_timing(1)
    s.step(steps)
    s.sync()
    names = (C.c_char_p * 32)()
    tot = (C.c_double * 32)()
    cnt = (C.c_int64 * 32)()
    nk = C.c_int32(0)
    lib.deme_kernel_times(32, names, tot, cnt, C.byref(nk))
    lib.deme_kernel_timing(0)
    return {names[i].decode(): tot[i] / steps for i in range(nk.value) if cnt[i] > 0}


def hopper_wedge_measure(args, stream):
    """This build on the plane-only wedge hopper (the same 4M log-normal spheres, volume equal to the cone's) from its
    lattice start with the gate closed, CD every 5 steps: the scene the reference's kernels are timed on for the
    polydisperse hopper workload."""
    import torch
    from deme_b200 import Solver, workloads
    built = workloads.hopper_wedge(n=args.hopper_spheres)
    s = Solver(built)
    s.lib.deme_set_streams(s.h, C.c_void_p(stream.cuda_stream), C.c_void_p(stream.cuda_stream))
    s.step(WEDGE_WARMUP)
    s.sync()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    s.step(WEDGE_STEPS)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    nC = s.num_contacts()
    s.close()
    return {"value": built.n_spheres * WEDGE_STEPS / (ms / 1e3) / 1e6, "unit": UNIT, "ms_per_step": ms / WEDGE_STEPS,
            "workload": wedge_workload(built), "n_spheres": built.n_spheres, "n_contacts": nC, "steps": WEDGE_STEPS,
            "warmup": WEDGE_WARMUP}


def wedge_workload(built) -> str:
    return (f"wedge hopper (planes only): {built.n_spheres} log-normal spheres, 30 deg walls, 40 mm outlet slot "
            f"(gate closed), length {built.info['L']:.3f} m for the cone's volume {built.info['cone_volume']:.4f} "
            f"m^3, lattice start, dt 2e-6, CD every 5 steps, margin 0.1 median radius")


def small_scene_measure(args, stream):
    """The small settling box (10,000 spheres of 5 mm in a 0.2 x 0.2 x 0.4 m box of six planes, dt 1e-5, CD every
    step): steps launched one by one, and whole steps replayed from CUDA graphs.  Device time with CUDA events after
    1,000 untimed steps."""
    import torch
    from deme_b200 import Solver, workloads
    built = workloads.settling_box(n=10000)
    out = {"workload": "settling box: 10,000 spheres r 5 mm, 0.2 x 0.2 x 0.4 m box of 6 planes, dt 1e-5, CD every step",
           "n_spheres": built.n_spheres, "steps": args.small_steps, "warmup": 1000}
    for graph in (False, True):
        s = Solver(built)
        s.lib.deme_set_streams(s.h, C.c_void_p(stream.cuda_stream), C.c_void_p(stream.cuda_stream))
        if graph:
            s.set_graph(True)
        s.step(1000)
        s.sync()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        s.step(args.small_steps)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        out["graph" if graph else "step_by_step"] = {
            "us_per_step": ms * 1e3 / args.small_steps,
            "value": built.n_spheres * args.small_steps / (ms / 1e3) / 1e6, "unit": UNIT,
            "n_contacts": s.num_contacts(), "graph_windows_replayed": s.graph_stats()[0]}
        s.close()
    return out


def shell_drum_measure(args, stream):
    """This build on the same shell drum the reference's GPU kernels are timed on (device time, CUDA events)."""
    import torch
    from deme_b200 import Solver
    built = shell_drum(args.clumps)
    s = Solver(built)
    s.lib.deme_set_streams(s.h, C.c_void_p(stream.cuda_stream), C.c_void_p(stream.cuda_stream))
    s.step(SHELL_WARMUP)
    s.sync()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    s.step(SHELL_STEPS)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    nC = s.num_contacts()
    s.close()
    return {"value": built.n_spheres * SHELL_STEPS / (ms / 1e3) / 1e6, "unit": UNIT, "ms_per_step": ms / SHELL_STEPS,
            "workload": f"drum shell variant: {built.info['n_clumps']} three-sphere clumps + {built.info['n_shell']} "
                        f"fixed shell spheres + 2 end planes, dense lattice (pitch {SAMPLE_SPACING}), dt 5e-6, CD "
                        f"every step",
            "n_spheres": built.n_spheres, "n_contacts": nC, "steps": SHELL_STEPS, "warmup": SHELL_WARMUP}


def mesh_drop_measure(args, stream):
    """Sphere--mesh contacts at scale: a free icosphere of 20,480 facets (radius 0.1 m) driven at 1 m/s, 1 mm deep,
    into a packed bed of ``--mesh-spheres`` spheres (r 2 mm, simple cubic, 20 layers, each sphere pressed into its
    neighbours) in a box of planes, dt 2e-6, CD every step; then the same bed without the ball, for the cost of the
    mesh.  Device time with CUDA events after 200 untimed steps, and the per-kernel split.  The reference detects no
    sphere--mesh contact, so there is no reference time for this scene."""
    import numpy as np
    import torch
    from deme_b200 import Solver, capi, workloads
    out = {}
    for ball in (True, False):
        built = workloads.mesh_ball_drop(n=args.mesh_spheres, ball_radius=0.1, subdivisions=5, layers=20, press=0.5,
                                         packed=True, ball=ball)
        s = Solver(built)
        s.lib.deme_set_streams(s.h, C.c_void_p(stream.cuda_stream), C.c_void_p(stream.cuda_stream))
        s.step(200)
        s.sync()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        s.step(args.mesh_steps)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        c = s.contacts()
        split = kernel_breakdown(s, 20)
        s.close()
        r = {"value": built.n_spheres * args.mesh_steps / (ms / 1e3) / 1e6, "unit": UNIT,
             "ms_per_step": ms / args.mesh_steps, "n_spheres": built.n_spheres, "n_contacts": len(c["idA"]),
             "kernel_ms_per_step": {k: round(v, 4) for k, v in sorted(split.items(), key=lambda kv: -kv[1])}}
        if ball:
            r.update(workload=f"mesh ball drop: icosphere of {built.info['n_tris']} facets (r 0.1 m, free, 1 m/s, "
                              f"pressed 1 mm) into {built.n_spheres} packed spheres (r 2 mm, 20 layers) in a box of 5 "
                              f"planes, dt 2e-6, CD every step",
                     n_facets=built.info["n_tris"],
                     n_sphere_mesh_contacts=int(np.sum(c["type"] == capi.SPHERE_MESH_CONTACT)),
                     steps=args.mesh_steps, warmup=200,
                     reference="unavailable: the reference declares the sphere--mesh contact type but detects no "
                               "such contact")
            out.update(r)
        else:
            out["same_bed_without_mesh"] = r
    return out


def mesh_drum_measure(args, stream, settled: dict):
    """The benchmark drum with its cylinder as a mesh body (`workloads.drum(mesh=True)`: a prism of flat facets
    touching the radius-R circle, turning with the end planes), started from the analytical drum's settled clumps,
    against the analytical drum from the same state, both launched step by step (meshes step without CUDA graphs):
    device time with CUDA events over ``--mesh-steps`` steps after 200 untimed ones (the first detects afresh)."""
    import numpy as np
    import torch
    from deme_b200 import Solver, capi, workloads
    out = {}
    for mesh in (True, False):
        built = workloads.drum(n_clumps=args.clumps, seed=2, mesh=mesh)
        s = Solver(built)
        s.lib.deme_set_streams(s.h, C.c_void_p(stream.cuda_stream), C.c_void_p(stream.cuda_stream))
        nC = built.info["n_clumps"]
        st = s.state()
        for k, v in settled.items():
            if not k.startswith("a"):
                st[k][:nC] = v[:nC]
        s.set_state({k: v for k, v in st.items() if not k.startswith("a")})
        s.step(200)
        s.sync()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        s.step(args.mesh_steps)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        c = s.contacts()
        r = {"value": built.n_spheres * args.mesh_steps / (ms / 1e3) / 1e6, "unit": UNIT,
             "ms_per_step": ms / args.mesh_steps, "n_contacts": len(c["idA"]),
             "kernel_ms_per_step": {k: round(v, 4) for k, v in
                                    sorted(kernel_breakdown(s, 20).items(), key=lambda kv: -kv[1])}}
        s.close()
        if mesh:
            r.update(workload=f"rotating drum, {nC} three-sphere clumps, cylinder as a mesh of {built.info['n_tris']} "
                              f"facets turning at 20 rpm with the end planes, dt 5e-6, CD every step, from the "
                              f"settled bed, kernels launched step by step",
                     n_facets=built.info["n_tris"],
                     n_sphere_mesh_contacts=int(np.sum(c["type"] == capi.SPHERE_MESH_CONTACT)),
                     steps=args.mesh_steps, warmup=200)
            out.update(r)
        else:
            out["analytical_cylinder_same_state"] = r
    return out


def cpu_baseline_sample(args):
    from deme_b200 import HandleSolver, capi
    lib_path = os.path.join(ROOT, "oracle", "_build", "libdeme_oracle.so")
    if not os.path.exists(lib_path):
        subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "oracle")])
    cores = os.cpu_count() or 1
    n_clumps = min(args.clumps, args.ref_clumps)
    built = build_drum(n_clumps, seed=1, spacing=SAMPLE_SPACING)
    orc = HandleSolver(capi.load_library(lib_path), "orc_", built, threads=cores)
    orc.step(1)
    k = max(1, args.ref_steps)
    t0 = time.perf_counter()
    orc.step(k)
    dt = time.perf_counter() - t0
    return {"value": built.n_spheres * k / dt / 1e6, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"C oracle (OpenMP, {cores} threads) on a dense drum lattice (pitch {SAMPLE_SPACING} x clump "
                      f"diameter, settled-bed contact density) with {n_clumps} clumps ({built.n_spheres} spheres, "
                      f"{orc.num_contacts()} contacts), {k} steps after 1 warm-up step"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--clumps", type=int, default=1_000_000)
    ap.add_argument("--ref-clumps", type=int, default=200_000)
    ap.add_argument("--ref-steps", type=int, default=10)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-shell", action="store_true", help="skip the shell-drum run (the reference-kernel comparison)")
    ap.add_argument("--no-hopper", action="store_true", help="skip the hopper run (detection every 5 steps, two streams)")
    ap.add_argument("--no-small", action="store_true", help="skip the small-scene run (step by step against graphs)")
    ap.add_argument("--autotune", type=int, default=1, help="1: pick the search shape with deme_autotune (untimed)")
    ap.add_argument("--graph", type=int, default=1, help="1: replay whole steps from CUDA graphs (deme_set_graph)")
    ap.add_argument("--small-steps", type=int, default=5000)
    ap.add_argument("--hopper-spheres", type=int, default=4_000_000)
    ap.add_argument("--hopper-steps", type=int, default=5000)
    ap.add_argument("--hopper-settle", type=int, default=40000, help="untimed settling steps of the hopper bed")
    ap.add_argument("--no-reference-gpu", action="store_true",
                    help="reference arm: skip timing the reference's kernels on the GPU")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint timing on the column collapse")
    ap.add_argument("--adjoint-steps", type=int, default=2000)
    ap.add_argument("--adjoint-checkpoint", type=int, default=100)
    ap.add_argument("--adjoint-drum-clumps", type=int, default=100_000,
                    help="clumps of the turning drum whose adjoint is timed beside the column collapse (0: skip)")
    ap.add_argument("--adjoint-drum-steps", type=int, default=400)
    ap.add_argument("--no-mesh", action="store_true", help="skip the sphere--mesh ball-drop measurement")
    ap.add_argument("--mesh-spheres", type=int, default=1_000_000)
    ap.add_argument("--mesh-steps", type=int, default=1000)
    ap.add_argument("--no-batched", action="store_true", help="skip the packed multi-scene measurement")
    ap.add_argument("--batch-scenes", type=int, default=512)
    ap.add_argument("--batch-steps", type=int, default=1000)
    ap.add_argument("--batch-checkpoint", type=int, default=100)
    ap.add_argument("--batch-sample", type=int, default=12)
    ap.add_argument("--settle-steps", type=int, default=15000,
                    help="untimed preparation: steps at --settle-dt that let the loose lattice fall into a bed")
    ap.add_argument("--settle-dt", type=float, default=2e-5)
    ap.add_argument("--calm-steps", type=int, default=1000, help="untimed steps at the workload's dt after settling")
    ap.add_argument("--save-state", default=None, help="write the prepared state and contact history to this .npz")
    ap.add_argument("--load-state", default=None, help="start from a state written by --save-state (no settling)")
    args = ap.parse_args()
    if args.load_state:
        args.settle_steps = 0
        args.calm_steps = 0

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank == 0:
            run_reference(args)
        return

    import torch
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    from deme_b200 import Solver, capi

    built = build_drum(args.clumps, seed=2 + rank)
    s = Solver(built)
    lib = s.lib
    lib.deme_launch_count.restype = C.c_int64
    lib.deme_kernel_timing.argtypes = [C.c_int32]
    lib.deme_kernel_times.argtypes = [C.c_int32, C.POINTER(C.c_char_p), C.POINTER(C.c_double),
                                      C.POINTER(C.c_int64), C.POINTER(C.c_int32)]
    lib.deme_set_streams.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    lib.deme_set_family_prescription.argtypes = [C.c_void_p, C.c_int32, C.POINTER(capi.FamilyPrescription)]
    stream = torch.cuda.Stream()
    lib.deme_set_streams(s.h, C.c_void_p(stream.cuda_stream), C.c_void_p(stream.cuda_stream))

    # ---- scene preparation (untimed): let the loose lattice settle into a bed ----
    t_prep = time.perf_counter()
    dt_work = float(built.params.h)
    if args.load_state:
        import numpy as np
        z = np.load(args.load_state)
        s.set_state({k[3:]: z[k] for k in z.files if k.startswith("st_")})
        s.set_contacts({k[2:]: z[k] for k in z.files if k.startswith("c_")})
    if args.settle_steps > 0:
        s.set_time_step(args.settle_dt)
        done = 0
        while done < args.settle_steps:
            chunk = min(1000, args.settle_steps - done)
            s.step(chunk)
            done += chunk
            if rank == 0:
                s.sync()
                print(f"[prepare] settled {done} steps, {s.num_contacts()} contacts, "
                      f"{time.perf_counter() - t_prep:.1f} s", file=sys.stderr, flush=True)
        s.set_time_step(dt_work)
    if args.calm_steps > 0:
        s.step(args.calm_steps)
    s.sync()
    prep_s = time.perf_counter() - t_prep
    if args.save_state and rank == 0:
        import numpy as np
        st = s.state()
        c = s.contacts()
        np.savez(args.save_state, **{"st_" + k: v for k, v in st.items() if not k.startswith("a")},
                 **{"c_" + k: c[k] for k in ("idA", "idB", "type", "wildcards")})

    if args.graph:
        s.set_graph(True)  # whole steps replayed from CUDA graphs (no host synchronisation inside a step)
    tuning = None
    if args.autotune:
        # untimed: time every search shape on a few steps from the prepared state, keep the fastest, restore the state
        tuning = s.autotune(steps_per_trial=10)

    # ---- warm-up (the clock sampler starts here so it has samples when the timed region is short) ----
    sampler = ClockSampler(local_rank)
    sampler.start()
    sampler.wait_first()
    s.step(args.warmup)
    s.sync()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()

    # ---- timed region ----
    n0 = lib.deme_launch_count()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    ev0.record(stream)
    s.step(args.steps)
    ev1.record(stream)
    torch.cuda.synchronize()
    launches = lib.deme_launch_count() - n0
    clocks = sampler.stop()
    ms = ev0.elapsed_time(ev1)
    nC = s.num_contacts()
    t = torch.tensor([ms], dtype=torch.float64, device="cuda")
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.barrier()
    ms_max = float(t.item())
    value = world * built.n_spheres * args.steps / (ms_max / 1e3) / 1e6

    # ---- per-kernel device times (roofline of the dominant kernel) ----
    k_steps = min(args.steps, 5)
    lib.deme_kernel_timing(1)
    s.step(k_steps)
    s.sync()
    names = (C.c_char_p * 32)()
    tot = (C.c_double * 32)()
    cnt = (C.c_int64 * 32)()
    nk = C.c_int32(0)
    lib.deme_kernel_times(32, names, tot, cnt, C.byref(nk))
    lib.deme_kernel_timing(0)
    kernels = {names[i].decode(): (tot[i], cnt[i]) for i in range(nk.value) if cnt[i] > 0}
    dominant = max(kernels, key=lambda k: kernels[k][0])
    d_ms, d_cnt = kernels[dominant]
    n_cells = int(s_grid_cells(built))
    bytes_per_launch = algorithmic_bytes(dominant, built.n_spheres, built.n_owners, s.num_contacts(), n_cells)
    avg_s = d_ms / d_cnt / 1e3
    peak, peak_kind = peaks()
    achieved = bytes_per_launch / avg_s / 1e9 if avg_s > 0 else 0.0
    traffic = read_traffic(dominant, built.n_spheres, s.num_contacts())
    roofline = {"bound": "hbm", "kernel": dominant, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_source": peak_kind, "traffic": traffic,
                "algorithmic_bytes_per_launch": bytes_per_launch, "avg_launch_ms": avg_s * 1e3,
                "kernel_ms_per_step": {k: v[0] / k_steps for k, v in kernels.items()}}

    # ---- e2e through the C ABI with host buffers ----
    drum_fam = 10
    presc = capi.FamilyPrescription()
    base = built.prescriptions[drum_fam]
    C.memmove(C.byref(presc), C.byref(base), C.sizeof(presc))
    ke = C.c_double(0.0)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    # every step: its input staged from pinned host memory, and its result (the kinetic energy) copied back and
    # read on the host; the read of step k waits only for step k, after step k + 1 has been queued
    prev = None
    for _ in range(args.steps):
        lib.deme_set_family_prescription(s.h, drum_fam, C.byref(presc))
        s.step(1)
        ticket = s.kinetic_energy_enqueue()
        if prev is not None:
            ke_val = s.kinetic_energy_collect(prev)
        prev = ticket
    ke_val = s.kinetic_energy_collect(prev)
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    te = torch.tensor([e2e_s], dtype=torch.float64, device="cuda")
    if dist:
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
    e2e_value = world * built.n_spheres * args.steps / float(te.item()) / 1e6

    def clocked(fn):
        """Runs a section with the SM clocks and throttle reasons sampled during it."""
        sampler = ClockSampler(local_rank)
        sampler.start()
        sampler.wait_first()
        out = fn()
        c = sampler.stop()
        if isinstance(out, dict):
            out["clocks"] = c
        return out

    # the adjoint and batched targets first, before the long hopper run heats the GPU
    adj = None if args.no_adjoint else clocked(lambda: adjoint_measure(args, stream))
    batched = None if args.no_batched else clocked(lambda: batched_measure(args, stream, rank, world, dist))
    shell = clocked(lambda: shell_drum_measure(args, stream)) if (rank == 0 and not args.no_shell) else None
    # the reference's kernels on the same shell drum (thread per bin, its faster variant), for the ratio
    ref_shell = reference_kernels_quick(args, "shell") if (rank == 0 and not args.no_shell) else None
    hopper = clocked(lambda: hopper_measure(args, stream)) if (rank == 0 and not args.no_hopper) else None
    wedge = clocked(lambda: hopper_wedge_measure(args, stream)) if (rank == 0 and not args.no_hopper) else None
    ref_wedge = reference_kernels_quick(args, "wedge") if (rank == 0 and not args.no_hopper) else None
    small = clocked(lambda: small_scene_measure(args, stream)) if (rank == 0 and not args.no_small) else None
    mesh = None
    # one GPU only: in a multi-GPU run the other ranks would wait at the closing barrier through it
    if rank == 0 and world == 1 and not args.no_mesh:
        try:
            mesh = clocked(lambda: mesh_drop_measure(args, stream))
        except Exception as e:  # the headline line is printed whatever happens to this secondary measurement
            mesh = {"unavailable": f"{type(e).__name__}: {e}"}
        try:
            settled = s.state()
            mesh["drum"] = clocked(lambda: mesh_drum_measure(args, stream, settled))
        except Exception as e:
            mesh["drum"] = {"unavailable": f"{type(e).__name__}: {e}"}
    # the CPU sample last: its OpenMP threads would otherwise share the host with the GPU sections' host code
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_sample(args)

    if rank == 0:
        def versus(ours, ref):
            if not ours or not ref or "value" not in ours or "value" not in ref:
                return {"unavailable": (ref or {}).get("unavailable", "not measured")}
            return {"this_build": ours["value"], "reference_kernels": ref["value"], "ratio": ours["value"] / ref["value"],
                    "unit": UNIT, "workload": ours["workload"]}

        line = {
            "metric": METRIC, "value": value, "unit": UNIT,
            # the same scene run by the reference's own kernels on this GPU (printed early, ahead of the details)
            "vs_reference_kernels": {"shell_drum": versus(shell, ref_shell), "hopper_wedge": versus(wedge, ref_wedge)},
            "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 forces/velocities, f64 positions on integer voxels",
            "data": "synthetic (seeded drum generator)",
            "config": {"workload": "rotating drum: 1M three-sphere clumps (3M spheres), analytical cylinder + 2 end "
                                   "planes, 20 rpm, dt 5e-6, CD every step" if args.clumps == 1_000_000 else
                       f"rotating drum: {args.clumps} three-sphere clumps",
                       "n_clumps": built.info["n_clumps"], "n_spheres": built.n_spheres,
                       "n_contacts": nC, "drum_R_m": built.info["R"], "drum_L_m": built.info["L"],
                       "initial_state": f"HCP lattice of non-overlapping clumps, settled {args.settle_steps} steps at "
                                        f"dt {args.settle_dt:g} + {args.calm_steps} steps at dt {dt_work:g} "
                                        f"(untimed, {prep_s:.1f} s)",
                       "l2": "inputs larger than L2 (no flush)", "parallelism": f"replicas x{world}",
                       "search_shape": tuning, "cuda_graphs": bool(args.graph)},
            "roofline": roofline, "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": C.sizeof(capi.FamilyPrescription),
                    "d2h_bytes_per_step": 8},
            "gpu_launches": int(launches), "clocks": clocks, "shell_drum": shell, "reference_kernels_shell_drum": ref_shell,
            "hopper": hopper, "hopper_wedge": wedge, "reference_kernels_hopper_wedge": ref_wedge, "small_scene": small,
            "adjoint": adj, "batched": batched, "mesh": mesh,
        }
        print(json.dumps(line), flush=True)
    s.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def adjoint_measure(args, stream):
    """Adjoint timing on the column collapse: plain forward steps, the checkpointed forward (record) and the
    backward pass (segment recomputation + reverse), each timed with CUDA events on the solver's stream."""
    import numpy as np
    import torch
    from deme_b200 import Solver, adjoint, workloads
    built = workloads.column_collapse()
    T, K = args.adjoint_steps, args.adjoint_checkpoint
    n = built.counts["s"]

    def solver():
        s = Solver(built)
        s.lib.deme_set_streams(s.h, C.c_void_p(stream.cuda_stream), C.c_void_p(stream.cuda_stream))
        return s

    def timed(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        r = fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1), r

    w = solver()  # warm-up: allocations and first launches of every kernel involved
    adjoint.record(w, min(T, 2 * K), K)
    adjoint.backward(w, d_pos=np.zeros((built.counts["o"], 3)))
    w.close()
    sf = solver()
    t_fwd, _ = timed(lambda: sf.step(T))
    sf.close()
    sa = solver()
    t_rec, _ = timed(lambda: adjoint.record(sa, T, K))
    pos, _, _ = adjoint.final_state(sa)
    init = built.decode_positions(built.initial_state(), kernel_literals=False)[:n]
    loss, g = workloads.collapse_loss(pos[:n], init[:, :2].mean(0), float(init[:, 2].min()))
    seed = np.zeros((built.counts["o"], 3))
    seed[:n] = g
    t_bwd, out = timed(lambda: adjoint.backward(sa, d_pos=seed))
    nC = sa.num_contacts()
    sa.close()
    res = {"workload": "column collapse: 20,000 spheres r U[2,3] mm released over a floor plane, dt 1e-5, CD every "
                       "step, contact margin 0", "steps": T, "checkpoint_every": K, "fwd_ms_per_step": t_fwd / T,
           "record_ms_per_step": t_rec / T, "adjoint_ms_per_step": t_bwd / T, "adjoint_over_forward": t_bwd / t_fwd,
           "loss": loss, "dL_dE_CoR_mu_Crr": [float(v) for v in out["d_material"][0]], "n_contacts_final": nC,
           "gradient_precision": "FP64 accumulators, FP32 state"}
    if args.adjoint_drum_clumps > 0:
        res["drum"] = adjoint_drum_measure(args, stream, timed)
    return res


def adjoint_drum_measure(args, stream, timed):
    """Adjoint of the turning drum (three-sphere clumps, analytical cylinder and end planes turning at 20 rpm,
    friction and rolling resistance) from a settled bed: loss = mean clump height after the window; the backward
    pass (segment recomputation + reverse) against the plain forward window, both timed with CUDA events."""
    import numpy as np
    from deme_b200 import Solver, adjoint, workloads
    built = workloads.drum(n_clumps=args.adjoint_drum_clumps)
    T, K = args.adjoint_drum_steps, 100
    s = Solver(built)
    s.lib.deme_set_streams(s.h, C.c_void_p(stream.cuda_stream), C.c_void_p(stream.cuda_stream))
    h0 = float(built.params.h)
    s.set_time_step(2e-5)
    s.step(15000)
    s.set_time_step(h0)
    s.sync()
    st = {k: v for k, v in s.state().items() if not k.startswith("a")}
    c = {k: np.array(v, copy=True) for k, v in s.contacts().items() if k in ("idA", "idB", "type", "wildcards")}
    nC0 = s.num_contacts()
    adjoint.record(s, 2 * K, K)  # warm-up: allocations and first launches
    seed = np.zeros((built.counts["o"], 3))
    seed[:args.adjoint_drum_clumps, 2] = 1.0 / args.adjoint_drum_clumps
    adjoint.backward(s, d_pos=seed)
    s.set_state(st)
    s.set_contacts(c)
    t_fwd, _ = timed(lambda: s.step(T))
    s.set_state(st)
    s.set_contacts(c)
    t_rec, _ = timed(lambda: adjoint.record(s, T, K))
    t_bwd, out = timed(lambda: adjoint.backward(s, d_pos=seed))
    s.close()
    return {"workload": f"turning drum: {args.adjoint_drum_clumps} three-sphere clumps, analytical cylinder and end "
                        f"planes at 20 rpm, dt {h0:g}, CD every step, settled 15000 steps at dt 2e-5; loss = mean "
                        f"clump height", "steps": T, "checkpoint_every": K, "n_contacts": nC0,
            "fwd_ms_per_step": t_fwd / T, "record_ms_per_step": t_rec / T, "adjoint_ms_per_step": t_bwd / T,
            "adjoint_over_forward": t_bwd / t_fwd, "dL_dE_CoR_mu_Crr": [float(v) for v in out["d_material"][0]]}


def batched_measure(args, stream, rank=0, world=1, dist=None):
    """The batched calibration sweep: all scenes packed into one run (each scene with its own search grid, shapes
    from the autotuner, whole steps replayed from CUDA graphs), a forward window and a forward + adjoint window
    (per-scene loss: the mean final height of its spheres; gradients for every scene's material), against the same
    windows run scene by scene.  The scenes start pressed (lattice pitch 1.98 r) so that contacts carry the load
    from the first step.  Scene by scene, the forward window is timed for every scene with CUDA graphs and on a
    sample spanning the sizes without them; the adjoint window on a sample (the sample times are fitted linearly in
    the sphere count and summed over all scenes).  With N ranks the scenes are split by sphere count (each rank packs
    its share; no exchange while stepping), times are the max over ranks, and the per-scene gradients are gathered
    with one all-reduce at the end; the scene-by-scene baseline is measured on one GPU only."""
    import numpy as np
    import torch
    from deme_b200 import Solver, adjoint, sharding, workloads
    all_specs = workloads.batch_scene_specs(args.batch_scenes)
    for sp in all_specs:
        sp.update(pitch=1.98, lift=0.98)
    shard = (sharding.partition_scenes([sp["n"] for sp in all_specs], world)[rank] if world > 1
             else list(range(len(all_specs))))
    specs = [all_specs[i] for i in shard]
    T, K = args.batch_steps, args.batch_checkpoint

    def solver(built, graph=False):
        s = Solver(built)
        s.lib.deme_set_streams(s.h, C.c_void_p(stream.cuda_stream), C.c_void_p(stream.cuda_stream))
        if graph:
            s.set_graph(True)
        return s

    def timed(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        r = fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / 1e3, r

    def height_seed(built, ranges):
        seed = np.zeros((built.counts["o"], 3))
        for first, n in ranges:
            seed[first:first + n, 2] = 1.0 / n
        return seed

    built = workloads.batched_settling(specs)
    ranges = built.info["scenes"]
    w = solver(built)
    tuning = w.autotune(steps_per_trial=3)  # untimed; the shapes apply to every packed run below
    w.close()

    def tuned(s):
        s.set_search_shape(tuning["shape"], tuning["cell_factor"])
        s.set_kernel_shapes(tuning["force_shape"], tuning["exact_threads"], tuning["integrate_threads"])
        return s

    sf = tuned(solver(built, graph=True))
    sf.step(3)
    t_fwd, _ = timed(lambda: sf.step(T))
    nC = sf.num_contacts()
    sf.close()
    sa = tuned(solver(built))
    t_rec, _ = timed(lambda: adjoint.record(sa, T, K))
    t_bwd, out = timed(lambda: adjoint.backward(sa, d_pos=height_seed(built, ranges)))
    sa.close()
    # each scene loads one material, in scene order: material row i is the gradient of local scene i
    grads = sharding.gather_scene_rows({shard[i]: out["d_material"][i] for i in range(len(shard))}, len(all_specs), 4,
                                       dist=dist, device="cuda")
    n_spheres = int(sum(sp["n"] for sp in specs))
    if world > 1:
        tt = torch.tensor([t_fwd, t_rec + t_bwd], dtype=torch.float64, device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t_fwd, t_adj = float(tt[0]), float(tt[1])
        n = len(all_specs)
        return {"workload": f"{n} settling scenes split over {world} GPUs by sphere count, each rank's share packed in "
                            "one run: 500-20,000 spheres (log-uniform), r 2-5 mm, box 0.05-0.2 m, dt 1e-5, CD every "
                            "step, pressed start",
                "n_scenes": n, "n_spheres": int(sum(sp["n"] for sp in all_specs)), "steps": T, "checkpoint_every": K,
                "forward_s": t_fwd, "forward_adjoint_s": t_adj, "scenes_per_s": n / t_fwd,
                "scenes_per_s_with_adjoint": n / t_adj, "scaling": "strong (fixed scene set)",
                "material_gradients_finite": bool(np.all(np.isfinite(grads))),
                "gathered_gradient_rows": int(np.count_nonzero(np.any(grads != 0, axis=1)))}
    # scene by scene: the forward window of every scene with CUDA graphs
    sizes = np.array([sp["n"] for sp in specs])
    seq_graph = 0.0
    for i in range(len(specs)):
        b1 = workloads.single_settling(specs[i])
        s1 = solver(b1, graph=True)
        s1.step(3)
        tf, _ = timed(lambda: s1.step(T))
        s1.close()
        seq_graph += tf
    # on a sample spanning the sizes: the forward window launched step by step, and the adjoint window
    pick = np.unique(np.argsort(sizes)[np.linspace(0, len(specs) - 1, args.batch_sample).astype(int)])
    rows = []
    for i in pick:
        b1 = workloads.single_settling(specs[i])
        s1 = solver(b1)
        s1.step(3)
        tf, _ = timed(lambda: s1.step(T))
        s1.close()
        s1 = solver(b1)
        tr, _ = timed(lambda: adjoint.record(s1, T, K))
        tb, _ = timed(lambda: adjoint.backward(s1, d_pos=height_seed(b1, [(0, specs[i]["n"])])))
        s1.close()
        rows.append((sizes[i], tf, tr + tb))
    rows = np.array(rows, dtype=np.float64)
    fit_f = np.polyfit(rows[:, 0], rows[:, 1], 1)
    fit_a = np.polyfit(rows[:, 0], rows[:, 2], 1)
    seq_f = float(np.sum(np.polyval(fit_f, sizes)))
    seq_a = float(np.sum(np.polyval(fit_a, sizes)))
    n = len(specs)
    return {"workload": f"{n} settling scenes packed in one run: 500-20,000 spheres (log-uniform), r 2-5 mm, box "
                        "0.05-0.2 m, friction and restitution U[0.2, 0.8] per scene, dt 1e-5, CD every step, pressed "
                        "start (lattice pitch 1.98 r)",
            "n_scenes": n, "n_spheres": n_spheres, "steps": T, "checkpoint_every": K,
            "n_contacts_final": nC, "contacts_per_sphere_final": nC / n_spheres,
            "packed_tuning": tuning,
            "forward_s": t_fwd, "forward_adjoint_s": t_rec + t_bwd,
            "scenes_per_s": n / t_fwd, "scenes_per_s_with_adjoint": n / (t_rec + t_bwd),
            "sequential_scenes_per_s_graphs": n / seq_graph,
            "sequential_scenes_per_s": n / seq_f, "sequential_scenes_per_s_with_adjoint": n / seq_a,
            "speedup_forward_vs_graphs": seq_graph / t_fwd,
            "speedup_forward": seq_f / t_fwd, "speedup_with_adjoint": seq_a / (t_rec + t_bwd),
            "sequential_sample": f"forward with graphs: all {n} scenes timed alone; step by step and with the "
                                 f"adjoint: {len(rows)} scenes timed alone, time fitted linearly in sphere count",
            "material_gradients_finite": bool(np.all(np.isfinite(out["d_material"])))}


def s_grid_cells(built):
    """Cells of the contact search grid (same rule as the library: cell >= max(bin, CD diameter))."""
    import math
    p = built.params
    r = built.arrays["radius"].max() + p.beta
    cs = max(p.bin_size, 2.0 * float(r)) * (1.0 + 1e-6)
    n = 1
    for a in range(3):
        n *= math.ceil(p.domain[a] / cs) + 1
    return n


def read_traffic(kernel, nS, nC):
    """DRAM bytes per launch of ``kernel`` from the committed ncu summary, scaled to this launch's size."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(path) as f:
            d = json.load(f)[kernel]
        scale = (nC / d["n_contacts"]) if d.get("per") == "contact" else (nS / d["n_spheres"])
        return d["dram_bytes_per_launch"] * scale
    except Exception:
        return None


if __name__ == "__main__":
    main()
