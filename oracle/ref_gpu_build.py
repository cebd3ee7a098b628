"""Recipe: build the reference's own kernels for the GPU (oracle/_ref/gpu-<key>/) and the driver that runs them
(oracle/_ref/libdeme_ref_gpu.so).

TEST AND BASELINE INFRASTRUCTURE ONLY.  The reference compiles its kernel templates at run time: JitHelper substitutes
the scene's placeholders into the text of ``src/kernel/*.cu`` (src/core/utils/JitHelper.cpp:36-59, substitution
table of DEMSolver::jitifyKernels, src/DEM/APIPrivate.cpp:203-220, 925-1380) and jitify hands the result to NVRTC
for the running device.  This recipe performs the same substitution (``ref_build.substitutions``), compiles each
program with NVRTC for sm_100a into a cubin, and records each kernel's lowered name, so that a machine without the
reference's sources (or its jitify dependency) can load and launch them.  Both contact-kernel variants are built: the
default block-per-bin one (src/kernel/DEMContactKernels_Blockwise.cu; ``useOneBinPerThread`` is false by default,
src/DEM/Structs.h:357) and the thread-per-bin one (src/kernel/DEMContactKernels.cu).

NVRTC gets the reference's include directory, the CUDA headers (for CUB), ``--device-as-default-execution-space``
(the helper ``matProxy2ContactParam`` carries no execution-space qualifier, src/kernel/DEMHelperKernels.cu:316-339)
and four small stand-in headers for the host headers ``src/DEM/Defines.h`` includes but the kernels do not use.
FMA contraction is NVRTC's default (on) unless ``fmad=False``; the parity tests build that variant so that the
reference's double-precision contact tests round as the oracle's do.

The cubin directory is keyed by ``scene_key(built)``, a hash of exactly the scene values the substitution reads
(world, materials, analytical components, prescriptions, integrator, template counts), so the key can be computed
where the reference's sources are absent.  Nothing is copied into the repository: outputs stay under the git-ignored
``oracle/_ref/``.
"""
from __future__ import annotations

import ctypes as C
import hashlib
import json
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
OUT_ROOT = os.path.join(HERE, "_ref")
HARNESS_SRC = os.path.join(HERE, "ref_gpu_harness.cu")
HARNESS_LIB = os.path.join(OUT_ROOT, "libdeme_ref_gpu.so")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")

PROGRAMS = {
    "DEMBinSphereKernels": ["getNumberOfBinsEachSphereTouches", "populateBinSphereTouchingPairs"],
    "DEMContactKernels_Blockwise": ["getNumberOfContactsEachBin", "populateContactPairsEachBin"],
    "DEMContactKernels": ["getNumberOfContactsEachBin", "populateContactPairsEachBin"],
    "DEMHistoryMappingKernels": ["fillRunLengthArray", "buildPersistentMap"],
    "DEMPrepForceKernels": ["prepareForceArrays", "rearrangeContactWildcards"],
    "DEMCalcForceKernels": ["calculateContactForces"],
    "DEMCollectForceKernels": ["cashInOwnerIndexA", "cashInOwnerIndexB", "forceToAcc", "forceToAngAcc", "stashElem"],
    "DEMIntegrationKernels": ["integrateOwners"],
}

# Stand-ins for the host headers src/DEM/Defines.h includes (<limits>, <stdint.h>, <algorithm>, <cmath>): the
# kernels use only the fixed-width integer types from them.
STAND_IN_HEADERS = {
    "limits": "#pragma once\n",
    "algorithm": "#pragma once\n",
    "cmath": "#pragma once\n",
    "stdint.h": ("#pragma once\n#include <cuda/std/cstdint>\n"
                 "using cuda::std::int8_t; using cuda::std::int16_t; using cuda::std::int32_t; using cuda::std::int64_t;\n"
                 "using cuda::std::uint8_t; using cuda::std::uint16_t; using cuda::std::uint32_t;\n"
                 "using cuda::std::uint64_t;\n"),
}


def _ref_build():
    if HERE not in sys.path:
        sys.path.insert(0, HERE)
    import ref_build  # noqa: E402
    return ref_build


def available() -> bool:
    """The reference's sources are here, so cubins can be built."""
    return _ref_build().available()


def scene_key(built, fmad: bool = True) -> str:
    """Hash of every scene value ``ref_build.substitutions`` reads (no reference file needed)."""
    p = built.params
    a = built.arrays
    h = hashlib.sha256()
    for name in ("nvXp2", "nvYp2", "nvZp2", "l", "voxel_size", "integrator"):
        h.update(repr(getattr(p, name)).encode())
    h.update(repr([float(v) for v in p.lbf]).encode())
    for k in ("m", "a", "o"):
        h.update(repr(built.counts[k]).encode())
    h.update(repr((int(built.info.get("n_templates", 1)), int(built.info["n_ext"]))).encode())
    for name in ("mat_E", "mat_nu", "mat_CoR", "mat_mu", "mat_Crr", "anal_owner", "anal_type", "anal_material",
                 "anal_normal", "anal_relX", "anal_relY", "anal_relZ", "anal_rotX", "anal_rotY", "anal_rotZ",
                 "anal_size1", "anal_size2", "anal_size3", "anal_mass"):
        if name in a:
            h.update(name.encode())
            h.update(np.ascontiguousarray(a[name]).tobytes())
    merged = getattr(built, "merged_prescriptions", None) or built.info.get("merged_prescriptions", {})
    for fam in sorted(merged):
        m = merged[fam]
        h.update(repr((fam, list(m.linVel), list(m.rotVel), list(m.linPos), m.linVelPrescribed, m.rotVelPrescribed,
                       m.linPosPrescribed, m.rotPosPrescribed)).encode())
    h.update(b"fmad" if fmad else b"nofmad")
    h.update(" ".join(PROGRAMS).encode())
    return h.hexdigest()[:16]


def cubin_dir(built, fmad: bool = True) -> str:
    return os.path.join(OUT_ROOT, "gpu-" + scene_key(built, fmad))


def _nvrtc():
    lib = C.CDLL(os.path.join(CUDA_HOME, "lib64", "libnvrtc.so"))
    lib.nvrtcGetErrorString.restype = C.c_char_p
    return lib


def _compile(nv, name: str, code: str, kernels: list, fmad: bool, ref_src: str) -> tuple[bytes, dict]:
    prog = C.c_void_p()
    hn = [k.encode() for k in STAND_IN_HEADERS]
    hs = [v.encode() for v in STAND_IN_HEADERS.values()]
    r = nv.nvrtcCreateProgram(C.byref(prog), code.encode(), (name + ".cu").encode(), len(hn),
                              (C.c_char_p * len(hs))(*hs), (C.c_char_p * len(hn))(*hn))
    if r:
        raise RuntimeError(f"nvrtcCreateProgram({name}): {nv.nvrtcGetErrorString(r).decode()}")
    try:
        for k in kernels:
            nv.nvrtcAddNameExpression(prog, k.encode())
        opts = ["-arch=sm_100a", "-std=c++17", "--device-as-default-execution-space", "-I" + ref_src,
                "-I" + os.path.join(CUDA_HOME, "include"), "-diag-suppress=1444,177,550,549,186"]
        if not fmad:
            opts.append("--fmad=false")
        ob = [o.encode() for o in opts]
        r = nv.nvrtcCompileProgram(prog, len(ob), (C.c_char_p * len(ob))(*ob))
        n = C.c_size_t()
        nv.nvrtcGetProgramLogSize(prog, C.byref(n))
        log = C.create_string_buffer(n.value)
        nv.nvrtcGetProgramLog(prog, log)
        if r:
            raise RuntimeError(f"NVRTC failed on {name}:\n" + log.value.decode(errors="replace")[-4000:])
        nv.nvrtcGetCUBINSize(prog, C.byref(n))
        cubin = C.create_string_buffer(n.value)
        nv.nvrtcGetCUBIN(prog, cubin)
        lowered = {}
        for k in kernels:
            out = C.c_char_p()
            r = nv.nvrtcGetLoweredName(prog, k.encode(), C.byref(out))
            if r:
                raise RuntimeError(f"no lowered name for {k} in {name}")
            lowered[k] = out.value.decode()
        return cubin.raw, lowered
    finally:
        nv.nvrtcDestroyProgram(C.byref(prog))


def build_cubins(built, fmad: bool = True) -> str:
    """Substitutes and compiles the reference's kernel programs for this scene; returns the cubin directory."""
    rb = _ref_build()
    d = cubin_dir(built, fmad)
    if os.path.exists(os.path.join(d, "kernels.txt")):
        return d
    if not rb.available():
        raise FileNotFoundError("reference kernel sources not found; cubins for this scene were not prebuilt: " + d)
    subs = rb.substitutions(built)
    nv = _nvrtc()
    os.makedirs(d, exist_ok=True)
    rows = []
    for prog, kernels in PROGRAMS.items():
        code = rb._read(os.path.join(rb.KERNEL_DIR, prog + ".cu"))
        for k, v in subs.items():
            code = code.replace(k, v)
        cubin, lowered = _compile(nv, prog, code, kernels, fmad, rb.REF_SRC)
        with open(os.path.join(d, prog + ".cubin"), "wb") as f:
            f.write(cubin)
        rows += [f"{prog} {k} {lowered[k]}" for k in kernels]
    with open(os.path.join(d, "scene.json"), "w") as f:
        json.dump({"workload": built.info.get("workload"), "n_spheres": built.counts["s"], "fmad": fmad}, f)
    tmp = os.path.join(d, "kernels.txt.tmp")
    with open(tmp, "w") as f:
        f.write("\n".join(rows) + "\n")
    os.replace(tmp, os.path.join(d, "kernels.txt"))
    return d


def build_harness(force: bool = False) -> str:
    """Compiles the driver (scene-independent) with nvcc against the reference's struct definitions."""
    rb = _ref_build()
    if os.path.exists(HARNESS_LIB) and not force and os.path.getmtime(HARNESS_LIB) >= os.path.getmtime(HARNESS_SRC):
        return HARNESS_LIB
    if not rb.available():
        if os.path.exists(HARNESS_LIB):
            return HARNESS_LIB
        raise FileNotFoundError("reference sources not found and no prebuilt " + HARNESS_LIB)
    os.makedirs(OUT_ROOT, exist_ok=True)
    tmp = HARNESS_LIB + ".tmp"
    cmd = [os.path.join(CUDA_HOME, "bin", "nvcc"), "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17",
           "-shared", "-Xcompiler", "-fPIC", "-w", "-I" + rb.REF_SRC, "-I" + os.path.join(ROOT, "include"),
           HARNESS_SRC, "-o", tmp, "-lcudart"]
    subprocess.check_call(cmd)
    os.replace(tmp, HARNESS_LIB)
    return HARNESS_LIB


def _workloads():
    pkg = os.path.join(ROOT, "dem-engine-sbel_b200")
    if pkg not in sys.path:
        sys.path.insert(0, pkg)
    from deme_b200 import workloads
    return workloads


# Scenes the GPU parity tests run against the reference's kernels (FMA contraction off), by name.
PARITY_SCENES = {
    "clumps_dense": lambda w: w.packed_clumps(n_clumps=300, seed=21, spacing=1.3),
    "spheres_masks": lambda w: w.packed_clumps(n_clumps=500, seed=22, three=False, families=True, beta=5e-4),
    "settle": lambda w: w.settling_box(n=600, r=5e-3, box=(0.08, 0.08, 0.12), spacing=1.99, jitter=0.03, seed=23,
                                       vel_scale=0.3, ang_scale=30.0),
    "drum_shell": lambda w: w.drum(20000, shell=True, spacing=0.745),
    "shaker": lambda w: w.shaker_box(),
}


def parity_scene(name: str):
    return PARITY_SCENES[name](_workloads())


def bench_shell_drum(n_clumps: int = 1_000_000, spacing: float = 0.745):
    """The drum the reference can express (shell of fixed spheres), on the dense start lattice."""
    return _workloads().drum(n_clumps, shell=True, spacing=spacing)


def prebuild(bench_clumps: int = 1_000_000, cpu_sample_clumps: int = 200_000, bench_hopper_spheres: int = 4_000_000) -> list:
    """For machines without the reference's sources: the driver, the parity scenes' cubins (FMA off), the benchmark
    drum's cubins (NVRTC default and FMA off), and the reference's CPU build for the benchmark's bounded CPU
    sample."""
    out = [build_harness()]
    for name in PARITY_SCENES:
        out.append(build_cubins(parity_scene(name), fmad=False))
    out.append(build_cubins(bench_shell_drum(bench_clumps), fmad=True))
    # the full-size parity test runs the benchmark drum against both builds
    out.append(build_cubins(bench_shell_drum(bench_clumps), fmad=False))
    # the plane-only wedge hopper the benchmark times the reference's kernels on
    out.append(build_cubins(_workloads().hopper_wedge(n=bench_hopper_spheres), fmad=True))
    out.append(_ref_build().build(bench_shell_drum(cpu_sample_clumps)))
    return out


if __name__ == "__main__":
    for d in prebuild():
        print(d)
