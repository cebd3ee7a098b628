"""Recipe: build the reference's own kernel code for the CPU (oracle/_ref).

TEST INFRASTRUCTURE ONLY.  Reads the reference kernel templates where they lie (``/root/reference/src/kernel``),
performs the placeholder substitution of the reference's JIT layer (JitHelper::buildProgram,
src/core/utils/JitHelper.cpp:36-59; the substitution table of DEMSolver::jitifyKernels and its equip* helpers,
src/DEM/APIPrivate.cpp:203-220, 925-1380), writes the substituted translation units to ``oracle/_ref/<hash>/``
and compiles them with g++ together with oracle/ref_harness.cpp into ``libdeme_ref.so``.  Nothing is copied into
the repository: generated files stay under the git-ignored ``oracle/_ref/``.

The substituted values depend on the scene's world, materials, analytical boundaries and family prescriptions,
exactly as the reference's jitified kernels do, so one library is built per scene template and cached by a hash
of its sources.  Defaults of the reference are used: flattened (non-jitified) clump templates and mass
properties (src/DEM/API.h:460-463), the thread-per-bin contact kernels (DEMContactKernels.cu) and the built-in
frictional Hertz-Mindlin model.
"""
from __future__ import annotations

import hashlib
import os
import re
import subprocess
import sys

import numpy as np

REF_ROOT = os.environ.get("DEME_REFERENCE_ROOT", "/root/reference")
REF_SRC = os.path.join(REF_ROOT, "src")
KERNEL_DIR = os.path.join(REF_SRC, "kernel")
POLICY_DIR = os.path.join(KERNEL_DIR, "DEMCustomizablePolicies")
HERE = os.path.dirname(os.path.abspath(__file__))
OUT_ROOT = os.path.join(HERE, "_ref")
CUDA_INC = "/usr/local/cuda/include"

KERNEL_FILES = [
    "DEMBinSphereKernels.cu",
    "DEMContactKernels.cu",
    "DEMHistoryMappingKernels.cu",
    "DEMPrepForceKernels.cu",
    "DEMCalcForceKernels.cu",
    "DEMCollectForceKernels.cu",
    "DEMIntegrationKernels.cu",
]


def available() -> bool:
    return os.path.isdir(KERNEL_DIR) and os.path.exists(os.path.join(KERNEL_DIR, "DEMBinSphereKernels.cu"))


def _read(path: str) -> str:
    with open(path) as f:
        return f.read()


def _fx(v) -> str:
    """to_string_with_precision: std::fixed, 17 decimals (src/DEM/HostSideHelpers.hpp:396-401)."""
    return "%.17f" % float(v)


def _whole_word(s: str, w: str) -> bool:
    return re.search(r"\b" + re.escape(w) + r"\b", s) is not None


def substitutions(built) -> dict:
    p = built.params
    a = built.arrays
    nA = built.counts["a"]
    nO = built.counts["o"]
    subs = {}
    # equipClumpTemplates (flattened)
    subs["_clumpTemplateDefs_"] = " "
    subs["_componentAcqStrat_"] = _read(os.path.join(POLICY_DIR, "ClumpCompAcqStratAllFlatten.cu"))
    # equipSimParams
    subs["_nvXp2_"] = str(p.nvXp2)
    subs["_nvYp2_"] = str(p.nvYp2)
    subs["_nvZp2_"] = str(p.nvZp2)
    subs["_l_"] = _fx(p.l)
    subs["_voxelSize_"] = _fx(p.voxel_size)
    subs["_LBFX_"] = _fx(p.lbf[0])
    subs["_LBFY_"] = _fx(p.lbf[1])
    subs["_LBFZ_"] = _fx(p.lbf[2])
    subs["_nActiveLoadingThreads_"] = "32"
    n_templates = int(built.info.get("n_templates", 1))
    subs["_nDistinctMassProperties_"] = str(n_templates + built.info["n_ext"])
    subs["_nJitifiableClumpComponents_"] = "0"
    subs["_nMatTuples_"] = str(built.counts["m"])
    # equipMassMoiVolume (flattened)
    subs["_massDefs_"] = " "
    subs["_moiDefs_"] = " "
    subs["_massAcqStrat_"] = _read(os.path.join(POLICY_DIR, "MassAcqStratFlatten.cu"))
    subs["_moiAcqStrat_"] = _read(os.path.join(POLICY_DIR, "MOIAcqStratFlatten.cu"))
    subs["_volumeDefs_"] = "__constant__ __device__ float volumeProperties[] = {0};\n"
    # equipMaterials: one constant array per property name, names in std::set order
    names = set(["E", "nu", "CoR", "mu", "Crr"])
    defs = " "
    for name in sorted(names):
        vals = a["mat_" + name] if ("mat_" + name) in a else np.zeros(built.counts["m"], np.float32)
        defs += "__constant__ __device__ float " + name + "[] = {"
        for v in vals:
            defs += _fx(np.float32(v)) + ","
        if built.counts["m"] == 0:
            defs += "0"
        defs += "};\n"
    subs["_materialDefs_"] = defs
    # equipAnalGeoTemplates
    lists = {k: "" for k in ("_objOwner_", "_objType_", "_objMaterial_", "_objNormal_", "_objRelPosX_",
                             "_objRelPosY_", "_objRelPosZ_", "_objRotX_", "_objRotY_", "_objRotZ_", "_objSize1_",
                             "_objSize2_", "_objSize3_", "_objMass_")}
    for i in range(nA):
        t = int(a["anal_type"][i])
        if t not in (0, 1):
            raise ValueError("the reference supports only plane and plate analytical components")
        lists["_objOwner_"] += str(int(a["anal_owner"][i])) + ","
        lists["_objType_"] += str(t) + ","
        lists["_objMaterial_"] += str(int(a["anal_material"][i])) + ","
        lists["_objNormal_"] += str(int(a["anal_normal"][i])) + ","
        for key, arr in (("_objRelPosX_", "anal_relX"), ("_objRelPosY_", "anal_relY"), ("_objRelPosZ_", "anal_relZ"),
                         ("_objRotX_", "anal_rotX"), ("_objRotY_", "anal_rotY"), ("_objRotZ_", "anal_rotZ"),
                         ("_objSize1_", "anal_size1"), ("_objSize2_", "anal_size2"), ("_objSize3_", "anal_size3"),
                         ("_objMass_", "anal_mass")):
            lists[key] += _fx(np.float32(a[arr][i])) + ","
    if nA == 0:
        for k in lists:
            lists[k] += "0"
    anal_defs = _read(os.path.join(POLICY_DIR, "AnalyticalCompDefJitify.cu"))
    for k, v in lists.items():
        anal_defs = anal_defs.replace(k, v)
    subs["_analyticalEntityDefs_"] = anal_defs
    subs["_objOwner_"] = lists["_objOwner_"]
    # equipFamilyPrescribedMotions
    vel, pos = " ", " "
    merged = getattr(built, "merged_prescriptions", None) or built.info.get("merged_prescriptions", {})
    for fam in sorted(merged):
        m = merged[fam]
        vel += "case " + str(fam) + ": {"
        pos += "case " + str(fam) + ": {"
        for k, c in enumerate("XYZ"):
            if m.linVel[k] != "none":
                vel += "v" + c + " = " + m.linVel[k] + ";"
        for k, c in enumerate("XYZ"):
            if m.rotVel[k] != "none":
                vel += "omgBar" + c + " = " + m.rotVel[k] + ";"
        vel += "LinPrescribed = " + str(int(m.linVelPrescribed)) + ";"
        vel += "RotPrescribed = " + str(int(m.rotVelPrescribed)) + ";"
        vel += "break; }"
        for k, c in enumerate("XYZ"):
            if m.linPos[k] != "none":
                pos += c + " = " + m.linPos[k] + ";"
        pos += "LinPrescribed = " + str(int(m.linPosPrescribed)) + ";"
        pos += "RotPrescribed = " + str(int(m.rotPosPrescribed)) + ";"
        pos += "break; }"
    subs["_velPrescriptionStrategy_"] = vel
    subs["_posPrescriptionStrategy_"] = pos
    # equipForceModel (built-in frictional Hertz-Mindlin) and Models.h ingredient injection
    model = _read(os.path.join(POLICY_DIR, "FullHertzianForceModel.cu"))
    definition, acqA, acqB = " ", " ", " "
    if _whole_word(model, "ts"):
        definition += "float ts = simParams->h;\n"
    if _whole_word(model, "AOwnerFamily"):
        definition += "deme::family_t AOwnerFamily;\n"
        acqA += "AOwnerFamily = granData->familyID[myOwner];\n"
    if _whole_word(model, "BOwnerFamily"):
        definition += "deme::family_t BOwnerFamily;\n"
        acqB += "BOwnerFamily = granData->familyID[myOwner];\n"
    if _whole_word(model, "ALinVel") or _whole_word(model, "BLinVel"):
        definition += "float3 ALinVel, BLinVel;\n"
        acqA += "ALinVel.x = granData->vX[myOwner];\nALinVel.y = granData->vY[myOwner];\nALinVel.z = granData->vZ[myOwner];\n"
        acqB += "BLinVel.x = granData->vX[myOwner];\nBLinVel.y = granData->vY[myOwner];\nBLinVel.z = granData->vZ[myOwner];\n"
    if _whole_word(model, "ARotVel") or _whole_word(model, "BRotVel"):
        definition += "float3 ARotVel, BRotVel;\n"
        acqA += ("ARotVel.x = granData->omgBarX[myOwner];\nARotVel.y = granData->omgBarY[myOwner];\n"
                 "ARotVel.z = granData->omgBarZ[myOwner];\n")
        acqB += ("BRotVel.x = granData->omgBarX[myOwner];\nBRotVel.y = granData->omgBarY[myOwner];\n"
                 "BRotVel.z = granData->omgBarZ[myOwner];\n")
    wc_acq, wc_write, wc_destroy = " ", " ", " "
    for i, name in enumerate(sorted(["delta_time", "delta_tan_x", "delta_tan_y", "delta_tan_z"])):
        wc_acq += "float " + name + " = granData->contactWildcards[" + str(i) + "][myContactID];\n"
        wc_write += "granData->contactWildcards[" + str(i) + "][myContactID] = " + name + ";\n"
        wc_destroy += name + " = 0;\n"
    subs["_DEMForceModel_"] = model
    subs["_forceModelIngredientDefinition_"] = definition
    subs["_forceModelIngredientAcqForA_"] = acqA
    subs["_forceModelIngredientAcqForB_"] = acqB
    subs["_forceModelContactWildcardAcq_"] = wc_acq
    subs["_forceModelContactWildcardWrite_"] = wc_write
    subs["_forceModelContactWildcardDestroy_"] = wc_destroy
    # equipIntegrationScheme
    integ = {0: "IntegrationVelPassOnForwardEuler.cu", 1: "IntegrationVelPassOnCenteredDiff.cu",
             2: "IntegrationVelPassOnExtendedTaylor.cu"}[int(p.integrator)]
    subs["_integrationVelocityPassOnStrategy_"] = _read(os.path.join(POLICY_DIR, integ))
    return subs


def generate(built, out_root: str = OUT_ROOT) -> tuple[str, list]:
    if not available():
        raise FileNotFoundError(f"reference sources not found under {KERNEL_DIR}")
    subs = substitutions(built)
    units = []
    h = hashlib.sha256()
    for fname in KERNEL_FILES:
        code = _read(os.path.join(KERNEL_DIR, fname))
        for k, v in subs.items():
            code = code.replace(k, v)
        units.append((fname.replace(".cu", ".cpp"), code))
        h.update(code.encode())
    for extra in ("ref_harness.cpp", "ref_prelude.h"):
        h.update(_read(os.path.join(HERE, extra)).encode())
    d = os.path.join(out_root, h.hexdigest()[:16])
    os.makedirs(os.path.join(d, "gen"), exist_ok=True)
    os.makedirs(os.path.join(out_root, "stub", "cub"), exist_ok=True)
    stub = os.path.join(out_root, "stub", "cub", "util_ptx.cuh")
    if not os.path.exists(stub):
        with open(stub, "w") as f:
            f.write("// empty stand-in: the thread-per-bin kernels need nothing from this header on the CPU\n")
    paths = []
    for name, code in units:
        path = os.path.join(d, "gen", name)
        if not os.path.exists(path) or _read(path) != code:
            with open(path, "w") as f:
                f.write(code)
        paths.append(path)
    return d, paths


INDEX = os.path.join(OUT_ROOT, "cpu-index.txt")


def _index_key(built) -> str:
    if HERE not in sys.path:
        sys.path.insert(0, HERE)
    import ref_gpu_build  # noqa: E402
    return ref_gpu_build.scene_key(built, fmad=False)


def _index_put(built, lib: str):
    rows = {}
    if os.path.exists(INDEX):
        with open(INDEX) as f:
            rows = dict(line.split() for line in f if line.strip())
    rows[_index_key(built)] = os.path.relpath(lib, OUT_ROOT)
    with open(INDEX + ".tmp", "w") as f:
        f.write("".join(f"{k} {v}\n" for k, v in sorted(rows.items())))
    os.replace(INDEX + ".tmp", INDEX)


def lookup(built) -> str | None:
    """The CPU build for this scene: built now where the reference's sources exist, else a prebuilt one found
    through the index (keyed by the scene values the substitution reads), else None."""
    if available():
        return build(built)
    if os.path.exists(INDEX):
        key = _index_key(built)
        with open(INDEX) as f:
            for line in f:
                k, v = line.split()
                if k == key and os.path.exists(os.path.join(OUT_ROOT, v)):
                    return os.path.join(OUT_ROOT, v)
    return None


def build(built, out_root: str = OUT_ROOT, verbose: bool = False) -> str:
    d, paths = generate(built, out_root)
    lib = os.path.join(d, "libdeme_ref.so")
    harness = os.path.join(HERE, "ref_harness.cpp")
    if os.path.exists(lib) and os.path.getmtime(lib) >= os.path.getmtime(harness):
        if out_root == OUT_ROOT:
            _index_put(built, lib)
        return lib
    objs = []
    flags = ["-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-fno-fast-math", "-fopenmp", "-w",
             "-I" + os.path.join(out_root, "stub"), "-I" + REF_SRC, "-I" + CUDA_INC,
             "-include", os.path.join(HERE, "ref_prelude.h")]
    procs = []
    for src in paths + [os.path.join(HERE, "ref_harness.cpp")]:
        obj = os.path.join(d, os.path.basename(src) + ".o")
        objs.append(obj)
        procs.append(subprocess.Popen(["g++", "-c", src, "-o", obj] + flags, stdout=subprocess.PIPE,
                                      stderr=subprocess.STDOUT))
    for pr in procs:
        out, _ = pr.communicate()
        if pr.returncode != 0:
            raise RuntimeError("reference CPU build failed:\n" + out.decode()[-4000:])
        if verbose and out:
            sys.stderr.write(out.decode())
    tmp = lib + ".tmp"
    subprocess.check_call(["g++", "-shared", "-fopenmp", "-o", tmp] + objs)
    os.replace(tmp, lib)
    if out_root == OUT_ROOT:
        _index_put(built, lib)
    return lib


MESH_DIR = os.path.join(REF_ROOT, "data", "mesh")
LOADER_HDR = os.path.join(REF_SRC, "core", "utils", "WavefrontMeshLoader.hpp")


def obj_loader_available() -> bool:
    return os.path.exists(LOADER_HDR)


def build_obj_dump(out_root: str = OUT_ROOT) -> str:
    """Compile oracle/ref_obj_dump.cpp against the reference's Wavefront parser (src/core/utils/
    WavefrontMeshLoader.hpp, the loader behind DEMMeshConnected::LoadWavefrontMesh) into ``_ref/ref_obj_dump``."""
    src = os.path.join(HERE, "ref_obj_dump.cpp")
    exe = os.path.join(out_root, "ref_obj_dump")
    if os.path.exists(exe) and os.path.getmtime(exe) >= max(os.path.getmtime(src), os.path.getmtime(LOADER_HDR)):
        return exe
    os.makedirs(out_root, exist_ok=True)
    tmp = exe + ".tmp"
    subprocess.check_call(["g++", "-O1", "-std=c++17", "-w", "-I" + REF_SRC, src, "-o", tmp])
    os.replace(tmp, exe)
    return exe


def read_obj_dump(path: str) -> dict:
    """The arrays ``ref_obj_dump`` writes: vertices, facet vertex indices, normals, facet normal indices."""
    raw = open(path, "rb").read()
    nv, nf, nn, nfn = np.frombuffer(raw[:16], np.int32)
    off, out = 16, {}
    for key, n, dt in (("vertices", nv, np.float32), ("faces", nf, np.int32), ("normals", nn, np.float32),
                       ("face_normals", nfn, np.int32)):
        a = np.frombuffer(raw, dt, 3 * int(n), off).reshape(-1, 3)
        off += a.nbytes
        out[key] = a
    return out


def build_csv_dump(out_root: str = OUT_ROOT) -> str:
    """Compile oracle/ref_csv_dump.cpp against the reference's CSV reader (src/core/utils/csv.hpp, the reader behind
    DEMClumpTemplate::ReadComponentFromFile and ReadClumpXyzFromCsv) into ``_ref/ref_csv_dump``."""
    src = os.path.join(HERE, "ref_csv_dump.cpp")
    hdr = os.path.join(REF_SRC, "core", "utils", "csv.hpp")
    exe = os.path.join(out_root, "ref_csv_dump")
    if os.path.exists(exe) and os.path.getmtime(exe) >= max(os.path.getmtime(src), os.path.getmtime(hdr)):
        return exe
    os.makedirs(out_root, exist_ok=True)
    tmp = exe + ".tmp"
    subprocess.check_call(["g++", "-O1", "-std=c++17", "-w", "-pthread", "-I" + REF_SRC, src, "-o", tmp])
    os.replace(tmp, exe)
    return exe


CLUMP_DIR = os.path.join(REF_ROOT, "data", "clumps")


def read_csv_dump(path: str) -> tuple[np.ndarray, list]:
    """The rows (n x 4 float32) and names ``ref_csv_dump`` writes."""
    raw = open(path, "rb").read()
    n = int(np.frombuffer(raw, np.int32, 1)[0])
    vals = np.frombuffer(raw, np.float32, 4 * n, 4).reshape(-1, 4)
    off, names = 4 + 16 * n, []
    while off < len(raw):
        ln = int(np.frombuffer(raw, np.int32, 1, off)[0])
        names.append(raw[off + 4:off + 4 + ln].decode())
        off += 4 + ln
    return vals, names
