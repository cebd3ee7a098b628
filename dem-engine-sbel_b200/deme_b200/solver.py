"""Python bindings of the C ABI (include/deme_b200.h).

``Solver`` drives the CUDA library through ``deme_*``.  ``HandleSolver`` is the same wrapper over any library
that exports the ABI's entry points under another prefix; tests use it to run the C oracle and the reference
kernels compiled for the CPU with identical calls.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import _capi as capi

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libdeme_b200.so")
_lib = None


def load_product_library(path: str = LIB_PATH) -> C.CDLL:
    """Load the CUDA product library; fails loudly if it was not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(path):
            raise RuntimeError(f"CUDA extension not built: {path} is missing (run __graft_entry__.build())")
        lib = capi.load_library(path)
        capi.bind(lib, "deme_")
        lib.deme_get_error.restype = C.c_char_p
        lib.deme_get_error.argtypes = [C.c_void_p]
        lib.deme_status_string.restype = C.c_char_p
        lib.deme_status_string.argtypes = [C.c_int32]
        lib.deme_get_num_contacts.restype = C.c_int32
        lib.deme_get_num_contacts.argtypes = [C.c_void_p, C.POINTER(C.c_uint32)]
        lib.deme_create.restype = C.c_int32
        lib.deme_create.argtypes = [C.POINTER(capi.SimParams), C.POINTER(capi.Scene), C.POINTER(C.c_void_p)]
        lib.deme_sync.restype = C.c_int32
        lib.deme_sync.argtypes = [C.c_void_p]
        lib.deme_kinetic_energy.restype = C.c_int32
        lib.deme_kinetic_energy.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
        lib.deme_get_time.restype = C.c_int32
        lib.deme_get_time.argtypes = [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int64)]
        lib.deme_set_force_model.restype = C.c_int32
        lib.deme_set_force_model.argtypes = [C.c_void_p, C.c_char_p, C.POINTER(C.c_char_p), C.c_int32]
        lib.deme_abi_version.restype = C.c_int32
        _lib = lib
    return _lib


class DemeError(RuntimeError):
    pass


class HandleSolver:
    """Wrapper over a library exporting the ABI under ``prefix`` (``orc_`` or ``ref_``)."""

    def __init__(self, lib: C.CDLL, prefix: str, built, threads: int | None = None):
        self.lib = lib
        self.prefix = prefix
        self.built = built
        capi.bind(lib, prefix)
        if threads is not None and hasattr(lib, prefix + "set_threads"):
            getattr(lib, prefix + "set_threads")(threads)
        scene, self._keep = built.scene_struct()
        self._params = built.params
        self.h = self._create(scene)
        self.nO = built.counts["o"]
        self.nS = built.counts["s"]
        self.nW = built.params.n_contact_wildcards

    def _fn(self, name):
        return getattr(self.lib, self.prefix + name)

    def _create(self, scene):
        h = self._fn("create")(C.byref(self._params), C.byref(scene))
        if not h:
            raise DemeError(f"{self.prefix}create failed")
        return h

    def _check(self, st, what):
        if st != capi.DEME_OK:
            raise DemeError(f"{self.prefix}{what}: {capi.STATUS_NAMES.get(st, st)}")

    def close(self):
        if getattr(self, "h", None):
            self._fn("destroy")(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def change_clump_sizes(self, owners, factors):
        """ChangeClumpSizes: the listed clumps' component spheres get their relative positions and radii multiplied by
        the factors (masses and moments stay); contacts are found anew at the next detection."""
        o = np.ascontiguousarray(owners, np.uint32)
        f = np.ascontiguousarray(factors, np.float32)
        if o.shape != f.shape:
            raise ValueError("one factor per clump")
        fn = self._fn("change_clump_sizes")
        fn.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p]
        fn.restype = C.c_int32
        self._check(fn(self.h, len(o), capi.ptr(o), capi.ptr(f)), "change_clump_sizes")

    # --- steps ---
    def detect_contacts(self):
        self._check(self._fn("detect_contacts")(self.h), "detect_contacts")

    def compute_forces(self):
        self._check(self._fn("compute_forces")(self.h), "compute_forces")

    def integrate(self):
        self._check(self._fn("integrate")(self.h), "integrate")

    def step(self, n: int = 1):
        self._check(self._fn("step")(self.h, n), "step")

    def sync(self):
        pass

    # --- transfer ---
    def num_contacts(self) -> int:
        return int(self._fn("num_contacts")(self.h))

    def state(self) -> dict:
        out = {name: np.zeros(self.nO, dt) for name, dt in capi.STATE_FIELDS}
        st, keep = capi.state_struct(out)
        self._check(self._fn("download_state")(self.h, C.byref(st)), "download_state")
        return out

    def set_state(self, arrays: dict):
        arrays = {k: np.ascontiguousarray(v, dtype=dict(capi.STATE_FIELDS)[k]) for k, v in arrays.items()}
        st, keep = capi.state_struct(arrays)
        self._check(self._fn("upload_state")(self.h, C.byref(st)), "upload_state")

    def contacts(self) -> dict:
        n = self.num_contacts()
        cap = max(n, 1)
        d = dict(idA=np.zeros(cap, np.uint32), idB=np.zeros(cap, np.uint32), type=np.zeros(cap, np.uint8),
                 mapping=np.zeros(cap, np.uint32), wildcards=np.zeros((max(self.nW, 1), cap), np.float32))
        c = capi.Contacts(cap, 0, capi.ptr(d["idA"]), capi.ptr(d["idB"]), capi.ptr(d["type"]),
                          capi.ptr(d["mapping"]), capi.ptr(d["wildcards"]))
        self._check(self._fn("download_contacts")(self.h, C.byref(c)), "download_contacts")
        n = c.n_contacts
        return dict(idA=d["idA"][:n], idB=d["idB"][:n], type=d["type"][:n], mapping=d["mapping"][:n],
                    wildcards=d["wildcards"][:self.nW, :n])

    def set_contacts(self, d: dict):
        n = len(d["idA"])
        cap = max(n, 1)
        idA = np.zeros(cap, np.uint32)
        idB = np.zeros(cap, np.uint32)
        tp = np.zeros(cap, np.uint8)
        wc = np.zeros((max(self.nW, 1), cap), np.float32)
        idA[:n] = d["idA"]
        idB[:n] = d["idB"]
        tp[:n] = d["type"]
        if self.nW and d.get("wildcards") is not None:
            wc[:self.nW, :n] = d["wildcards"]
        c = capi.Contacts(cap, n, capi.ptr(idA), capi.ptr(idB), capi.ptr(tp), None, capi.ptr(wc))
        self._check(self._fn("upload_contacts")(self.h, C.byref(c)), "upload_contacts")

    def contact_forces(self) -> dict:
        n = self.num_contacts()
        cap = max(n, 1)
        d = {k: np.zeros((cap, 3), np.float32) for k in ("force", "torque_only_force", "cpA", "cpB")}
        c = capi.ContactForces(cap, 0, capi.ptr(d["force"]), capi.ptr(d["torque_only_force"]), capi.ptr(d["cpA"]),
                               capi.ptr(d["cpB"]))
        self._check(self._fn("download_contact_forces")(self.h, C.byref(c)), "download_contact_forces")
        return {k: v[:c.n_contacts] for k, v in d.items()}

    # ---- output in DEM-Engine's CSV formats (deme_b200.io; WriteSphereFile etc., src/DEM/API.h:319-324) ----
    def SetOutputContent(self, content: int):
        self._out_content = int(content)

    def SetContactOutputContent(self, content: int):
        self._cnt_out_content = int(content)

    def DisableFamilyOutput(self, fam: int):
        self._no_output = tuple(sorted(set(getattr(self, "_no_output", ())) | {int(fam)}))

    def WriteSphereFile(self, path: str):
        from . import io
        io.write_sphere_file(path, self.built, self.state(), getattr(self, "_out_content", io.DEFAULT_CONTENT),
                             getattr(self, "_no_output", ()))

    def WriteClumpFile(self, path: str):
        from . import io
        io.write_clump_file(path, self.built, self.state(), getattr(self, "_out_content", io.DEFAULT_CONTENT),
                            getattr(self, "_no_output", ()))

    def WriteContactFile(self, path: str):
        """Forces, points and normals need the per-contact forces of the last step (the CUDA solver keeps them after
        keep_contact_forces(True))."""
        from . import io
        content = getattr(self, "_cnt_out_content", io.DEFAULT_CONTACT_CONTENT)
        forces = self.contact_forces() if content != io.OWNERS else None
        io.write_contact_file(path, self.built, self.state(), self.contacts(), forces, content)

    def bin_assignment(self, with_pairs: bool = True) -> dict:
        nb = np.zeros(max(self.nS, 1), np.uint16)
        na = np.zeros(max(self.nS, 1), np.uint8)
        npairs = C.c_uint32(0)
        self._check(self._fn("bin_assignment")(self.h, capi.ptr(nb), capi.ptr(na), 0, None, None, C.byref(npairs)),
                    "bin_assignment")
        out = dict(n_bins=nb[:self.nS], n_anal=na[:self.nS], n_pairs=int(npairs.value))
        if with_pairs:
            cap = max(int(npairs.value), 1)
            bins = np.zeros(cap, np.uint32)
            sph = np.zeros(cap, np.uint32)
            self._check(self._fn("bin_assignment")(self.h, None, None, cap, capi.ptr(bins), capi.ptr(sph),
                                                   C.byref(npairs)), "bin_assignment")
            out["bins"] = bins[:npairs.value]
            out["spheres"] = sph[:npairs.value]
        return out

    def kinetic_energy(self) -> float:
        return float(self._fn("kinetic_energy")(self.h))


class Solver(HandleSolver):
    """The CUDA product path (``deme_*``)."""

    def __init__(self, built, lib_path: str = LIB_PATH):
        lib = load_product_library(lib_path)
        self.lib = lib
        self.prefix = "deme_"
        self.built = built
        scene, self._keep = built.scene_struct()
        self._params = built.params
        h = C.c_void_p()
        st = lib.deme_create(C.byref(self._params), C.byref(scene), C.byref(h))
        if st != capi.DEME_OK:
            msg = lib.deme_get_error(h.value) if h.value else b""
            if h.value:
                lib.deme_destroy(h.value)
            self.h = None
            raise DemeError(f"deme_create: {capi.STATUS_NAMES.get(st, st)}: {msg.decode() if msg else ''}")
        self.h = h.value
        self.nO = built.counts["o"]
        self.nS = built.counts["s"]
        self.nW = built.params.n_contact_wildcards
        motion = built.info.get("motion_expressions") if isinstance(built.info, dict) else None
        if motion:
            try:
                self.set_prescribed_motion(motion)
            except DemeError:
                self.close()
                raise

    def _check(self, st, what):
        if st != capi.DEME_OK:
            msg = self.lib.deme_get_error(self.h)
            raise DemeError(f"deme_{what}: {capi.STATUS_NAMES.get(st, st)}: {msg.decode() if msg else ''}")

    def num_contacts(self) -> int:
        n = C.c_uint32(0)
        self._check(self.lib.deme_get_num_contacts(self.h, C.byref(n)), "get_num_contacts")
        return int(n.value)

    def sync(self):
        self._check(self.lib.deme_sync(self.h), "sync")

    def kinetic_energy(self) -> float:
        ke = C.c_double(0)
        self._check(self.lib.deme_kinetic_energy(self.h, C.byref(ke)), "kinetic_energy")
        return float(ke.value)

    def kinetic_energy_enqueue(self) -> int:
        """Queues the kinetic-energy sum after the work queued so far; returns a ticket for kinetic_energy_collect."""
        t = C.c_int64(0)
        self.lib.deme_kinetic_energy_enqueue.argtypes = [C.c_void_p, C.POINTER(C.c_int64)]
        self.lib.deme_kinetic_energy_enqueue.restype = C.c_int32
        self._check(self.lib.deme_kinetic_energy_enqueue(self.h, C.byref(t)), "kinetic_energy_enqueue")
        return int(t.value)

    def kinetic_energy_collect(self, ticket: int) -> float:
        """Waits for an enqueued kinetic-energy sum and returns it."""
        ke = C.c_double(0)
        self.lib.deme_kinetic_energy_collect.argtypes = [C.c_void_p, C.c_int64, C.POINTER(C.c_double)]
        self.lib.deme_kinetic_energy_collect.restype = C.c_int32
        self._check(self.lib.deme_kinetic_energy_collect(self.h, int(ticket), C.byref(ke)), "kinetic_energy_collect")
        return float(ke.value)

    def set_time_step(self, h: float):
        self.lib.deme_set_time_step.argtypes = [C.c_void_p, C.c_float]
        self._check(self.lib.deme_set_time_step(self.h, h), "set_time_step")

    def time(self) -> tuple[float, float, int]:
        """(time, the reference's float time, steps taken)."""
        t, tf, n = C.c_double(0), C.c_float(0), C.c_int64(0)
        self.lib.deme_get_time.argtypes = [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int64)]
        self.lib.deme_get_time_float.argtypes = [C.c_void_p, C.POINTER(C.c_float)]
        self._check(self.lib.deme_get_time(self.h, C.byref(t), C.byref(n)), "get_time")
        self._check(self.lib.deme_get_time_float(self.h, C.byref(tf)), "get_time_float")
        return float(t.value), float(tf.value), int(n.value)

    def set_time(self, t: float, t_float: float, steps: int):
        """Carries a run's time and step counter over into this handle."""
        self.lib.deme_set_time.argtypes = [C.c_void_p, C.c_double, C.c_float, C.c_int64]
        self._check(self.lib.deme_set_time(self.h, t, t_float, int(steps)), "set_time")

    def set_streams(self, kt_stream: int | None, dt_stream: int | None):
        self.lib.deme_set_streams.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        self._check(self.lib.deme_set_streams(self.h, kt_stream, dt_stream), "set_streams")

    def set_async_cd(self, lag: int):
        """kT/dT on two streams: detections adopted ``lag`` steps after the poses they were made from (0: in step)."""
        self.lib.deme_set_async_cd.argtypes = [C.c_void_p, C.c_int32]
        self._check(self.lib.deme_set_async_cd(self.h, int(lag)), "set_async_cd")

    def set_graph(self, enable: bool = True):
        """Replay whole steps from CUDA graphs (see deme_set_graph)."""
        self.lib.deme_set_graph.argtypes = [C.c_void_p, C.c_int32]
        self._check(self.lib.deme_set_graph(self.h, int(enable)), "set_graph")

    def graph_stats(self) -> tuple[int, int]:
        """(windows replayed from graphs, batches rolled back)."""
        r, b = C.c_int64(0), C.c_int64(0)
        self.lib.deme_graph_stats.argtypes = [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
        self._check(self.lib.deme_graph_stats(self.h, C.byref(r), C.byref(b)), "graph_stats")
        return int(r.value), int(b.value)

    def change_family(self, family_from: int, family_to: int):
        """ChangeFamily: every owner of one family moves to another now."""
        self.lib.deme_change_family.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32]
        self._check(self.lib.deme_change_family(self.h, int(family_from), int(family_to)), "change_family")

    def DisableContactBetweenFamilies(self, a: int, b: int):
        """Contact between families a and b is off from the next detection (the reference's call on an initialized
        solver)."""
        self._set_family_contact(a, b, True)

    def EnableContactBetweenFamilies(self, a: int, b: int):
        """Contact between families a and b is on again from the next detection."""
        self._set_family_contact(a, b, False)

    def _set_family_contact(self, a: int, b: int, prevent: bool):
        self.lib.deme_set_family_contact.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_int32]
        self._check(self.lib.deme_set_family_contact(self.h, int(a), int(b), int(prevent)), "set_family_contact")

    def set_family_change_rules(self, rules):
        """ChangeFamilyWhen rules, a list of (from, to, condition) applied every step (see
        deme_set_family_change_rules); an empty list removes them."""
        n = len(rules)
        fr = (C.c_uint32 * max(n, 1))(*[int(r[0]) for r in rules])
        to = (C.c_uint32 * max(n, 1))(*[int(r[1]) for r in rules])
        cond = (C.c_char_p * max(n, 1))(*[r[2].encode() for r in rules])
        self.lib.deme_set_family_change_rules.argtypes = [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p]
        self._check(self.lib.deme_set_family_change_rules(self.h, n, fr, to, cond), "set_family_change_rules")

    def set_prescribed_motion(self, families):
        """Prescribed motions written as expressions, one dict per family with keys family, lin_vel, ang_vel,
        lin_pos (three strings each, "none" = free) and the four *_prescribed flags (see
        deme_set_prescribed_motion); an empty list returns every family to its constant table entry."""
        n = len(families)
        arr = (capi.MotionExpressions * max(n, 1))()
        keep = []

        def enc(x):
            if x is None or x == "none":
                return None
            b = str(x).encode()
            keep.append(b)
            return b
        for i, f in enumerate(families):
            e = arr[i]
            e.family = int(f["family"])
            for k in ("lin_vel_prescribed", "rot_vel_prescribed", "lin_pos_prescribed", "rot_pos_prescribed"):
                setattr(e, k, int(bool(f.get(k, False))))
            for k in ("lin_vel", "ang_vel", "lin_pos"):
                xs = list(f.get(k, ["none"] * 3))
                for c in range(3):
                    getattr(e, k)[c] = enc(xs[c])
        self.lib.deme_set_prescribed_motion.argtypes = [C.c_void_p, C.c_int32, C.c_void_p]
        self._check(self.lib.deme_set_prescribed_motion(self.h, n, arr), "set_prescribed_motion")

    def set_search_shape(self, shape: int, cell_factor: float = 1.0):
        """Block shape of the pooled pair search and search-cell scale (see deme_set_search_shape)."""
        self.lib.deme_set_search_shape.argtypes = [C.c_void_p, C.c_int32, C.c_float]
        self._check(self.lib.deme_set_search_shape(self.h, int(shape), float(cell_factor)), "set_search_shape")

    def set_kernel_shapes(self, force_shape: int = 0, exact_threads: int = 256, integrate_threads: int = 256):
        """Block shapes of the force kernel, the exact pair test and the integration (see deme_set_kernel_shapes)."""
        self.lib.deme_set_kernel_shapes.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.c_int32]
        self._check(self.lib.deme_set_kernel_shapes(self.h, int(force_shape), int(exact_threads),
                                                    int(integrate_threads)), "set_kernel_shapes")

    def autotune(self, steps_per_trial: int = 5) -> dict:
        """Times every search shape and keeps the fastest; the state is left as it was (see deme_autotune)."""
        t = capi.Tuning()
        self.lib.deme_autotune.argtypes = [C.c_void_p, C.c_int32, C.POINTER(capi.Tuning)]
        self._check(self.lib.deme_autotune(self.h, int(steps_per_trial), C.byref(t)), "autotune")
        return {name: getattr(t, name) for name, _ in capi.Tuning._fields_}

    def keep_contact_forces(self, enable: bool = True):
        self.lib.deme_keep_contact_forces.argtypes = [C.c_void_p, C.c_int32]
        self._check(self.lib.deme_keep_contact_forces(self.h, int(enable)), "keep_contact_forces")

    def set_force_model(self, src: str | None, wildcards=()):
        names = (C.c_char_p * max(len(wildcards), 1))(*[w.encode() for w in wildcards])
        self._check(self.lib.deme_set_force_model(self.h, src.encode() if src else None, names, len(wildcards)),
                    "set_force_model")
        self.nW = len(wildcards) if src else self._params.n_contact_wildcards
