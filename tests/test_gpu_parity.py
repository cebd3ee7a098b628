"""CUDA path (through the C ABI) against the reference's outputs and the C oracle.

Bars (the reference fixtures were recorded from the reference's own kernels compiled for the CPU):
  * bin assignment, contact list (canonical order), history partners and remapped history: bit-exact;
  * per-contact force / torque-only force / local contact points: within 1e-5 relative (floor 1e-6 of the largest
    magnitude), the only differences being CUDA's logf/powf against glibc's;
  * owner accelerations: within 1e-5 of the sum of the magnitudes of their contributions (float atomics sum in a
    different order than the reference's reduce-by-key);
  * one-step state update: velocities within 1e-5 relative, positions within 1e-9 m, quaternions within 1e-6.
"""
import numpy as np
import pytest

from _util import (GOLDEN, canonical, contact_key, load_golden, oracle, partner_keys, workloads, capi)

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def gpu_solver(built, keep=True):
    from deme_b200 import Solver
    s = Solver(built)
    s.lib.deme_keep_contact_forces.argtypes = [__import__("ctypes").c_void_p, __import__("ctypes").c_int32]
    s.lib.deme_keep_contact_forces(s.h, 1 if keep else 0)
    return s


def rec_contacts(rec, prefix):
    return {k: rec[prefix + k] for k in ("idA", "idB", "type", "mapping", "wildcards")}


def owner_scale(built, c, f):
    """Per owner: sum over contacts of |F|/m (the magnitude of what gets accumulated)."""
    a = built.arrays
    nO = built.counts["o"]
    owner = a["sphere_owner"]
    oA = owner[c["idA"]]
    ss = c["type"] == capi.SPHERE_SPHERE_CONTACT
    me = c["type"] == capi.SPHERE_MESH_CONTACT
    an = ~ss & ~me
    oB = np.where(ss, owner[np.where(ss, c["idB"], 0)], a["anal_owner"][np.where(an, c["idB"], 0)] if len(
        a["anal_owner"]) else 0)
    if me.any():
        oB = np.where(me, a["tri_owner"][np.where(me, c["idB"], 0)], oB)
    Fm = np.linalg.norm(f["force"].astype(np.float64), axis=1) + np.linalg.norm(
        f["torque_only_force"].astype(np.float64), axis=1)
    lin = np.zeros(nO)
    np.add.at(lin, oA, Fm)
    np.add.at(lin, oB, Fm)
    return lin / a["mass"].astype(np.float64)


@pytest.mark.parametrize("name", GOLDEN)
def test_gpu_matches_reference_fixture_step_by_step(name):
    built, rec = load_golden(name)
    g = gpu_solver(built)
    # inject the reference's state and contact history at the start of the recorded window
    g.set_state({k: rec["pre_st_" + k] for k in ("voxel", "locX", "locY", "locZ", "oriQw", "oriQx", "oriQy", "oriQz",
                                                  "vX", "vY", "vZ", "omgX", "omgY", "omgZ", "family")})
    g.set_contacts(rec_contacts(rec, "pre_c_"))
    prev_ref = rec_contacts(rec, "pre_c_")
    for step in range(int(rec["steps"])):
        ref_c = rec_contacts(rec, f"s{step}_c_")
        g.detect_contacts()
        gc = g.contacts()
        # contact set and canonical order: bit-exact
        rc = canonical(ref_c)
        for k in ("idA", "idB", "type"):
            np.testing.assert_array_equal(gc[k], rc[k], err_msg=f"{name} step {step} {k}")
        # history partners: the same (idA, idB, type) in the previous list; remapped history bit-exact.  The
        # previous list on the GPU is the reference's list as injected (canonicalised on upload).
        ref_partner = partner_keys(ref_c, prev_ref)[rc["perm"]]
        gp = partner_keys(gc, canonical_contacts_of_upload(prev_ref))
        np.testing.assert_array_equal(gp, ref_partner, err_msg=f"{name} step {step} partners")
        np.testing.assert_array_equal(gc["wildcards"], rc["wildcards"], err_msg=f"{name} step {step} history")
        # forces
        g.compute_forces()
        gf = g.contact_forces()
        rf = {k: rec[f"s{step}_f_{k}"][rc["perm"]] for k in ("force", "torque_only_force", "cpA", "cpB")}
        active = np.any(rf["force"] != 0, axis=1)
        for k in ("force", "torque_only_force", "cpA", "cpB"):
            a, b = gf[k][active].astype(np.float64), rf[k][active].astype(np.float64)
            floor = 1e-6 * max(np.abs(b).max(initial=0), 1e-30)
            err = np.abs(a - b) / (np.abs(b) + floor)
            assert err.max(initial=0) <= 1e-5, f"{name} step {step} {k} rel err {err.max()}"
        gs = g.state()
        scale = owner_scale(built, {k: rc[k] for k in ("idA", "idB", "type")}, rf)
        for k in ("aX", "aY", "aZ"):
            d = np.abs(gs[k].astype(np.float64) - rec[f"s{step}_acc_{k}"])
            assert np.all(d <= 1e-5 * scale + 1e-30), f"{name} step {step} {k} max {np.max(d / (scale + 1e-30))}"
        # integrate
        g.integrate()
        gs = g.state()
        ref_st = {k: rec[f"s{step}_st_{k}"] for k in gs}
        for k in ("vX", "vY", "vZ", "omgX", "omgY", "omgZ"):
            a, b = gs[k].astype(np.float64), ref_st[k].astype(np.float64)
            assert np.all(np.abs(a - b) <= 1e-5 * np.abs(b) + 1e-5 * np.abs(b).max() + 1e-12), f"{name} {k}"
        pg, pr = built.decode_positions(gs), built.decode_positions(ref_st)
        assert np.abs(pg - pr).max() <= 1e-9, f"{name} step {step} position diff {np.abs(pg - pr).max()}"
        for k in ("oriQw", "oriQx", "oriQy", "oriQz"):
            assert np.abs(gs[k] - ref_st[k]).max() <= 1e-6, f"{name} step {step} {k}"
        # updated history within float rounding of the reference's
        post = g.contacts()["wildcards"].astype(np.float64)
        ref_post = rec[f"s{step}_cpost_wildcards"][:, rc["perm"]].astype(np.float64)
        assert np.all(np.abs(post - ref_post) <= 1e-5 * np.abs(ref_post) + 1e-6 * np.abs(ref_post).max(initial=0)
                      + 1e-30), f"{name} step {step} updated history"
        # re-inject the reference's state and history so every step starts from identical input
        g.set_state({k: ref_st[k] for k in ref_st if not k.startswith("a")})
        g.set_contacts({"idA": ref_c["idA"], "idB": ref_c["idB"], "type": ref_c["type"],
                        "wildcards": rec[f"s{step}_cpost_wildcards"]})
        prev_ref = ref_c


def canonical_contacts_of_upload(c):
    cc = canonical(c)
    return {"idA": cc["idA"], "idB": cc["idB"], "type": cc["type"]}


@pytest.mark.parametrize("name", GOLDEN)
def test_gpu_bin_assignment_bit_exact(name):
    built, rec = load_golden(name)
    g = gpu_solver(built, keep=False)
    g.set_state({k: rec["pre_st_" + k] for k in ("voxel", "locX", "locY", "locZ", "oriQw", "oriQx", "oriQy", "oriQz",
                                                  "family")})
    b = g.bin_assignment()
    for k in ("n_bins", "n_anal", "bins", "spheres"):
        np.testing.assert_array_equal(b[k], rec["bin_" + k], err_msg=f"{name} {k}")


@pytest.mark.parametrize("n,bits", [(1, 8), (1000, 9), (3841, 16), (100_000, 23), (1_000_003, 32), (2_000_000, 20)])
def test_onesweep_radix_sort_is_stable_and_exact(n, bits):
    import ctypes as C
    from deme_b200 import solver
    lib = solver.load_product_library()
    rng = np.random.default_rng(n + bits)
    hi = min(1 << bits, 1 << 32)
    keys = rng.integers(0, min(hi, max(2, n // 3)), n, dtype=np.uint64).astype(np.uint32)  # many duplicates
    vals = np.arange(n, dtype=np.uint32)
    dev = torch.device("cuda")
    kin = torch.from_numpy(keys.view(np.int32)).to(dev)
    vin = torch.from_numpy(vals.view(np.int32)).to(dev)
    kout = torch.empty_like(kin)
    vout = torch.empty_like(vin)
    lib.deme_radix_sort_scratch_bytes.restype = C.c_size_t
    lib.deme_radix_sort_scratch_bytes.argtypes = [C.c_uint32]
    nb = lib.deme_radix_sort_scratch_bytes(n)
    scratch = torch.empty(nb, dtype=torch.uint8, device=dev)
    lib.deme_radix_sort_pairs_device.argtypes = [C.c_void_p] * 4 + [C.c_uint32, C.c_int32, C.c_void_p, C.c_size_t,
                                                                     C.c_void_p]
    st = torch.cuda.current_stream().cuda_stream
    rc = lib.deme_radix_sort_pairs_device(kin.data_ptr(), vin.data_ptr(), kout.data_ptr(), vout.data_ptr(), n, bits,
                                          scratch.data_ptr(), nb, st)
    assert rc == 0
    torch.cuda.synchronize()
    order = np.argsort(keys, kind="stable")
    np.testing.assert_array_equal(kout.cpu().numpy().view(np.uint32), keys[order])
    np.testing.assert_array_equal(vout.cpu().numpy().view(np.uint32), vals[order])


def test_gpu_free_running_matches_oracle_statistics():
    """20 free-running steps of a dense clump scene: the contact list stays bit-identical while the states stay
    within float rounding, and the kinetic energies agree to 1e-4."""
    built = workloads.packed_clumps(n_clumps=400, seed=31, spacing=1.35)
    g = gpu_solver(built, keep=False)
    o = oracle(built)
    for step in range(20):
        g.step(1)
        o.step(1)
        gc, oc = g.contacts(), canonical(o.contacts())
        if step < 5:
            np.testing.assert_array_equal(contact_key(gc), contact_key(oc), err_msg=f"step {step}")
    ke_g, ke_o = g.kinetic_energy(), o.kinetic_energy()
    assert abs(ke_g - ke_o) <= 1e-4 * abs(ke_o), (ke_g, ke_o)


def test_gpu_empty_and_sparse_scenes():
    """No contacts at all (spheres far apart), then a step: the pipeline handles zero-length lists."""
    built = workloads.settling_box(n=27, r=2e-3, box=(0.2, 0.2, 0.2), spacing=10.0, jitter=0.0, seed=3)
    g = gpu_solver(built)
    g.detect_contacts()
    assert g.num_contacts() == 0
    g.compute_forces()
    g.integrate()
    o = oracle(built)
    o.step(1)
    st, so = g.state(), o.state()
    np.testing.assert_allclose(st["vZ"], so["vZ"], rtol=1e-6)


def test_cell_sort_variants_agree():
    """The counting sort (default) and the onesweep radix sort order spheres differently inside a cell; the contact
    list and its history must not depend on it."""
    import ctypes as C
    built = workloads.packed_clumps(n_clumps=500, seed=41, spacing=1.3)
    lists = []
    for onesweep in (0, 1):
        g = gpu_solver(built, keep=False)
        g.lib.deme_set_cell_sort.argtypes = [C.c_void_p, C.c_int32]
        g.lib.deme_set_cell_sort(g.h, onesweep)
        for _ in range(3):
            g.step(1)
        lists.append(g.contacts())
    for k in ("idA", "idB", "type", "mapping"):
        np.testing.assert_array_equal(lists[0][k], lists[1][k], err_msg=k)
