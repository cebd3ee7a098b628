"""The CUDA path against the reference's own kernels running on the same GPU.

The reference's kernel templates are substituted for each scene and compiled with NVRTC for sm_100a, with FMA
contraction off, by oracle/ref_gpu_build.py; oracle/ref_gpu_harness.cu launches them in the order of the reference's
kT and dT threads, with CUB for its device-wide primitives, with either of its two contact-kernel variants (block per
active bin, the default, or thread per active bin).  Each step starts both from the CUDA path's state, so the
comparison isolates one step:
  * contact list (canonical order: the reference's block-per-bin kernels write pairs in a nondeterministic order
    within a bin, which its stable sort by idA keeps), history partners and remapped history: bit-exact;
  * which contacts carry a force: identical; per-contact force, torque-only force and local contact points of those:
    within 1e-5 relative (floor 1e-6 of the largest magnitude);
  * owner accelerations: within 1e-5 of the sum of the magnitudes of their contributions (the reference sums by a
    radix sort and CUB's reduce-by-key, the CUDA path by warp segments and float atomics).
"""
import numpy as np
import pytest

from _util import canonical, partner_keys, capi

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

from oracle import ref_gpu, ref_gpu_build  # noqa: E402

STEPS = 6


def owner_scale(built, c, f):
    a = built.arrays
    nO = built.counts["o"]
    owner = a["sphere_owner"]
    oA = owner[c["idA"]]
    ss = c["type"] == capi.SPHERE_SPHERE_CONTACT
    anal_owner = a["anal_owner"] if len(a["anal_owner"]) else np.zeros(1, np.uint32)
    oB = np.where(ss, owner[np.where(ss, c["idB"], 0)], anal_owner[np.where(ss, 0, c["idB"])])
    Fm = np.linalg.norm(f["force"].astype(np.float64), axis=1) + np.linalg.norm(
        f["torque_only_force"].astype(np.float64), axis=1)
    tot = np.zeros(nO)
    np.add.at(tot, oA, Fm)
    np.add.at(tot, oB, Fm)
    return tot / a["mass"].astype(np.float64)


@pytest.mark.parametrize("one_bin_per_thread", [False, True], ids=["block_per_bin", "thread_per_bin"])
@pytest.mark.parametrize("name", list(ref_gpu_build.PARITY_SCENES))
def test_cuda_path_matches_reference_kernels_on_gpu(name, one_bin_per_thread):
    from deme_b200 import Solver
    built = ref_gpu_build.parity_scene(name)
    if not ref_gpu.prebuilt(built, fmad=False) and not ref_gpu_build.available():
        pytest.skip("reference kernels for this scene were not prebuilt and the reference sources are absent")
    ours = Solver(built)
    ours.keep_contact_forces(True)
    ref = ref_gpu.RefGPU(built, fmad=False)
    ref.set_one_bin_per_thread(one_bin_per_thread)
    prev_o = prev_r = None
    n_contacts = []
    worst_force = 0.0
    for step in range(STEPS):
        ref.set_state(ours.state())
        ours.detect_contacts()
        ref.detect_contacts()
        co, cr = ours.contacts(), ref.contacts()
        rc = canonical(cr)
        for k in ("idA", "idB", "type"):
            np.testing.assert_array_equal(co[k], rc[k], err_msg=f"{name} step {step} {k}")
        if prev_o is not None:
            np.testing.assert_array_equal(partner_keys(co, prev_o), partner_keys(cr, prev_r)[rc["perm"]],
                                          err_msg=f"{name} step {step} history partners")
        np.testing.assert_array_equal(co["wildcards"], rc["wildcards"], err_msg=f"{name} step {step} history")
        ours.compute_forces()
        ref.compute_forces()
        fo, fr = ours.contact_forces(), ref.contact_forces()
        fr = {k: v[rc["perm"]] for k, v in fr.items()}
        # contacts found with the expand margin but not touching get no force; the reference leaves their contact
        # points unwritten (prepareForceArrays clears forces only), so points are compared where a force acts
        active = np.any(fr["force"] != 0, axis=1)
        np.testing.assert_array_equal(np.any(fo["force"] != 0, axis=1), active, err_msg=f"{name} step {step} active")
        for k in ("force", "torque_only_force", "cpA", "cpB"):
            a, b = fo[k][active].astype(np.float64), fr[k][active].astype(np.float64)
            floor = 1e-6 * max(np.abs(b).max(initial=0), 1e-30)
            err = (np.abs(a - b) / (np.abs(b) + floor)).max(initial=0)
            worst_force = max(worst_force, err)
            assert err <= 1e-5, f"{name} step {step} {k} rel err {err}"
        so, sr = ours.state(), ref.state()
        scale = owner_scale(built, co, fr)
        for k in ("aX", "aY", "aZ"):
            d = np.abs(so[k].astype(np.float64) - sr[k].astype(np.float64))
            assert np.all(d <= 1e-5 * scale + 1e-30), f"{name} step {step} {k}"
        ours.integrate()
        ref.integrate()
        prev_o, prev_r = co, cr
        n_contacts.append(len(co["idA"]))
    assert max(n_contacts) > 0
    print(f"{name}: {n_contacts[-1]} contacts, largest per-contact force difference {worst_force:.2e} relative")
    ref.close()
    ours.close()
