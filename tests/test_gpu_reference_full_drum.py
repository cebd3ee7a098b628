"""The headline contact-list claim at full size: the 1M-clump shell drum (1M three-sphere clumps + 129k fixed shell
spheres + two end planes, 3.13M spheres, on the dense start lattice with the settled bed's contact density), the
scene the benchmark times the reference's own kernels on.

From one injected state per step, this build's contact detection and the reference's kernels (NVRTC-compiled for
sm_100a and launched in the order of its kT and dT threads by oracle/ref_gpu_harness.cu) must give:

* with FMA contraction off in the reference's build (the build that reproduces its arithmetic operation by
  operation): bit-exact contact lists in canonical order, bit-exact history partners and remapped history, and
  per-contact forces within 1e-5 relative;
* with the reference's stock build (NVRTC's default FMA contraction, the build the benchmark times): the lists may
  differ only where contraction moves a rounding-sensitive decision -- a pair whose overlap margin, contact-point
  bin coordinate or bin-range bound lies within 1e-6 (relative) of its threshold.  The differing pairs are counted
  and printed; every one of them must be such a tie.

The tie test restates in numpy, operation by operation, the decisions of the reference's bin assignment and pair
test (src/kernel/DEMBinSphereKernels.cu:39-64, src/kernel/DEMHelperKernels.cu:93-110, 137-148, 195-222, 266-273).
"""
import numpy as np
import pytest

from _util import canonical, capi, partner_keys

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

from oracle import ref_gpu, ref_gpu_build  # noqa: E402

f32 = np.float32


def _scene():
    built = ref_gpu_build.bench_shell_drum()
    return built


def _need(built, fmad):
    if not ref_gpu.prebuilt(built, fmad=fmad) and not ref_gpu_build.available():
        pytest.skip("reference kernels for the full drum were not prebuilt and the reference sources are absent")


def sphere_centres(built, st):
    """Sphere centres as the kernels form them: owner position decoded in double, relative position rotated in
    float (no contraction), the sum in double."""
    p = built.params
    a = built.arrays
    owner = a["sphere_owner"].astype(np.int64)
    v = st["voxel"].astype(np.uint64)[owner]
    mx = np.uint64((1 << p.nvXp2) - 1)
    my = np.uint64((1 << p.nvYp2) - 1)
    vx = (v & mx).astype(np.float64)
    vy = ((v >> np.uint64(p.nvXp2)) & my).astype(np.float64)
    vz = (v >> np.uint64(p.nvXp2 + p.nvYp2)).astype(np.float64)
    vs, l = float(p.voxel_size_kernel), float(p.l_kernel)
    X = vx * vs + st["locX"].astype(np.float64)[owner] * l
    Y = vy * vs + st["locY"].astype(np.float64)[owner] * l
    Z = vz * vs + st["locZ"].astype(np.float64)[owner] * l
    w, x, y, z = (st[k][owner].astype(f32) for k in ("oriQw", "oriQx", "oriQy", "oriQz"))
    ox, oy, oz = (a[k].astype(f32) for k in ("relX", "relY", "relZ"))
    two, one = f32(2), f32(1)
    rx = (two * (w * w + x * x) - one) * ox + (two * (x * y - w * z)) * oy + (two * (x * z + w * y)) * oz
    ry = (two * (x * y + w * z)) * ox + (two * (w * w + y * y) - one) * oy + (two * (y * z - w * x)) * oz
    rz = (two * (x * z - w * y)) * ox + (two * (y * z + w * x)) * oy + (two * (w * w + z * z) - one) * oz
    return X + rx.astype(np.float64), Y + ry.astype(np.float64), Z + rz.astype(np.float64)


def _frac_dist(q):
    return np.abs(q - np.round(q))


def tie_margin(built, st, A, B):
    """For sphere pairs (A, B), the smallest distance of any rounding-sensitive decision from its threshold: the
    overlap test of the expanded radii (relative margin), the contact point's bin coordinate and the four bin-range
    bounds per axis (distance from the nearest integer, in bins)."""
    p = built.params
    X, Y, Z = sphere_centres(built, st)
    rf = (built.arrays["radius"].astype(f32) + f32(p.beta)).astype(np.float64)
    bs = float(p.bin_size)
    ax, ay, az, bx, by, bz = X[A], Y[A], Z[A], X[B], Y[B], Z[B]
    ra, rb = rf[A], rf[B]
    d2 = (ax - bx) ** 2 + (ay - by) ** 2 + (az - bz) ** 2
    s2 = (ra + rb) ** 2
    m = np.abs(s2 - d2) / s2
    nx, ny, nz = (ax - bx).astype(f32), (ay - by).astype(f32), (az - bz).astype(f32)
    nn = np.sqrt(nx * nx + ny * ny + nz * nz)
    nx, ny, nz = nx / nn, ny / nn, nz / nn
    half = (ra + rb - np.sqrt(d2)) / 2.0
    for c, n, r in ((bx, nx, rb), (by, ny, rb), (bz, nz, rb)):
        cp = c + (r - half) * n.astype(np.float64)
        m = np.minimum(m, _frac_dist(cp / bs))
    rD = (built.arrays["radius"].astype(np.float64) + float(f32(p.beta)))
    for P in (X, Y, Z):
        for ids in (A, B):
            q, span = P[ids] / bs, rD[ids] / bs
            m = np.minimum(m, np.minimum(_frac_dist(q - span), _frac_dist(q + span)))
    return m


def _keys(c):
    return (c["idA"].astype(np.int64) << 35) | (c["idB"].astype(np.int64) << 3) | c["type"].astype(np.int64)


@pytest.mark.parametrize("one_bin_per_thread", [True, False], ids=["thread_per_bin", "block_per_bin"])
def test_full_drum_bit_exact_against_reference_kernels_fma_off(one_bin_per_thread):
    from deme_b200 import Solver
    built = _scene()
    _need(built, False)
    ours = Solver(built)
    ours.keep_contact_forces(True)
    ref = ref_gpu.RefGPU(built, fmad=False)
    ref.set_one_bin_per_thread(one_bin_per_thread)
    prev_o = prev_r = None
    worst = 0.0
    n = []
    for step in range(3):
        ref.set_state(ours.state())
        ours.detect_contacts()
        ref.detect_contacts()
        co, cr = ours.contacts(), ref.contacts()
        rc = canonical(cr)
        for k in ("idA", "idB", "type"):
            np.testing.assert_array_equal(co[k], rc[k], err_msg=f"step {step} {k}")
        if prev_o is not None:
            np.testing.assert_array_equal(partner_keys(co, prev_o), partner_keys(cr, prev_r)[rc["perm"]],
                                          err_msg=f"step {step} history partners")
        np.testing.assert_array_equal(co["wildcards"], rc["wildcards"], err_msg=f"step {step} history")
        ours.compute_forces()
        ref.compute_forces()
        fo, fr = ours.contact_forces(), ref.contact_forces()
        fr = {k: v[rc["perm"]] for k, v in fr.items()}
        active = np.any(fr["force"] != 0, axis=1)
        np.testing.assert_array_equal(np.any(fo["force"] != 0, axis=1), active, err_msg=f"step {step} active")
        for k in ("force", "torque_only_force", "cpA", "cpB"):
            a, b = fo[k][active].astype(np.float64), fr[k][active].astype(np.float64)
            floor = 1e-6 * max(np.abs(b).max(initial=0), 1e-30)
            err = (np.abs(a - b) / (np.abs(b) + floor)).max(initial=0)
            worst = max(worst, err)
            assert err <= 1e-5, f"step {step} {k} rel err {err}"
        ours.integrate()
        prev_o, prev_r = co, cr
        n.append(len(co["idA"]))
    assert min(n) > 3_000_000
    print(f"full drum, FMA off, {'thread' if one_bin_per_thread else 'block'} per bin: {n} contacts bit-exact, "
          f"largest per-contact force difference {worst:.2e} relative")
    ref.close()
    ours.close()


def test_full_drum_against_stock_reference_kernels_fma_on():
    """The stock build contracts multiplies and adds into FMAs, so its per-contact forces are not the FMA-off
    build's.  Where the normal spring and damper nearly cancel (contacts about to separate) the contracted rounding
    moves a small force by a large fraction of itself, so the differences are measured and printed per component
    (floor 1e-6 of the largest) and per contact as a vector, and bounded over the whole list (norm of all
    differences over norm of all forces, 1e-5); the contact lists are the claim here."""
    from deme_b200 import Solver
    built = _scene()
    _need(built, True)
    ours = Solver(built)
    ours.keep_contact_forces(True)
    ref = ref_gpu.RefGPU(built, fmad=True)
    ref.set_one_bin_per_thread(True)
    total_diff = 0
    worst_tie = 0.0
    worst_comp = worst_vec = worst_all = 0.0
    n = []
    for step in range(3):
        st = ours.state()
        ref.set_state(st)
        ours.detect_contacts()
        ref.detect_contacts()
        co, cr = ours.contacts(), ref.contacts()
        ko, kr = _keys(co), _keys(cr)
        only_o = np.setdiff1d(ko, kr)
        only_r = np.setdiff1d(kr, ko)
        diff = np.concatenate([only_o, only_r])
        total_diff += len(diff)
        n.append(len(ko))
        if len(diff):
            t = diff & 7
            assert np.all(t == capi.SPHERE_SPHERE_CONTACT), "a sphere--plane contact differs"
            A, B = (diff >> 35).astype(np.int64), ((diff >> 3) & ((1 << 32) - 1)).astype(np.int64)
            m = tie_margin(built, st, A, B)
            worst_tie = max(worst_tie, float(m.max()))
            assert np.all(m <= 1e-6), f"step {step}: differing pairs that are not rounding ties: {m[m > 1e-6]}"
        ours.compute_forces()
        ref.compute_forces()
        fo, fr = ours.contact_forces(), ref.contact_forces()
        _, io, ir = np.intersect1d(ko, kr, return_indices=True)
        a, b = fo["force"][io].astype(np.float64), fr["force"][ir].astype(np.float64)
        active = np.any(b != 0, axis=1)
        a, b = a[active], b[active]
        floor = 1e-6 * max(np.abs(b).max(initial=0), 1e-30)
        worst_comp = max(worst_comp, float((np.abs(a - b) / (np.abs(b) + floor)).max(initial=0)))
        nb = np.linalg.norm(b, axis=1)
        worst_vec = max(worst_vec, float((np.linalg.norm(a - b, axis=1) / (nb + floor)).max(initial=0)))
        # over the whole list: the norm of all differences against the norm of all forces
        worst_all = max(worst_all, float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)))
        assert worst_all <= 1e-5, f"step {step}: forces far from the stock build's ({worst_all})"
        ours.integrate()
    print(f"full drum against the stock (FMA on) reference build: {n} contacts, {total_diff} differing pairs over "
          f"3 steps, all rounding ties (largest margin {worst_tie:.1e}); per-contact forces against its contracted "
          f"arithmetic: largest difference {worst_comp:.2e} per component, {worst_vec:.2e} per contact vector, "
          f"{worst_all:.2e} over the whole list")
    ref.close()
    ours.close()
