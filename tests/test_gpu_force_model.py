"""User force-model strings compiled at run time (NVRTC) into the force-kernel template, through the C ABI.

* A string that states the frictional Hertz-Mindlin model in the force-model dialect (the reference's variable
  names and helpers) reproduces the built-in model on the same contacts within 1e-5 relative.
* A string that writes its inputs out (normal, overlap depth, radius, mass) binds every name to the right value:
  checked against the geometry recomputed in float64 from the downloaded state.
* Per-contact wildcards persist through the history map; a string that does not compile reports DEME_ERR_NVRTC
  with the compiler log; NULL restores the built-in model.
"""
import ctypes as C

import numpy as np
import pytest

from _util import workloads, capi
from test_gpu_parity import gpu_solver

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

HERTZ_MINDLIN = r"""
float E_cnt, G_cnt, CoR_cnt, mu_cnt, Crr_cnt;
matProxy2ContactParam<float>(E_cnt, G_cnt, CoR_cnt, mu_cnt, Crr_cnt, E[bodyAMatType], nu[bodyAMatType],
                             CoR[bodyAMatType], mu[bodyAMatType], Crr[bodyAMatType], E[bodyBMatType],
                             nu[bodyBMatType], CoR[bodyBMatType], mu[bodyBMatType], Crr[bodyBMatType]);
float3 rotVelCPA = cross(ARotVel, locCPA);
float3 rotVelCPB = cross(BRotVel, locCPB);
applyOriQToVector3<float, deme::oriQ_t>(rotVelCPA.x, rotVelCPA.y, rotVelCPA.z, AoriQw, AoriQx, AoriQy, AoriQz);
applyOriQToVector3<float, deme::oriQ_t>(rotVelCPB.x, rotVelCPB.y, rotVelCPB.z, BoriQw, BoriQx, BoriQy, BoriQz);
const float3 velB2A = (ALinVel + rotVelCPA) - (BLinVel + rotVelCPB);
const float projection = dot(velB2A, B2A);
const float3 vrel_tan = velB2A - projection * B2A;
float3 delta_tan = make_float3(delta_tan_x, delta_tan_y, delta_tan_z);
delta_tan += ts * vrel_tan;
delta_tan -= dot(delta_tan, B2A) * B2A;
delta_time += ts;
const float mass_eff = (AOwnerMass * BOwnerMass) / (AOwnerMass + BOwnerMass);
const float sqrt_Rd = (float)sqrt(overlapDepth * (double)(ARadius * BRadius) / (double)(ARadius + BRadius));
const float Sn = (float)(2. * (double)E_cnt * (double)sqrt_Rd);
const float loge = (float)(((double)CoR_cnt < DEME_TINY_FLOAT) ? log(DEME_TINY_FLOAT) : (double)logf(CoR_cnt));
const float beta = (float)((double)loge / sqrt((double)(loge * loge) + deme::PI_SQUARED));
const float k_n = (float)(deme::TWO_OVER_THREE * (double)Sn);
const float gamma_n = (float)(deme::TWO_TIMES_SQRT_FIVE_OVER_SIX * (double)beta * (double)sqrtf(Sn * mass_eff));
force += (float)((double)k_n * overlapDepth + (double)(gamma_n * projection)) * B2A;
if (mu_cnt > 0.0f) {
    const float kt = (float)(8. * (double)G_cnt * (double)sqrt_Rd);
    const float gt = (float)(-deme::TWO_TIMES_SQRT_FIVE_OVER_SIX * (double)beta * (double)sqrtf(mass_eff * kt));
    float3 tangent_force = (-kt) * delta_tan - gt * vrel_tan;
    const float ft = length(tangent_force);
    if (ft > DEME_TINY_FLOAT) {
        const float ft_max = length(force) * mu_cnt;
        if (ft > ft_max) {
            tangent_force = (ft_max / ft) * tangent_force;
            delta_tan = (tangent_force + gt * vrel_tan) / (-kt);
        }
    } else {
        tangent_force = make_float3(0.f, 0.f, 0.f);
    }
    force += tangent_force;
}
delta_tan_x = delta_tan.x;
delta_tan_y = delta_tan.y;
delta_tan_z = delta_tan.z;
"""
HM_WILDCARDS = ("delta_tan_x", "delta_tan_y", "delta_tan_z", "delta_time")

PROBE = r"""
force = B2A;
torque_only_force = make_float3((float)overlapDepth, ARadius, BOwnerMass);
steps_seen += 1.0f;
"""


def set_model(g, src, names):
    arr = (C.c_char_p * max(len(names), 1))(*[n.encode() for n in names])
    g.lib.deme_set_force_model.argtypes = [C.c_void_p, C.c_char_p, C.POINTER(C.c_char_p), C.c_int32]
    return g.lib.deme_set_force_model(g.h, src.encode() if src is not None else None, arr, len(names))


def test_user_string_reproduces_builtin_model():
    built = workloads.packed_clumps(n_clumps=300, seed=41, spacing=1.3)
    g_ref = gpu_solver(built)
    g_usr = gpu_solver(built)
    assert set_model(g_usr, HERTZ_MINDLIN, HM_WILDCARDS) == 0, g_usr.lib.deme_get_error(g_usr.h)
    for step in range(6):
        for g in (g_ref, g_usr):
            g.detect_contacts()
            g.compute_forces()
        fr, fu = g_ref.contact_forces(), g_usr.contact_forces()
        cr, cu = g_ref.contacts(), g_usr.contacts()
        np.testing.assert_array_equal(cr["idB"], cu["idB"])
        big = max(np.abs(fr["force"]).max(initial=0), 1e-30)
        # rolling resistance is not part of the string: compare the forces, which it does not change
        np.testing.assert_allclose(fu["force"], fr["force"], rtol=1e-5, atol=1e-6 * big, err_msg=f"step {step}")
        np.testing.assert_allclose(cu["wildcards"][:3], cr["wildcards"][:3], rtol=1e-5,
                                   atol=1e-6 * max(np.abs(cr["wildcards"][:3]).max(initial=0), 1e-30))
        # same state for both before the next step
        for g in (g_ref, g_usr):
            g.integrate()
        g_usr.set_state({k: v for k, v in g_ref.state().items() if not k.startswith("a")})


def sphere_positions(built, st):
    a = built.arrays
    o = a["sphere_owner"].astype(np.int64)
    P = built.decode_positions(st)[o]
    q = np.stack([st[k][o] for k in ("oriQw", "oriQx", "oriQy", "oriQz")], 1).astype(np.float64)
    v = np.stack([a["relX"], a["relY"], a["relZ"]], 1).astype(np.float64)
    w, x, y, z = q.T
    u = np.stack([x, y, z], 1)
    t = 2 * np.cross(u, v)
    return P + v + w[:, None] * t + np.cross(u, t)


def test_probe_string_binds_names_to_the_kernel_values():
    built = workloads.packed_clumps(n_clumps=200, seed=42, spacing=1.3)
    g = gpu_solver(built)
    assert set_model(g, PROBE, ["steps_seen"]) == 0, g.lib.deme_get_error(g.h)
    K = 4
    for _ in range(K):
        g.detect_contacts()
        g.compute_forces()
    c, f, st = g.contacts(), g.contact_forces(), g.state()
    ss = c["type"] == capi.SPHERE_SPHERE_CONTACT
    assert ss.sum() > 20
    pos = sphere_positions(built, st)
    A, B = c["idA"][ss].astype(np.int64), c["idB"][ss].astype(np.int64)
    d = pos[A] - pos[B]
    dist = np.linalg.norm(d, axis=1)
    rA = built.arrays["radius"][A].astype(np.float64)
    rB = built.arrays["radius"][B].astype(np.float64)
    depth = rA + rB - dist
    active = depth > 0
    n_exp = d / dist[:, None]
    np.testing.assert_allclose(f["force"][ss][active], n_exp[active], atol=1e-5)
    np.testing.assert_allclose(f["torque_only_force"][ss][active][:, 0], depth[active], atol=1e-6 * rA.max())
    np.testing.assert_allclose(f["torque_only_force"][ss][active][:, 1], rA[active], rtol=1e-7)
    mass = built.arrays["mass"][built.arrays["sphere_owner"][B]].astype(np.float64)
    np.testing.assert_allclose(f["torque_only_force"][ss][active][:, 2], mass[active], rtol=1e-7)
    # the wildcard counts the steps each contact has been active (the state is unchanged, so all persist)
    wc = c["wildcards"][0][ss][active]
    assert np.all(wc == K), np.unique(wc)


def test_bad_string_reports_the_compiler_log_and_null_restores_builtin():
    built = workloads.packed_clumps(n_clumps=100, seed=43, spacing=1.3)
    g = gpu_solver(built)
    rc = set_model(g, "force = this is not C++;", [])
    assert rc == 5  # DEME_ERR_NVRTC
    msg = g.lib.deme_get_error(g.h).decode()
    assert "force_model_string" in msg, msg
    assert set_model(g, "force = make_float3(0.f, 0.f, 0.f);", ["a", "b", "c", "d", "e"]) == 1  # too many wildcards
    # back to the built-in model: forces equal a fresh solver's
    assert set_model(g, None, []) == 0
    ref = gpu_solver(built)
    for s in (g, ref):
        s.detect_contacts()
        s.compute_forces()
    np.testing.assert_array_equal(g.contact_forces()["force"], ref.contact_forces()["force"])
