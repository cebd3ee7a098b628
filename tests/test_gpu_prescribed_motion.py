"""Prescribed motions written as expressions of the time (deme_set_prescribed_motion) on the GPU.

The shaker box (workloads.shaker_box) moves three families by expressions: a piston layer with a dictated vertical
velocity that switches on at t = 1e-4 s, a slider whose X follows a line in t, and a layer whose spin is added to
its integrated motion.

* Against the reference's own integration kernel, NVRTC-compiled on the same GPU with the same strings pasted in
  (oracle/ref_gpu_*): from the same state, one step at a time, the prescribed components come out bit for bit
  (velocities, spins, voxel codes), and the rest within the force tolerance.
* Against the C oracle, given before each step the values the expressions take at that step's float time: whole
  runs step by step and replayed from CUDA graphs keep the oracle's contact lists, and the prescribed components
  equal the oracle's.
* An expression that does not compile is refused with the compiler's log.
"""
import numpy as np
import pytest

from _util import canonical, oracle, set_oracle_motion, shaker_motion, workloads

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def test_prescribed_components_match_reference_kernels_on_gpu():
    from deme_b200 import Solver
    from oracle import ref_gpu, ref_gpu_build
    built = ref_gpu_build.parity_scene("shaker")
    if not ref_gpu.prebuilt(built, fmad=False) and not ref_gpu_build.available():
        pytest.skip("reference kernels for this scene were not prebuilt and the reference sources are absent")
    ours = Solver(built)
    ref = ref_gpu.RefGPU(built, fmad=False)
    fam = built.initial_state()["family"]
    piston, slider, spinner = fam == 1, fam == 2, fam == 3
    seen_piston = False
    for step in range(30):
        ref.set_state(ours.state())
        for s in (ours, ref):
            s.detect_contacts()
        co, cr = ours.contacts(), canonical(ref.contacts())
        for k in ("idA", "idB", "type"):
            np.testing.assert_array_equal(co[k], cr[k], err_msg=f"step {step} {k}")
        for s in (ours, ref):
            s.compute_forces()
            s.integrate()
        so, sr = ours.state(), ref.state()
        for k in ("vX", "vY", "vZ", "omgX", "omgY", "omgZ"):
            np.testing.assert_array_equal(so[k][piston], sr[k][piston], err_msg=f"step {step} piston {k}")
        for k in ("voxel", "locX", "locY", "locZ", "oriQw", "oriQx", "oriQy", "oriQz"):
            np.testing.assert_array_equal(so[k][slider], sr[k][slider], err_msg=f"step {step} slider {k}")
        # the spinner layer integrates its forces too; its spin is the expression plus alpha * h
        d = np.abs(so["omgZ"][spinner].astype(np.float64) - sr["omgZ"][spinner].astype(np.float64))
        assert d.max() <= 1e-5 * np.abs(sr["omgZ"][spinner]).max() + 1e-6, d.max()
        pos_o = built.decode_positions(so, kernel_literals=False)
        pos_r = built.decode_positions(sr, kernel_literals=False)
        assert np.abs(pos_o - pos_r).max() <= 1e-9, np.abs(pos_o - pos_r).max()
        seen_piston |= bool(np.any(so["vZ"][piston] != 0))
    assert seen_piston
    ref.close()
    ours.close()


@pytest.mark.parametrize("graph", [False, True], ids=["step_by_step", "graph"])
def test_expressions_match_the_oracle(graph):
    from deme_b200 import Solver
    built = workloads.shaker_box()
    g = Solver(built)
    if graph:
        g.set_graph(True)
    o = oracle(built)
    h = np.float32(built.params.h)
    t = np.float32(0.0)
    fam = built.initial_state()["family"]
    piston, slider = fam == 1, fam == 2
    for chunk in range(4):
        g.step(10)
        for _ in range(10):
            set_oracle_motion(o, shaker_motion(t))
            o.step(1)
            t = np.float32(t + h)
        sg, so = g.state(), o.state()
        cg, co = g.contacts(), canonical(o.contacts())
        for k in ("idA", "idB", "type"):
            np.testing.assert_array_equal(cg[k], co[k], err_msg=f"chunk {chunk} {k}")
        np.testing.assert_array_equal(sg["vZ"][piston], so["vZ"][piston], err_msg=f"chunk {chunk} piston vZ")
        np.testing.assert_array_equal(sg["voxel"][slider], so["voxel"][slider], err_msg=f"chunk {chunk} slider")
        np.testing.assert_array_equal(sg["locX"][slider], so["locX"][slider], err_msg=f"chunk {chunk} slider")
        pg = built.decode_positions(sg, kernel_literals=False)
        po = built.decode_positions(so, kernel_literals=False)
        assert np.abs(pg - po).max() <= 1e-8, np.abs(pg - po).max()
    # the piston switched on (t passed 1e-4 s) and the host's float time matches the device's
    assert np.any(g.state()["vZ"][piston] != 0)
    if graph:
        assert g.graph_stats()[0] > 0
    g.close()


def test_expression_that_does_not_compile_is_refused():
    from deme_b200 import Solver
    from deme_b200.solver import DemeError
    g = Solver(workloads.shaker_box())
    with pytest.raises(DemeError, match="family_7_lin_vel_z"):
        g.set_prescribed_motion([dict(family=7, lin_vel=["0", "0", "sin(q * t)"], ang_vel=["none"] * 3,
                                      lin_pos=["none"] * 3, lin_vel_prescribed=True, rot_vel_prescribed=True)])
    g.step(2)  # the earlier set stays in place
    g.set_prescribed_motion([])  # back to the constant table for every family
    g.step(2)
    g.close()
