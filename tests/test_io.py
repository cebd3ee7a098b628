"""CSV output and input in DEM-Engine's formats (deme_b200.io) on a run of the C oracle, no GPU needed: the files hold
what the state and the contact list hold, and a clump file reads back."""
import numpy as np

from _util import oracle, workloads
from deme_b200 import io
from deme_b200 import statistics as stats


def _read(path):
    lines = open(path).read().splitlines()
    return lines[0].split(","), [line.split(",") for line in lines[1:]]


def test_sphere_clump_and_contact_files(tmp_path):
    built = workloads.packed_clumps(n_clumps=200, seed=5, spacing=1.3)
    o = oracle(built)
    o.step(3)
    o.SetOutputContent(io.ABSV | io.VEL | io.FAMILY)
    o.SetContactOutputContent(io.FORCE | io.POINT | io.NORMAL | io.TORQUE_ONLY_FORCE)
    o.WriteSphereFile(str(tmp_path / "s.csv"))
    o.WriteClumpFile(str(tmp_path / "c.csv"))
    o.WriteContactFile(str(tmp_path / "k.csv"))
    st = o.state()

    head, rows = _read(tmp_path / "s.csv")
    assert head == ["X", "Y", "Z", "r", "absv", "v_x", "v_y", "v_z", "family"]
    assert len(rows) == built.n_spheres
    r = np.array([float(x[3]) for x in rows])
    np.testing.assert_allclose(r, built.arrays["radius"], rtol=1e-5)

    head, rows = _read(tmp_path / "c.csv")
    assert head == ["X", "Y", "Z", "Qw", "Qx", "Qy", "Qz", "clump_type", "absv", "v_x", "v_y", "v_z", "family"]
    n = built.info["n_clumps"]
    xyz = np.array([[float(v) for v in x[:3]] for x in rows])
    np.testing.assert_allclose(xyz, stats.world_positions(built, st)[:n], rtol=1e-5, atol=1e-7)
    names = built.info["template_names"]
    assert [x[7] for x in rows] == [names[t] for t in built.info["owner_template"]]
    back = io.read_clump_xyz_from_csv(str(tmp_path / "c.csv"))
    for name, pts in back.items():
        sel = np.array([x[7] == name for x in rows])
        np.testing.assert_allclose(pts, xyz[sel].astype(np.float32), rtol=1e-5, atol=1e-7)
    q = io.read_clump_quat_from_csv(str(tmp_path / "c.csv"))
    assert sum(len(v) for v in q.values()) == n

    head, rows = _read(tmp_path / "k.csv")
    assert head[:3] == ["A", "B", "contact_type"] and len(head) == 15
    c = o.contacts()
    assert len(rows) == len(c["idA"]) > 0
    owner = built.arrays["sphere_owner"]
    assert [int(x[0]) for x in rows] == list(owner[c["idA"]])
    f = o.contact_forces()
    np.testing.assert_allclose(np.array([[float(v) for v in x[3:6]] for x in rows]), f["force"], rtol=1e-5,
                               atol=1e-6 * np.abs(f["force"]).max())
    nrm = np.array([[float(v) for v in x[9:12]] for x in rows])
    active = np.any(f["force"] != 0, axis=1)
    np.testing.assert_allclose(np.linalg.norm(nrm[active], axis=1), 1.0, rtol=1e-4)
