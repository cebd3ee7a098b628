"""CSV numbers read as the reference's CSV reader forms them, in both front ends.

The reference reads clump templates (DEMClumpTemplate::ReadComponentFromFile, src/DEM/Structs.h:419-437) and restart
positions (ReadClumpXyzFromCsv, src/DEM/API.h:328-347) with a CSV reader whose float parse is not correctly rounded
(io::detail::parse_float<float>, src/core/utils/csv.hpp:936-997).  On random decimal strings a correctly rounded
parse differs from it in about 40 % of the values, by a few units in the last place, so a template read that way would
not be the reference's template.  deme_b200.io.csv_floats and deme::csv_float restate that parse; here both are
checked bit for bit against the reference's reader, compiled here (oracle/ref_build.py, ``oracle/_ref/ref_csv_dump``),
on the reference's six clump files (data/clumps), on 20,000 random decimal strings, and on a clump file written by
this project's writer.  Without the reference's sources, the two front ends are checked against each other and
against fixed values.
"""
import os
import subprocess

import numpy as np
import pytest

from _util import ROOT
from deme_b200 import solver
from deme_b200.io import csv_floats, read_clump_xyz_from_csv
from deme_b200.scene import read_clump_components

f32 = np.float32
CUDA_INC = "/usr/local/cuda/include"


def _ref():
    from oracle import ref_build
    if not os.path.exists(os.path.join(ref_build.REF_SRC, "core", "utils", "csv.hpp")):
        return None
    return ref_build


@pytest.fixture(scope="module")
def cpp_exe(tmp_path_factory):
    d = tmp_path_factory.mktemp("csvcpp")
    exe = str(d / "csv_dump")
    libdir = os.path.dirname(solver.LIB_PATH)
    subprocess.check_call(["g++", "-std=c++17", "-O1", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), "-I",
                           CUDA_INC, os.path.join(ROOT, "tests", "cpp", "csv_dump.cpp"), "-o", exe, "-L", libdir,
                           "-ldeme_b200", f"-Wl,-rpath,{libdir}"])
    return exe


def _dump(exe, mode, path, tmp_path):
    from oracle.ref_build import read_csv_dump
    out = tmp_path / f"{os.path.basename(exe)}_{mode}.bin"
    subprocess.check_call([exe, mode, str(path), str(out)])
    return read_csv_dump(str(out))


def _bits(a):
    return np.ascontiguousarray(a, f32).view(np.uint32)


def _random_cells(n=20000, seed=0):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        k = int(rng.integers(0, 5))
        if k == 0:
            s = repr(float(rng.normal()))
        elif k == 1:
            s = f"{rng.normal() * 10.0 ** int(rng.integers(-8, 8)):.{int(rng.integers(1, 18))}g}"
        elif k == 2:
            s = f"{rng.uniform(-1, 1):.{int(rng.integers(1, 20))}f}"
        elif k == 3:
            s = f"{rng.normal():.6e}"
        else:
            s = str(int(rng.integers(-100000, 100000)))
        out.append(s.replace("e+", "e"))  # the reference's reader rejects an exponent written with '+'
    return out


def _clump_files():
    rb = _ref()
    if rb is None or not os.path.isdir(rb.CLUMP_DIR):
        return []
    return sorted(os.path.join(rb.CLUMP_DIR, f) for f in os.listdir(rb.CLUMP_DIR) if f.endswith(".csv"))


@pytest.mark.parametrize("path", _clump_files() or [pytest.param(None, marks=pytest.mark.skip("no reference"))],
                         ids=lambda p: os.path.basename(p) if p else "none")
def test_reference_clump_files_read_as_the_reference_reads_them(path, cpp_exe, tmp_path):
    ref, _ = _dump(_ref().build_csv_dump(), "comp", path, tmp_path)
    r, p = read_clump_components(path)
    py = np.concatenate([p, r[:, None]], 1)
    assert py.shape == ref.shape
    np.testing.assert_array_equal(_bits(py), _bits(ref))
    cpp, _ = _dump(cpp_exe, "comp", path, tmp_path)
    np.testing.assert_array_equal(_bits(cpp), _bits(ref))


def test_random_decimals_read_as_the_reference_reads_them(cpp_exe, tmp_path):
    cells = _random_cells()
    path = tmp_path / "random.csv"
    with open(path, "w") as fh:
        fh.write("x,y,z,r\n")
        for i in range(0, len(cells), 4):
            fh.write(",".join(cells[i:i + 4]) + "\n")
    py = csv_floats(cells).reshape(-1, 4)
    cpp, _ = _dump(cpp_exe, "comp", path, tmp_path)
    np.testing.assert_array_equal(_bits(cpp), _bits(py))
    nearest = np.array(cells, np.float64).astype(f32).reshape(-1, 4)
    assert np.abs(py.astype(np.float64) - nearest).max() <= 8 * np.spacing(np.abs(nearest)).max()
    rb = _ref()
    if rb is not None:
        ref, _ = _dump(rb.build_csv_dump(), "comp", path, tmp_path)
        np.testing.assert_array_equal(_bits(py), _bits(ref))
        # the reader is not correctly rounded: a correctly rounded parse is not the reference's template
        assert np.sum(_bits(nearest) != _bits(ref)) > len(cells) // 10


def test_clump_position_file_reads_as_the_reference_reads_it(cpp_exe, tmp_path):
    """ReadClumpXyzFromCsv on a clump file in the reference writer's number format (6 significant digits, small
    values with a negative exponent), three template names, blank lines, spaces around cells."""
    rng = np.random.default_rng(3)
    xyz = (rng.normal(0, 0.05, (300, 3)) * (10.0 ** rng.integers(-6, 1, (300, 1)))).astype(f32)
    names = [("sphere_a", "clump_b", "x")[int(i)] for i in rng.integers(0, 3, 300)]
    path = tmp_path / "clumps.csv"
    with open(path, "w") as fh:
        fh.write("X,Y,Z,clump_type,Qw\n")
        for k, (p, n) in enumerate(zip(xyz, names)):
            cells = [f"{float(v):g}".replace("e+", "e") for v in p]
            fh.write(" " + ", ".join(cells) + f",{n},1\n")
            if k % 97 == 0:
                fh.write("\n")
    py = read_clump_xyz_from_csv(str(path))
    cpp, cpp_names = _dump(cpp_exe, "xyz", path, tmp_path)
    order = sorted(py)
    np.testing.assert_array_equal(_bits(cpp[:, :3]), _bits(np.concatenate([py[k] for k in order])))
    assert cpp_names == [k for k in order for _ in range(len(py[k]))]
    rb = _ref()
    if rb is not None:
        ref, ref_names = _dump(rb.build_csv_dump(), "xyz", path, tmp_path)
        assert ref_names == names
        for k in order:
            np.testing.assert_array_equal(_bits(py[k]), _bits(ref[np.array(ref_names) == k, :3]))


def test_fixed_values_and_malformed_cells():
    # values whose float sums are exact, an empty cell, signs, spaces and tabs
    got = csv_floats(["1", "-2.5", "+0.25", "", " 3 ", "\t4.5\t", "1e3", "25e-1", "-0.5E1", "7,5"])
    np.testing.assert_array_equal(got, np.array([1, -2.5, 0.25, 0, 3, 4.5, 1000, 2.5, -5, 7.5], f32))
    # the float accumulation: 0.1 formed as 1 * (1 / 10) in float is the nearest float; 0.3 is 3 * 0.1f
    assert csv_floats(["0.3"])[0] == f32(3) * (f32(1) / f32(10))
    for bad in ("1.2.3", "abc", "1e", "1e-x", "--1", "1 2"):
        if bad == "1e":
            assert csv_floats([bad])[0] == 1  # an empty exponent reads as none, as in the reference
            continue
        with pytest.raises(ValueError):
            csv_floats([bad])
