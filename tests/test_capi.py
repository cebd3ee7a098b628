"""The C-ABI library loads without a GPU and exports every entry point include/deme_b200.h declares; struct layouts
of the ctypes mirror match the header's sizes."""
import ctypes as C
import os
import re
import subprocess

import pytest

from _util import ROOT, capi
from deme_b200 import solver

HEADER = os.path.join(ROOT, "include", "deme_b200.h")


def declared_functions():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^[a-z_0-9 ]+\*?\s*\*?(deme_[a-z_0-9]+)\(", text, re.M)))


def test_header_declares_entry_points():
    names = declared_functions()
    assert "deme_create" in names and "deme_step" in names and len(names) >= 25


def test_library_exports_every_declared_symbol():
    lib = solver.load_product_library()
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_abi_version_and_status_strings():
    lib = solver.load_product_library()
    assert lib.deme_abi_version() == 5
    assert lib.deme_status_string(0) == b"DEME_OK"
    assert lib.deme_status_string(6) == b"DEME_ERR_TIMEOUT"


def test_struct_sizes_match_header(tmp_path):
    # compile a tiny C program against the header and compare sizeof with the ctypes mirror
    src = r"""
    #include <stdio.h>
    #include "deme_b200.h"
    int main(void) {
        printf("%zu %zu %zu %zu %zu %zu\n", sizeof(deme_sim_params), sizeof(deme_family_prescription),
               sizeof(deme_scene), sizeof(deme_state), sizeof(deme_contacts), sizeof(deme_contact_forces));
        return 0;
    }
    """
    tmp = str(tmp_path / "sizes")
    with open(tmp + ".c", "w") as f:
        f.write(src)
    subprocess.check_call(["gcc", "-I", os.path.join(ROOT, "include"), tmp + ".c", "-o", tmp])
    sizes = [int(x) for x in subprocess.check_output([tmp]).split()]
    mirror = [C.sizeof(capi.SimParams), C.sizeof(capi.FamilyPrescription), C.sizeof(capi.Scene),
              C.sizeof(capi.State), C.sizeof(capi.Contacts), C.sizeof(capi.ContactForces)]
    assert sizes == mirror


def test_create_without_gpu_reports_no_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from _util import workloads
    built = workloads.packed_clumps(n_clumps=8, seed=1)
    with pytest.raises(solver.DemeError, match="NO_DEVICE"):
        solver.Solver(built)
