"""deme_radix_sort_pairs_static, the sort whose scratch is a fixed __device__ array of the library (no device
allocation in the call), against deme_radix_sort_pairs_device on the same inputs.  It exists for callers that
cannot allocate: a host application whose own memory pool already holds the GPU's memory, or per-step code that
must not synchronise the device with a cudaMalloc.

This file is collected last so that it also runs after every other GPU test in the same process; it must pass
alone in a fresh process too (the first call does the per-device set-up)."""
import ctypes as C
import os
import subprocess
import sys

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from _util import ROOT
from deme_b200 import solver

pytestmark = pytest.mark.gpu

MAX_N = 1048576  # DEME_SORT_STATIC_MAX_N
DEME_ERR_INVALID = 1
DEME_ERR_TOO_LARGE = 9


def _lib():
    lib = solver.load_product_library()
    lib.deme_radix_sort_pairs_static.restype = C.c_int32
    lib.deme_radix_sort_pairs_static.argtypes = [C.c_void_p] * 4 + [C.c_uint32, C.c_int32, C.c_void_p]
    lib.deme_radix_sort_pairs_device.restype = C.c_int32
    lib.deme_radix_sort_pairs_device.argtypes = [C.c_void_p] * 4 + [C.c_uint32, C.c_int32, C.c_void_p, C.c_size_t,
                                                                     C.c_void_p]
    lib.deme_radix_sort_scratch_bytes.restype = C.c_size_t
    lib.deme_radix_sort_scratch_bytes.argtypes = [C.c_uint32]
    lib.deme_radix_sort_status.restype = C.c_int32
    lib.deme_radix_sort_status.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p, C.POINTER(C.c_uint32)]
    return lib


def _status(lib, scratch, n, st):
    word = C.c_uint32(0xDEADBEEF)
    rc = lib.deme_radix_sort_status(scratch, n, st, C.byref(word))
    return rc, word.value


def _inputs(n, bits, seed):
    rng = np.random.default_rng(seed)
    hi = min(1 << bits, 1 << 32)
    keys = rng.integers(0, min(hi, max(2, n // 3)), n, dtype=np.uint64).astype(np.uint32)  # many duplicates
    vals = rng.permutation(n).astype(np.uint32)
    dev = torch.device("cuda")
    return keys, vals, torch.from_numpy(keys.view(np.int32)).to(dev), torch.from_numpy(vals.view(np.int32)).to(dev)


def _sort_device(lib, kin, vin, n, bits, st):
    kout, vout = torch.empty_like(kin), torch.empty_like(vin)
    nb = lib.deme_radix_sort_scratch_bytes(n)
    scratch = torch.empty(nb, dtype=torch.uint8, device=kin.device)
    rc = lib.deme_radix_sort_pairs_device(kin.data_ptr(), vin.data_ptr(), kout.data_ptr(), vout.data_ptr(), n, bits,
                                          scratch.data_ptr(), nb, st)
    assert rc == 0
    # the sort's error word, in the last bytes of the caller's scratch, reports a completed sort
    assert _status(lib, scratch.data_ptr(), n, st) == (0, 0)
    return kout, vout


def _sort_static(lib, kin, vin, n, bits, st):
    kout = torch.full_like(kin, -1)
    vout = torch.full_like(vin, -1)
    rc = lib.deme_radix_sort_pairs_static(kin.data_ptr(), vin.data_ptr(), kout.data_ptr(), vout.data_ptr(), n, bits,
                                          st)
    assert rc == 0, rc
    assert _status(lib, None, n, st) == (0, 0)
    return kout, vout


def test_static_sort_matches_device_entry_on_two_calls_in_a_row():
    lib = _lib()
    st = torch.cuda.current_stream().cuda_stream
    # the second call is smaller and uses fewer passes: left-over scratch of the first must not leak into it
    for n, bits, seed in ((MAX_N, 32, 1), (100_003, 17, 2)):
        keys, vals, kin, vin = _inputs(n, bits, seed)
        ks, vs = _sort_static(lib, kin, vin, n, bits, st)
        kd, vd = _sort_device(lib, kin, vin, n, bits, st)
        torch.cuda.synchronize()
        assert torch.equal(ks, kd) and torch.equal(vs, vd), (n, bits)
        order = np.argsort(keys, kind="stable")
        np.testing.assert_array_equal(ks.cpu().numpy().view(np.uint32), keys[order])
        np.testing.assert_array_equal(vs.cpu().numpy().view(np.uint32), vals[order])


def test_static_sort_rejects_sizes_beyond_its_maximum():
    lib = _lib()
    st = torch.cuda.current_stream().cuda_stream
    _, _, kin, vin = _inputs(1024, 10, 3)
    kout = torch.full_like(kin, 7)
    vout = torch.full_like(vin, 7)
    # rejected before anything is launched, so the short buffers are never touched
    rc = lib.deme_radix_sort_pairs_static(kin.data_ptr(), vin.data_ptr(), kout.data_ptr(), vout.data_ptr(), MAX_N + 1,
                                          10, st)
    assert rc == DEME_ERR_TOO_LARGE
    assert lib.deme_status_string(rc) == b"DEME_ERR_TOO_LARGE"
    rc = lib.deme_radix_sort_pairs_static(kin.data_ptr(), vin.data_ptr(), kout.data_ptr(), vout.data_ptr(), 1024, 33,
                                          st)
    assert rc == DEME_ERR_INVALID
    torch.cuda.synchronize()
    assert bool((kout == 7).all()) and bool((vout == 7).all())


_FRESH = r"""
import sys, ctypes as C
import numpy as np, torch
sys.path.insert(0, sys.argv[1])
from deme_b200 import solver
lib = solver.load_product_library()
lib.deme_radix_sort_pairs_static.restype = C.c_int32
lib.deme_radix_sort_pairs_static.argtypes = [C.c_void_p] * 4 + [C.c_uint32, C.c_int32, C.c_void_p]
lib.deme_radix_sort_status.restype = C.c_int32
lib.deme_radix_sort_status.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p, C.POINTER(C.c_uint32)]
n = 50_000
rng = np.random.default_rng(5)
keys = rng.integers(0, 1 << 12, n, dtype=np.uint32)
vals = np.arange(n, dtype=np.uint32)
kin = torch.from_numpy(keys.view(np.int32)).cuda(); vin = torch.from_numpy(vals.view(np.int32)).cuda()
kout = torch.empty_like(kin); vout = torch.empty_like(vin)
st = torch.cuda.current_stream().cuda_stream
free = []
for _ in range(4):
    rc = lib.deme_radix_sort_pairs_static(kin.data_ptr(), vin.data_ptr(), kout.data_ptr(), vout.data_ptr(), n, 12, st)
    assert rc == 0, rc
    w = C.c_uint32(1)
    assert lib.deme_radix_sort_status(None, n, st, C.byref(w)) == 0 and w.value == 0
    torch.cuda.synchronize()
    o = np.argsort(keys, kind="stable")
    assert (kout.cpu().numpy().view(np.uint32) == keys[o]).all() and (vout.cpu().numpy().view(np.uint32) == vals[o]).all()
    free.append(torch.cuda.mem_get_info()[0])
# after the first call (which loads the library's device code), further calls take no device memory
assert len(set(free[1:])) == 1, free
print("ok")
"""


def test_static_sort_first_call_in_a_fresh_process():
    pkg = os.path.join(ROOT, "dem-engine-sbel_b200")
    r = subprocess.run([sys.executable, "-c", _FRESH, pkg], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), r.stdout + r.stderr
