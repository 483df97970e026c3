"""The C-ABI library builds for sm_100a, loads, and exports every entry point
declared in include/rspace_b200.h; host-side logic runs without a GPU."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(ROOT, "include", "rspace_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(rs_\w+)\s*\(", src, flags=re.M)))


def test_header_declares_entry_points():
    names = declared_functions()
    assert "rs_hpsi_f32" in names and "rs_hartree_cg" in names and len(names) >= 20


def test_library_exports_every_declared_symbol(built_lib):
    from rspacedist_b200 import lib
    out = subprocess.run(["nm", "-D", "--defined-only", lib.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = set(line.split()[-1] for line in out.splitlines() if line.strip())
    missing = [n for n in declared_functions() if n not in exported]
    assert not missing, missing
    for n in declared_functions():
        assert hasattr(built_lib, n)


def test_ctypes_signatures_cover_header(built_lib):
    from rspacedist_b200 import lib
    missing = [n for n in declared_functions()
               if n not in lib.SIGNATURES and n not in lib.RESTYPES and n != "rs_geom_entries"]
    assert not missing, missing


def test_version_and_error_plumbing(built_lib):
    from rspacedist_b200 import lib
    assert b"sm_100a" in built_lib.rs_version()
    # a host-side argument error sets the message without touching a GPU
    rc = built_lib.rs_sphere_lists(0, None, None, None, None, 0, 0, 0, 1.0, 1.0, 1.0, 1, 1, 1, 4,
                                   0, None, None, None, None, None, None, None, None)
    assert rc == -1
    assert "bad dimensions" in lib.last_error()


@pytest.mark.parametrize("cellkind", ["si8", "c8"])
def test_sphere_lists_bit_exact_vs_oracle(oracle, built_lib, cellkind):
    import conftest
    cell = conftest.make_si8(32, 0.05, 4) if cellkind == "si8" else conftest.make_c8(24)
    st, d = oracle.sphere_lists(cell.atoms, cell.ds["rcut"] * 1.05, cell.nmax, cell.h,
                                cell.npmax, 4, cell.num_list)
    assert st == 0
    assert np.array_equal(d["natinf"], cell.natinf)
    for k in ("natx", "naty", "natz"):
        assert np.array_equal(d[k], cell.natxyz["xyz".index(k[-1])])
    A, L = cell.natom, cell.num_list
    for a in range(A):
        n = cell.natinf[a]
        assert np.array_equal(d["lst"][a * L:a * L + n], cell.lst[a * L:a * L + n])
        for k, lk in zip(("lstx", "lsty", "lstz"), cell.lstxyz):
            assert np.array_equal(d[k][a * L:a * L + n], lk[a * L:a * L + n])


def test_sphere_lists_capacity_error(built_lib):
    from rspacedist_b200 import lib, system as S
    ds = S.load_dataset("si_paw")
    cell = S.Cell(shape=(32, 32, 32), h=(10.26 / 32,) * 3, xmax=(5.13,) * 3, nmax=(16,) * 3,
                  atoms=np.zeros((1, 3)), ds=ds)
    npm, nl = S.list_dims(cell)
    out = [np.zeros(1, np.int32) for _ in range(4)] + [np.zeros(100, np.int32) for _ in range(4)]
    dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    ip = lambda a: a.ctypes.data_as(C.POINTER(C.c_int))
    z = np.zeros(1)
    rc = np.array([ds["rcut"] * 1.05])
    st = built_lib.rs_sphere_lists(1, dp(z), dp(z), dp(z), dp(rc), 16, 16, 16, cell.h[0],
                                   cell.h[1], cell.h[2], npm[0], npm[1], npm[2], 4, 100,
                                   *[ip(a) for a in out])
    assert st == -1 and "num_list is too small" in lib.last_error()


def test_state_handle_reports_errors_without_a_device(built_lib):
    """Without a GPU, rs_create fails with a status and a message instead of
    crashing, and rs_destroy accepts a null handle."""
    import ctypes as C
    import pytest
    import torch
    from rspacedist_b200 import lib
    if torch.cuda.is_available():
        pytest.skip("needs a machine without a CUDA device")
    L = lib.load()
    h = C.c_void_p()
    rc = L.rs_create(C.byref(h), 32, 16, 16, 16, 4, 0.3, 0.3, 0.3, 4, None)
    assert rc != 0 and not h.value
    assert lib.last_error()
    assert L.rs_create(C.byref(h), 16, 16, 16, 16, 4, 0.3, 0.3, 0.3, 4, None) != 0
    assert "precision" in lib.last_error()
    assert L.rs_destroy(None) == 0
