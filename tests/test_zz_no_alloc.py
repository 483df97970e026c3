"""The Hartree solve that allocates nothing, checked against the ordinary one.

rs_hartree_cg_noalloc exists for callers that cannot allocate device memory
when they solve (their memory is already handed to a pool or a caching
allocator).  It keeps its work vectors in a fixed array inside the library,
shared by every call.  Two calls in a row, the second warm-started from the
first with a new density, must give exactly what rs_hartree_cg gives: the
array's leftover contents from the first call must not leak into the second.
This file is collected last so that a run stopping at the first failure has
already run every other test."""
import ctypes as C

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _solve(lib, name, shape, xmax, rho, vh0):
    nx, ny, nz = shape
    d_rho = torch.tensor(rho, dtype=torch.float64, device="cuda")
    d_vh = torch.tensor(vh0, dtype=torch.float64, device="cuda")
    it, dp = C.c_int(0), C.c_double(0.0)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    lib.call(name, nx, ny, nz, 4, xmax[0], xmax[1], xmax[2], 1e-12, 1, 800, 801,
             C.c_void_p(d_rho.data_ptr()), C.c_void_p(d_vh.data_ptr()), C.byref(it),
             C.byref(dp), stream)
    torch.cuda.synchronize()
    return d_vh.cpu().numpy(), it.value, dp.value


def test_noalloc_hartree_matches_allocating_entry_point(built_lib, cuda):
    from rspacedist_b200 import lib
    shape = (48, 40, 36)
    h = (0.31, 0.33, 0.29)
    xmax = tuple(n * hh / 2 for n, hh in zip(shape, h))
    rng = np.random.default_rng(21)
    N = int(np.prod(shape))
    vh = np.zeros(N)
    for call in range(2):
        rho = rng.standard_normal(N)
        ref, it_ref, dp_ref = _solve(lib, "rs_hartree_cg", shape, xmax, rho, vh)
        got, it, dp = _solve(lib, "rs_hartree_cg_noalloc", shape, xmax, rho, vh)
        assert it == it_ref and dp == dp_ref, (call, it, it_ref, dp, dp_ref)
        assert np.array_equal(got, ref), call
        vh = got  # warm start of the second call, as scf_hartree does

    # grids beyond the fixed array are refused with a message, not run
    rc = built_lib.rs_hartree_cg_noalloc(72, 64, 64, 4, 10.0, 10.0, 10.0, 1e-12, 1, 800, 801,
                                         None, None, None, None, None)
    assert rc == -1
    assert "262144" in lib.last_error()
