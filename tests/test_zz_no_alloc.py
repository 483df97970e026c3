"""The Hartree solve that allocates nothing, checked against the ordinary one.

rs_hartree_cg_noalloc exists for callers that cannot allocate device memory
when they solve (their memory is already handed to a pool or a caching
allocator).  It keeps its work vectors in a fixed array inside the library,
shared by every call.  Two calls in a row, the second warm-started from the
first with a new density, must give exactly what rs_hartree_cg gives: the
array's leftover contents from the first call must not leak into the second.
The check runs on the legacy stream and on a stream of its own (where
rs_hartree_cg replays a CUDA graph and the no-allocation call does not), and
on a grid of exactly the array's limit, so that the last words of the array
(the partial sums and the CG scalars) are used.  This file is collected last
so that a run stopping at the first failure has already run every other
test."""
import ctypes as C

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _solve(lib, name, shape, xmax, rho, vh0, stream):
    nx, ny, nz = shape
    with torch.cuda.stream(stream):
        d_rho = torch.tensor(rho, dtype=torch.float64, device="cuda")
        d_vh = torch.tensor(vh0, dtype=torch.float64, device="cuda")
        it, dp = C.c_int(0), C.c_double(0.0)
        lib.call(name, nx, ny, nz, 4, xmax[0], xmax[1], xmax[2], 1e-12, 1, 800, 801,
                 C.c_void_p(d_rho.data_ptr()), C.c_void_p(d_vh.data_ptr()), C.byref(it),
                 C.byref(dp), C.c_void_p(stream.cuda_stream))
    torch.cuda.synchronize()
    return d_vh.cpu().numpy(), it.value, dp.value


@pytest.mark.parametrize("shape,h,side", [
    ((48, 40, 36), (0.31, 0.33, 0.29), False),
    ((48, 40, 36), (0.31, 0.33, 0.29), True),
    ((64, 64, 64), (0.32, 0.32, 0.32), True),
])
def test_noalloc_hartree_matches_allocating_entry_point(built_lib, cuda, shape, h, side):
    from rspacedist_b200 import lib
    stream = torch.cuda.Stream() if side else torch.cuda.current_stream()
    xmax = tuple(n * hh / 2 for n, hh in zip(shape, h))
    rng = np.random.default_rng(21)
    N = int(np.prod(shape))
    vh = np.zeros(N)
    for call in range(2):
        rho = rng.standard_normal(N)
        ref, it_ref, dp_ref = _solve(lib, "rs_hartree_cg", shape, xmax, rho, vh, stream)
        got, it, dp = _solve(lib, "rs_hartree_cg_noalloc", shape, xmax, rho, vh, stream)
        assert it == it_ref and dp == dp_ref, (call, it, it_ref, dp, dp_ref)
        assert np.array_equal(got, ref), call
        vh = got  # warm start of the second call, as scf_hartree does


def test_noalloc_hartree_limits(built_lib, cuda):
    from rspacedist_b200 import lib
    # grids beyond the fixed array are refused with a message, not run
    rc = built_lib.rs_hartree_cg_noalloc(72, 64, 64, 4, 10.0, 10.0, 10.0, 1e-12, 1, 800, 801,
                                         None, None, None, None, None)
    assert rc == -1
    assert "262144" in lib.last_error()
    # a solve stopped by the iteration limit leaves the same diagnostic as
    # rs_hartree_cg does
    shape, xmax = (24, 24, 24), (4.0, 4.0, 4.0)
    rho = np.random.default_rng(5).standard_normal(24 ** 3)
    d_rho = torch.tensor(rho, dtype=torch.float64, device="cuda")
    for name in ("rs_hartree_cg", "rs_hartree_cg_noalloc"):
        d_vh = torch.zeros_like(d_rho)
        it, dp = C.c_int(0), C.c_double(0.0)
        lib.call(name, *shape, 4, *xmax, 1e-12, 1, 3, 801, C.c_void_p(d_rho.data_ptr()),
                 C.c_void_p(d_vh.data_ptr()), C.byref(it), C.byref(dp), None)
        torch.cuda.synchronize()
        assert it.value >= 3 and dp.value > 1e-12
        assert lib.last_error() == name + ": ncgmax reached"
