"""Many small cells in one persistent launch (rs_hpsi_batch_*): the setting of
32 independent Si8/C8 cells of uneven grids.  Each cell's H psi equals its
single-cell result: bit for bit where the single-cell call takes the
per-point gather path, within FP32 rounding where it takes the z-march
stencil; the CUDA-graph replay equals the direct launch."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def test_batch_equals_single_cell(cuda, built_lib):
    from rspacedist_b200 import kukan as K, system as S
    cells = S.small_cell_set(6)
    geoms = [K.Geometry(c) for c in cells]
    nb = [20] * len(cells)
    veff = [torch.tensor(S.smooth_veff(c, i), dtype=torch.float32, device="cuda")
            for i, c in enumerate(cells)]
    dij = [torch.tensor(c.dij, dtype=torch.float64, device="cuda") for c in cells]
    psi = [torch.tensor(S.random_bands(c, 20, i), dtype=torch.float32, device="cuda")
           for i, c in enumerate(cells)]
    rp = [K.nonlocaloperation_01(g, p) for g, p in zip(geoms, psi)]
    single = [K.hpsi(g, v, d, r, p) for g, v, d, r, p in zip(geoms, veff, dij, rp, psi)]
    out = [torch.full_like(p, float("nan")) for p in psi]
    plan = K.HpsiBatch(geoms, nb)
    plan.set(veff, dij, rp, psi, out)
    plan.run()
    torch.cuda.synchronize()
    assert plan.info()["threads_per_cta"] in (64, 128, 256)
    for c, s, o in zip(cells, single, out):
        zmarch = c.shape[0] % 4 == 0 and c.shape[1] % 2 == 0 and c.nprjmx % 4 == 0
        if zmarch:
            tol = 2e-5 * float(s.abs().max())
            assert float((s - o).abs().max()) <= tol
        else:
            assert torch.equal(s, o), c.shape
    # graph capture and replay on a side stream give the same bits
    st = torch.cuda.Stream()
    ref = [o.clone() for o in out]
    with torch.cuda.stream(st):
        for o in out:
            o.fill_(float("nan"))
        plan.run(graph=True)
        for o in out:
            o.fill_(float("nan"))
        plan.run(graph=True)
    st.synchronize()
    for r, o in zip(ref, out):
        assert torch.equal(r, o)
    plan.close()


def test_batch_shapes_same_bits(cuda, built_lib):
    """Every launch shape (threads per CTA, bands per work item, CTAs per SM)
    gives the same bits, on cells of uneven grids and band counts."""
    from rspacedist_b200 import kukan as K, system as S
    cells = S.small_cell_set(8)
    geoms = [K.Geometry(c) for c in cells]
    nb = [20, 7, 20, 13, 20, 20, 5, 20]
    veff = [torch.tensor(S.smooth_veff(c, i), dtype=torch.float32, device="cuda")
            for i, c in enumerate(cells)]
    dij = [torch.tensor(c.dij, dtype=torch.float64, device="cuda") for c in cells]
    psi = [torch.tensor(S.random_bands(c, n, i), dtype=torch.float32, device="cuda")
           for i, (c, n) in enumerate(zip(cells, nb))]
    rp = [K.nonlocaloperation_01(g, p) for g, p in zip(geoms, psi)]
    out = [torch.full_like(p, float("nan")) for p in psi]
    plan = K.HpsiBatch(geoms, nb)
    plan.set(veff, dij, rp, psi, out)
    plan.set_shape(128, 4, 8)
    plan.run()
    torch.cuda.synchronize()
    ref = [o.clone() for o in out]
    for shape in [(64, 1, 16), (256, 8, 4), (128, 2, 2)]:
        for o in out:
            o.fill_(float("nan"))
        plan.set_shape(*shape)
        plan.run()
        torch.cuda.synchronize()
        assert plan.info()["threads_per_cta"] == shape[0]
        for r, o in zip(ref, out):
            assert torch.equal(r, o), shape
    plan.close()
