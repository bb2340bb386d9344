"""Allocation-free global residual against the context's own global residual.

``ccfd_global_residual_noalloc`` (C ABI) sums area * u_t^2 of a caller-held
device residual field with a static scratch array; ``ccfd_global_residual``
sums the per-tile partials the stage kernel wrote in the same residual
evaluation.  Both are globalResidual of the reference (src/analyze.c:521-539)
and differ only in summation order, hence the relative tolerance below.
The file is named to be collected last so the entry point also runs after
every other GPU test has used the device in the same process.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np
import pytest

RTOL = 1e-12


def _call(lib, ut_dev, area_dev, n, total_area_q, res_dev, stream):
    return lib.ccfd_global_residual_noalloc(
        C.c_void_p(ut_dev.data_ptr()), C.c_void_p(area_dev.data_ptr()), C.c_long(n),
        C.c_double(total_area_q), C.c_void_p(res_dev.data_ptr()), C.c_void_p(stream))


@pytest.mark.gpu
def test_noalloc_global_residual_matches(tmp_path):
    import torch

    import ccfd_b200 as cc
    from ccfd_b200 import _native as N
    from ccfd_b200 import meshgen

    cc.set_device(0)
    torch.cuda.set_device(0)
    meshgen.dmr_mesh(200, 50).write_gmsh(os.path.join(tmp_path, "dmr.msh"))
    case = cc.CaseData.from_text(meshgen.dmr_ini("dmr"), str(tmp_path))
    mesh = case.mesh()
    n = mesh["n_cells"]
    assert n % 256 != 0 or n > 256
    area = torch.from_numpy(np.ascontiguousarray(mesh["cell_geo"][:, 0])).cuda()
    res_dev = torch.full((4,), np.nan, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    s = cc.Solver(case, reorder=True)
    try:
        # two calls in a row on two different residual fields
        for time in (0.0, 0.05):
            ut = s.fv_time_derivative(time)
            want = s.global_residual()
            ut_dev = torch.from_numpy(np.ascontiguousarray(ut)).cuda()
            torch.cuda.synchronize()
            st = _call(N.lib, ut_dev, area, n, mesh["total_area_q"], res_dev, stream)
            assert st == 0, N.lib.ccfd_strerror(st)
            torch.cuda.synchronize()
            got = res_dev.cpu().numpy()
            assert np.all(np.isfinite(got))
            np.testing.assert_allclose(got, want, rtol=RTOL, atol=0.0)
    finally:
        s.close()


@pytest.mark.gpu
@pytest.mark.parametrize("n", [300_001, 1 << 20])
def test_noalloc_large_fields_match_float64_sum(n):
    """Synthetic fields well above 65,536 cells (the final pass then walks
    many partials per thread) and at the scratch's full size, two calls in a
    row, against a float64 sum of the same terms."""
    import torch

    from ccfd_b200 import _native as N

    assert n <= N.NOALLOC_MAX_CELLS
    torch.cuda.set_device(0)
    stream = torch.cuda.current_stream().cuda_stream
    res_dev = torch.full((4,), np.nan, dtype=torch.float64, device="cuda")
    for seed in (1, 2):
        rng = np.random.default_rng(seed)
        ut = rng.standard_normal((n, 4)) * np.array([1.0, 10.0, 0.1, 100.0])
        area = rng.uniform(0.5, 2.0, n) * 1e-4
        taq = 1.0 / area.sum()
        want = np.sqrt((area[:, None] * ut * ut).sum(axis=0) * taq)
        ut_dev = torch.from_numpy(ut).cuda()
        area_dev = torch.from_numpy(area).cuda()
        torch.cuda.synchronize()
        st = _call(N.lib, ut_dev, area_dev, n, taq, res_dev, stream)
        assert st == 0, N.lib.ccfd_strerror(st)
        torch.cuda.synchronize()
        np.testing.assert_allclose(res_dev.cpu().numpy(), want, rtol=RTOL, atol=0.0)


@pytest.mark.gpu
def test_noalloc_rejects_sizes_beyond_scratch():
    import torch

    from ccfd_b200 import _native as N

    torch.cuda.set_device(0)
    buf = torch.zeros(8, dtype=torch.float64, device="cuda")
    too_many = int(N.NOALLOC_MAX_CELLS) + 1
    for n in (0, -1, too_many):
        st = _call(N.lib, buf, buf, n, 1.0, buf, 0)
        assert st == N.CCFD_ERR_ARG
