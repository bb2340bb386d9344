"""Autotuner of the stage kernel's launch shape (ccfd_autotune): it must
pick a valid candidate, leave the context uploaded with the given state, and
— since tiling, cell order and CTA size change only the storage and launch
shape — give residuals and states bit-identical to the default shape (the
global residual, a sum of per-tile partials, to the last bits)."""
import tempfile

import numpy as np
import pytest

import ccfd_b200 as cc
from tests.golden import cases as CASES

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("key", ["dmr_f05_vk", "zoo_ns_vk", "dmr_f02_bj"])
def test_autotuned_shape_gives_identical_results(ref_small, key):
    spec = CASES.residual_cases()[key]
    with tempfile.TemporaryDirectory() as tmp:
        case, _, _ = CASES.load_case(spec, tmp)
    prim = ref_small[f"{key}/prim"].reshape(-1, 4)
    base = cc.Solver(case)
    base.set_state(prim)
    ut0 = base.fv_time_derivative(spec["time"])
    tuned = cc.Solver(case)
    info = tuned.autotune(prim)
    assert info["tile_cells"] in (128, 192, 256, 320, 384)
    assert info["threads"] in (256, 320, 384)
    assert info["ms_per_residual"] > 0.0
    assert np.array_equal(tuned.get_state(), prim)
    ut1 = tuned.fv_time_derivative(spec["time"])
    assert np.array_equal(ut0, ut1)
    rep0, rep1 = base.run(7), tuned.run(7)
    assert np.array_equal(base.get_state(), tuned.get_state())
    assert rep0["t"] == rep1["t"]
    # the global residual sums per-tile partials, so its last bits follow
    # the tiling (as the reference's OpenMP reduction follows the threads)
    np.testing.assert_allclose(rep0["residual"], rep1["residual"], rtol=1e-13, atol=0.0)
    base.close()
    tuned.close()


@pytest.mark.parametrize("threads", [256, 320])
def test_smaller_cta_gives_identical_results(ref_small, threads, monkeypatch):
    # every CTA size within the launch bounds: same residual and run
    spec = CASES.residual_cases()["dmr_f05_vk"]
    with tempfile.TemporaryDirectory() as tmp:
        case, _, _ = CASES.load_case(spec, tmp)
    prim = ref_small["dmr_f05_vk/prim"].reshape(-1, 4)
    base = cc.Solver(case)
    monkeypatch.setenv("CCFD_STAGE_THREADS", str(threads))
    other = cc.Solver(case)
    try:
        base.set_state(prim)
        other.set_state(prim)
        assert np.array_equal(base.fv_time_derivative(spec["time"]), other.fv_time_derivative(spec["time"]))
        base.run(5)
        other.run(5)
        assert np.array_equal(base.get_state(), other.get_state())
    finally:
        base.close()
        other.close()
