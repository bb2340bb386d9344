"""Mixed precision (``precision = 1``): FP32 reconstruction and face fluxes,
FP64 per-cell flux sums, state and update.

The mixed path is not expected to equal the reference bit for bit; each test
states its error against the FP64 reference outputs (committed fixtures) and
bounds it.  Tolerances: residual evaluations within MIX_RES_TOL of max|R| per
variable; explicit runs within MIX_RUN_TOL in L1 and L-infinity of the state.
"""
import tempfile

import numpy as np
import pytest

import ccfd_b200 as cc
from tests.golden import cases as CASES
from tests.helpers import l1_linf, rel_max_err

pytestmark = pytest.mark.gpu

MIX_RES_TOL = 2e-5
MIX_RUN_TOL = 5e-6


def _mixed(ini: str) -> str:
    if "precision = 0" in ini:
        return ini.replace("precision = 0", "precision = 1")
    return ini + "\nprecision = 1\n"


@pytest.mark.parametrize("key", sorted(CASES.residual_cases()))
def test_mixed_residual_error_vs_reference(ref_small, key):
    spec = dict(CASES.residual_cases()[key])
    spec["ini"] = _mixed(spec["ini"])
    with tempfile.TemporaryDirectory() as tmp:
        case, _, _ = CASES.load_case(spec, tmp)
        assert case.c.params.precision == 1
        prim = ref_small[f"{key}/prim"].reshape(-1, 4)
        s = cc.Solver(case, reorder=True)
        s.set_state(prim)
        ut = s.fv_time_derivative(spec["time"])
        s.close()
    err = rel_max_err(ut, ref_small[f"{key}/u_t"])
    print(f"{key}: mixed residual rel err {err:.2e}")
    assert err <= MIX_RES_TOL
    assert err > 0.0  # the FP32 path really ran


@pytest.mark.parametrize("key", ["dmr_hllc_vk_run", "dmr_roe_bj_run", "zoo_euler_run"])
def test_mixed_run_error_vs_reference(ref_small, key):
    spec = dict(CASES.run_cases()[key])
    spec["ini"] = _mixed(spec["ini"])
    with tempfile.TemporaryDirectory() as tmp:
        case, _, _ = CASES.load_case(spec, tmp)
        s = cc.Solver(case, reorder=True)
        rep = s.run(spec["steps"])
        prim = s.get_state()
        s.close()
    info = ref_small[f"{key}/info"]
    want = ref_small[f"{key}/pvar"].reshape(-1, 4)
    # the time steps follow the (slightly different) mixed-precision state;
    # both runs end at tEnd
    assert abs(rep["iterations"] - int(info[1])) <= 1
    assert abs(rep["t"] - info[0]) <= 1e-14
    scale = np.abs(want).max(axis=0)
    l1, linf = l1_linf(prim / scale, want / scale)
    print(f"{key}: mixed run L1 {l1:.2e} Linf {linf:.2e} after {rep['iterations']} steps")
    assert l1 <= MIX_RUN_TOL and linf <= MIX_RUN_TOL


# Implicit steps in mixed precision: the preconditioner is built from
# FP32-flux residuals, so GMRES follows its own path and every step is
# solved only to the Newton tolerance; after the few unconverged steps of
# these cases the state is 5.8e-6 (Euler, preconditioned), 9.9e-7
# (Navier-Stokes) and 5.9e-9 (no preconditioner) from the FP64 reference.
# Converged, the mixed steady state is the FP64 one within 1e-6
# (tests/test_gpu_implicit_oracle.py).
MIX_IMP_TOL = 2e-5


@pytest.mark.parametrize("key", ["naca_euler_imp_pc", "naca_euler_imp_nopc", "naca_ns_imp_pc"])
def test_mixed_implicit_error_vs_reference(ref_small, key):
    # FP32 Krylov basis, LU-SGS blocks and preconditioner columns, FP64
    # Newton / matrix-vector residuals and Newton update:
    # the iterates follow a different GMRES path, so the state after a few
    # steps differs from the FP64 reference by the inexact-Newton tolerance,
    # not by rounding
    spec = dict(CASES.implicit_cases()[key])
    spec["ini"] = _mixed(spec["ini"])
    with tempfile.TemporaryDirectory() as tmp:
        case, _, _ = CASES.load_case(spec, tmp)
        s = cc.Solver(case, reorder=True)
        rep = s.run(spec["steps"])
        prim = s.get_state()
        s.close()
    ref = ref_small[f"{key}/pvar"].reshape(-1, 4)
    clcd = ref_small[f"{key}/clcd"]
    err = float((np.abs(prim - ref).max(axis=0) / np.abs(ref).max(axis=0)).max())
    print(f"{key}: mixed implicit state rel err {err:.2e}, CL err {abs(rep['cl'] - clcd[0]):.2e}, "
          f"CD err {abs(rep['cd'] - clcd[1]):.2e}, newton {rep['newton_iterations']}, "
          f"gmres {rep['gmres_iterations']}")
    assert rep["status"] == 0
    assert err <= MIX_IMP_TOL
    assert abs(rep["cl"] - clcd[0]) <= MIX_IMP_TOL and abs(rep["cd"] - clcd[1]) <= MIX_IMP_TOL
