"""The restated implicit path of the oracle (block-sparse buildMatrix /
calcDinv / LUSGS, implicitTimeStep with GMRES_M) pinned to the compiled
reference, whose dense Jacobian ((4N)^2 doubles, src/linearSolver.c:99) is
affordable on these small meshes only.

* buildMatrix: every diagonal and face-neighbour entry equal bit for bit
  (the same residual arithmetic per column); the state after the column
  evaluations (perturbed and restored in place) equal bit for bit.
* calcDinv / LUSGS: <= 1e-12 relative (the oracle's own 4x4 inverse).
* implicit runs (with and without LU-SGS, Euler and Navier-Stokes, the
  relative stop): the same step, Newton and GMRES counts, state and lift /
  drag within 1e-8; bit for bit without LU-SGS.  Under the
  switched-evolution-relaxation CFL ramp the time steps follow the
  residuals (1e-6 on dt and on the transient state, 1e-8 on lift / drag).
"""
import os
import tempfile

import numpy as np
import pytest

from ccfd_b200 import meshgen
from oracle import refdump, restated
from tests.golden import cases as CASES

needs_ref = pytest.mark.skipif(not refdump.have_ref() or not refdump.have_ref("navierstokes"),
                               reason="compiled reference not built")

RUN_TOL = 1e-8


def _rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


JAC_CASES = ["naca_euler_imp_pc", "naca_ns_imp_pc", "sine_periodic_imp"]


@needs_ref
@pytest.mark.parametrize("key", JAC_CASES)
def test_restated_build_matrix_equals_reference_dense_jacobian(key):
    spec = CASES.implicit_cases()[key]
    with tempfile.TemporaryDirectory() as tmp:
        case, ini, files = CASES.load_case(spec, tmp)
        if "precond = F" in ini:
            pytest.skip("no preconditioner")
        n = case.n_cells
        rng = np.random.default_rng(7)
        prim = case.prim0() * (1.0 + 0.05 * rng.uniform(-1.0, 1.0, (n, 4)))
        vec = rng.standard_normal((n, 4))
        d = refdump.run_ref(ini, "jacobian", 0.0, 0.01, eqn=spec["eqn"], state=prim, vector=vec, files=files)
    rxk = d["r_xk_used"].reshape(n, 4)
    after, D, Di, O = restated.build_matrix(case, prim, rxk, 0.0, 0.01, in_place=True)
    assert np.array_equal(after, d["pvar_after"].reshape(n, 4))
    assert np.array_equal(D, d["jac_d"].reshape(n, 4, 4))
    assert np.array_equal(O, d["jac_off"].reshape(-1, 4, 4))
    assert _rel(Di, d["jac_dinv"].reshape(n, 4, 4)) <= 1e-12
    # D^-1 D = I
    assert np.abs(np.einsum("nij,njk->nik", Di, D) - np.eye(4)).max() <= 1e-10
    x = restated.lusgs(case, Di, O, vec)
    assert _rel(x, d["lusgs"].reshape(n, 4)) <= 1e-12
    # restoring the saved value instead of subtracting the step again gives
    # the same blocks here ((p + e) - e rounds back to p unless it ties)
    _, D2, _, O2 = restated.build_matrix(case, prim, rxk, 0.0, 0.01, in_place=False)
    assert np.array_equal(D2, D) and np.array_equal(O2, O)


@needs_ref
@pytest.mark.parametrize("key", ["naca_euler_imp_pc", "naca_euler_imp_nopc", "naca_ns_imp_pc",
                                 "naca_euler_imp_rel", "sine_periodic_imp"])
def test_restated_implicit_run_matches_reference(key):
    spec = CASES.implicit_cases()[key]
    with tempfile.TemporaryDirectory() as tmp:
        case, ini, files = CASES.load_case(spec, tmp)
        d = refdump.run_ref(ini, "coef", spec["steps"], eqn=spec["eqn"], files=files,
                            rel_abort=spec.get("rel_abort"))
    prim, info, hist = restated.run_implicit(case, spec["steps"])
    assert info["status"] == 0
    ri = d["run_info"]
    assert info["iterations"] == int(ri[1])
    assert info["converged"] == bool(ri[4])
    assert info["newton_iterations"] == int(ri[5])
    assert info["gmres_iterations"] == int(ri[6])
    ref = d["pvar"].reshape(-1, 4)
    assert (np.abs(prim - ref).max(axis=0) / np.abs(ref).max(axis=0)).max() <= RUN_TOL
    if "clcd" in d:
        assert abs(info["cl"] - d["clcd"][0]) <= RUN_TOL and abs(info["cd"] - d["clcd"][1]) <= RUN_TOL
    if "precond = F" in ini:  # no 4x4 inverse involved: the run is the reference's, bit for bit
        assert np.array_equal(prim, ref)


def _ser_case(ns: bool, cfl: float, max_iter: int, rel: float = 1e-8):
    return {"mesh": ("naca", 32, 12) if ns else ("naca", 32, 12, 101),
            "ini": meshgen.airfoil_ini("naca", mach=0.5, alpha=2.0, navier_stokes=ns, reynolds=500.0, flux=2,
                                       implicit=True, precond=True, n_kdim=30, cfl=cfl, max_iter=max_iter,
                                       rel_res=rel),
            "eqn": "navierstokes" if ns else "euler"}


@needs_ref
def test_restated_ser_cfl_ramp_matches_reference():
    # 12 steps of the ramp (CFL 20 -> ~400, capped at 300) around the
    # reference's own implicitTimeStep
    spec = _ser_case(False, 20.0, 12)
    with tempfile.TemporaryDirectory() as tmp:
        case, ini, files = CASES.load_case(spec, tmp)
        d = refdump.run_ref(ini, "coef", 12, eqn="euler", files=files, rel_abort=1e-8, ser_cfl_max=300.0)
    prim, info, hist = restated.run_implicit(case, 12, ser_cfl_max=300.0)
    assert info["status"] == 0
    ri = d["run_info"]
    assert info["iterations"] == int(ri[1]) == 12
    assert info["newton_iterations"] == int(ri[5])
    assert info["gmres_iterations"] == int(ri[6])
    # the ramped time steps follow the residuals, whose rounding differs
    # (4x4 inverse) at the 1e-9 level and grows relative to the residual as
    # it falls; the transient state follows the time steps (a converged
    # steady state does not depend on them)
    h = d["history"].reshape(-1, 8)
    np.testing.assert_allclose(hist[:, 1], h[:, 1], rtol=1e-6)
    assert hist[-1, 1] > 5.0 * hist[0, 1]
    ref = d["pvar"].reshape(-1, 4)
    assert (np.abs(prim - ref).max(axis=0) / np.abs(ref).max(axis=0)).max() <= 1e-6
    assert abs(info["cl"] - d["clcd"][0]) <= RUN_TOL and abs(info["cd"] - d["clcd"][1]) <= RUN_TOL


def test_restated_ser_reaches_steady_state():
    # the same airfoil converged to a relative residual of 1e-8, which the
    # reference's fixed CFL does not reach in hundreds of steps
    spec = _ser_case(False, 20.0, 1500)
    with tempfile.TemporaryDirectory() as tmp:
        case, _, _ = CASES.load_case(spec, tmp)
    prim, info, hist = restated.run_implicit(case, 0, ser_cfl_max=300.0)
    assert info["status"] == 0 and info["converged"]
    assert hist[-1, 2] <= 1e-8 * hist[0, 2]
