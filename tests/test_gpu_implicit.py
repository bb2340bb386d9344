"""Implicit path (Newton / matrix-free GMRES / LU-SGS) against the compiled
reference on a small NACA 0012 O-grid, where the reference's dense Jacobian
is affordable.  Tolerance: 1e-8 relative on the state and on CL / CD after
the same number of implicit steps (the Krylov, Jacobian and 4x4-inverse
arithmetic is reordered, so the iterates agree to rounding, not bitwise)."""
import os
import tempfile

import numpy as np
import pytest

import ccfd_b200 as cc
from ccfd_b200 import meshgen
from tests.golden import cases as CASES

pytestmark = pytest.mark.gpu

TOL = 1e-8


@pytest.mark.parametrize("key", sorted(CASES.implicit_cases()))
def test_implicit_steps_match_reference(ref_small, key):
    spec = CASES.implicit_cases()[key]
    with tempfile.TemporaryDirectory() as tmp:
        case, _, _ = CASES.load_case(spec, tmp)
        s = cc.Solver(case, reorder=True)
        rep = s.run(spec["steps"])
        prim = s.get_state()
        s.close()
    ref = ref_small[f"{key}/pvar"].reshape(-1, 4)
    info = ref_small[f"{key}/info"]
    assert rep["iterations"] == int(info[1])
    assert bool(rep["converged"]) == bool(info[4])  # relative stop: both at the same step
    assert rep["newton_iterations"] == int(info[5])
    assert rep["gmres_iterations"] == int(info[6])
    err = np.abs(prim - ref).max(axis=0) / np.abs(ref).max(axis=0)
    assert err.max() <= TOL, err
    if f"{key}/clcd" in ref_small:
        clcd = ref_small[f"{key}/clcd"]
        assert abs(rep["cl"] - clcd[0]) <= TOL and abs(rep["cd"] - clcd[1]) <= TOL
    hist = ref_small[f"{key}/history"].reshape(-1, 8)
    np.testing.assert_allclose(rep["residual"][:4], hist[-1, 2:6], rtol=1e-6)


@pytest.mark.parametrize("key", ["naca_euler_imp_pc", "naca_ns_imp_pc"])
def test_wall_pressure_coefficient_matches_reference_files(ref_small, key, tmp_path):
    # the reference writes CP along the wing with "%15.7f" (calcCoef,
    # src/analyze.c:302-367); the state agrees to 1e-8, so the files agree to
    # their printed precision
    spec = CASES.implicit_cases()[key]
    with tempfile.TemporaryDirectory() as tmp:
        case, _, _ = CASES.load_case(spec, tmp)
    s = cc.Solver(case, reorder=True)
    s.run(spec["steps"])
    x, y, cp, npres = s.wall_cp()
    base = str(tmp_path / "naca")
    s.write_cp(base)
    s.close()
    for side, lo, hi in (("pressure", 0, npres), ("suction", npres, len(cp))):
        want = ref_small[f"{key}/cp_{side}"].reshape(-1, 4)
        assert hi - lo == len(want)
        np.testing.assert_allclose(x[lo:hi], want[:, 0], atol=1e-7, rtol=0)
        np.testing.assert_allclose(y[lo:hi], want[:, 1], atol=1e-7, rtol=0)
        np.testing.assert_allclose(cp[lo:hi], want[:, 3], atol=2e-7, rtol=0)
        got = np.genfromtxt(f"{base}_CP_{side}Side.csv", delimiter=",", skip_header=1).reshape(-1, 4)
        np.testing.assert_allclose(got, want, atol=2e-7, rtol=0)


def test_implicit_with_source_term_fails_like_the_reference():
    # the reference's Newton iteration does not converge on the manufactured
    # solution with the source term (first step, relative residual 0.55 after
    # nNewtonIter = 100 iterations: "Newton NOT converged"); the solver
    # reports the same outcome as a status
    with tempfile.TemporaryDirectory() as tmp:
        meshgen.sinewave_mesh(8, periodic=True).write_gmsh(os.path.join(tmp, "sine.msh"))
        case = cc.CaseData.from_text(
            meshgen.sinewave_ini("sine", order=2, limiter=2, periodic=True, implicit=True, cfl=1.0,
                                 t_end=1.0), tmp)
        s = cc.Solver(case)
        with pytest.raises(cc.CcfdError) as e:
            s.run(5)
        s.close()
    assert e.value.status == 5  # CCFD_ERR_NEWTON
