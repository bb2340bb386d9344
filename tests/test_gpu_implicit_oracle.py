"""The implicit path on the GPU against the restated oracle (block-sparse
buildMatrix / calcDinv / LUSGS and implicitTimeStep of oracle/ccfd_oracle.c,
pinned to the compiled reference in tests/test_oracle_implicit.py), at sizes
where the reference's dense Jacobian cannot run.

* Jacobian blocks: the coloured finite-difference blocks of the GPU equal
  the column-by-column ones of the oracle (the same residual arithmetic per
  entry); LU-SGS of a vector to 1e-12.
* The NACA 0012 Navier-Stokes O-grid of the implicit steady configuration
  (256 x 128 quads, 32,768 cells, first cell 1e-4 chord, far field at 20
  chords, Mach 0.5, Re 5,000, AoA 1 deg, Roe, Venkatakrishnan K = 5,
  JFNK-GMRES with Krylov 30 and LU-SGS): implicit steps with the same Newton
  / GMRES counts, state and lift / drag within 1e-8.
* Steady states: the small airfoil converged to a relative residual of 1e-8
  (switched-evolution-relaxation CFL ramp) on both sides agrees in density
  and lift / drag within 1e-8.
* Mixed precision: the preconditioner's blocks from FP32-flux residuals are
  FP32 values close to the FP64 blocks, GMRES needs about as many
  iterations, and the converged states and lift / drag equal the FP64
  oracle's within 1e-6.
"""
import os
import tempfile

import numpy as np
import pytest

import ccfd_b200 as cc
from ccfd_b200 import meshgen
from oracle import restated
from tests.golden import cases as CASES

pytestmark = pytest.mark.gpu

TOL = 1e-8


def _rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _airfoil(tmp, ni, nj, ns, cfl, max_iter, h0=1e-2, r_far=5.0, kdim=30, rel=1e-8, mach=0.5, alpha=2.0,
             reynolds=500.0, precision=0, ser=None, dfl=None):
    wall = 201 if ns else 101
    meshgen.naca_ogrid(0.0, 0.0, 0.12, ni, nj, r_far=r_far, h0=h0, wall_code=wall).write_gmsh(
        os.path.join(tmp, "af.msh"))
    ini = meshgen.airfoil_ini("af", mach=mach, alpha=alpha, navier_stokes=ns, reynolds=reynolds, flux=2,
                              implicit=True, precond=True, n_kdim=kdim, cfl=cfl, max_iter=max_iter,
                              rel_res=rel, precision=precision, dfl=dfl, ser_cfl_max=ser)
    return cc.CaseData.from_text(ini, tmp)


@pytest.mark.parametrize("ns,ni,nj", [(False, 32, 12), (True, 32, 12), (True, 128, 48)])
def test_jacobian_blocks_and_lusgs_match_restated(ns, ni, nj):
    with tempfile.TemporaryDirectory() as tmp:
        case = _airfoil(tmp, ni, nj, ns, cfl=10.0, max_iter=5)
    n = case.n_cells
    rng = np.random.default_rng(11)
    prim = case.prim0() * (1.0 + 0.05 * rng.uniform(-1.0, 1.0, (n, 4)))
    vec = rng.standard_normal((n, 4))
    t, dt = 0.0, 0.02
    s = cc.Solver(case, reorder=True)
    try:
        s.set_state(prim)
        D, Di, O = s.build_matrix(t, dt)
        x = s.lusgs(vec)
    finally:
        s.close()
    rxk = restated.residual(case, prim, t + dt)
    _, Dr, Dir, Or = restated.build_matrix(case, prim, rxk, t, dt)
    assert _rel(D, Dr) <= 1e-12 and _rel(O, Or) <= 1e-12 and _rel(Di, Dir) <= 1e-12
    assert _rel(x, restated.lusgs(case, Dir, Or, vec)) <= 1e-12


# Mixed precision builds the preconditioner's blocks from FP32-flux residuals
# with a perturbation of sqrt(FLT_EPSILON) (a step below the FP32 resolution
# of the state would vanish).  Its columns differ from the FP64 ones by the
# finite-difference truncation, by FP32 rounding and -- the largest part --
# where the step crosses a branch of the Venkatakrishnan limiter; measured
# on this case: 1.7e-2 (D), 1.4e-1 (D^-1), 7.6e-2 (off-diagonal) of the
# largest entry.  The blocks only steer GMRES: the iteration counts stay
# close to FP64 (next test) and the converged state is the FP64 one (steady
# tests below).
MIXED_BLOCK_TOL = 0.25


def test_mixed_precision_blocks_approximate_fp64_blocks():
    with tempfile.TemporaryDirectory() as tmp:
        case = _airfoil(tmp, 32, 12, True, cfl=10.0, max_iter=5, precision=1)
    n = case.n_cells
    rng = np.random.default_rng(12)
    prim = case.prim0() * (1.0 + 0.05 * rng.uniform(-1.0, 1.0, (n, 4)))
    s = cc.Solver(case, reorder=True)
    try:
        s.set_state(prim)
        D, Di, O = s.build_matrix(0.0, 0.02)
    finally:
        s.close()
    _, Dr, Dir, Or = restated.build_matrix(case, prim, restated.residual(case, prim, 0.02), 0.0, 0.02)
    errs = (_rel(D, Dr), _rel(Di, Dir), _rel(O, Or))
    assert max(errs) <= MIXED_BLOCK_TOL, errs
    # D^-1 and the off-diagonal blocks are FP32 values
    assert np.array_equal(Di, Di.astype(np.float32).astype(np.float64))
    assert np.array_equal(O, O.astype(np.float32).astype(np.float64))


@pytest.mark.parametrize("ns", [False, True])
def test_mixed_precision_preconditioner_keeps_gmres_counts(ns):
    # the same implicit steps in FP64 and in mixed precision: the FP32-flux
    # blocks precondition GMRES about as well as the FP64 ones
    reps = {}
    for precision in (0, 1):
        with tempfile.TemporaryDirectory() as tmp:
            case = _airfoil(tmp, 32, 12, ns, cfl=10.0, max_iter=20, precision=precision)
        s = cc.Solver(case, reorder=True)
        try:
            reps[precision] = s.run(20)
        finally:
            s.close()
    assert reps[0]["status"] == 0 and reps[1]["status"] == 0
    assert reps[1]["iterations"] == reps[0]["iterations"]
    assert reps[1]["gmres_iterations"] <= 1.25 * reps[0]["gmres_iterations"], (reps[0], reps[1])


def test_c3_airfoil_implicit_steps_match_restated():
    with tempfile.TemporaryDirectory() as tmp:
        case = _airfoil(tmp, 256, 128, True, cfl=10.0, max_iter=100, h0=1e-4, r_far=20.0, alpha=1.0,
                        reynolds=5000.0)
    assert case.n_cells == 32768
    steps = 3
    s = cc.Solver(case, reorder=True)
    try:
        rep = s.run(steps)
        prim = s.get_state()
    finally:
        s.close()
    po, info, hist = restated.run_implicit(case, steps)
    assert info["status"] == 0 and rep["status"] == 0
    assert rep["iterations"] == info["iterations"] == steps
    assert rep["newton_iterations"] == info["newton_iterations"]
    assert rep["gmres_iterations"] == info["gmres_iterations"]
    err = np.abs(prim - po).max(axis=0) / np.abs(po).max(axis=0)
    assert err.max() <= TOL, err
    assert abs(rep["cl"] - info["cl"]) <= TOL and abs(rep["cd"] - info["cd"]) <= TOL


@pytest.mark.parametrize("ns", [False, True])
def test_steady_state_matches_restated(ns):
    # Euler: CFL 20 ramped to at most 300; Navier-Stokes (Re 500): CFL and
    # DFL 10 ramped to at most 3000
    with tempfile.TemporaryDirectory() as tmp:
        if ns:
            case = _airfoil(tmp, 32, 12, True, cfl=10.0, max_iter=1500, ser=3000.0, dfl=10.0)
        else:
            case = _airfoil(tmp, 32, 12, False, cfl=20.0, max_iter=1500, ser=300.0)
    s = cc.Solver(case, reorder=True)
    try:
        rep = s.run(0)
        prim = s.get_state()
    finally:
        s.close()
    po, info, hist = restated.run_implicit(case, 0, ser_cfl_max=case.params.ser_cfl_max)
    assert info["converged"] and rep["converged"]
    # both at a relative residual of 1e-8 (possibly a step apart)
    assert abs(rep["iterations"] - info["iterations"]) <= 2
    assert rep["residual"][0] <= 1e-8 * hist[0, 2] * 1.5
    rho = np.abs(prim[:, 0] - po[:, 0]).max() / np.abs(po[:, 0]).max()
    assert rho <= TOL
    assert abs(rep["cl"] - info["cl"]) <= TOL and abs(rep["cd"] - info["cd"]) <= TOL


def test_mixed_precision_steady_state_matches_fp64_oracle():
    # FP32 Krylov basis and LU-SGS sweeps, FP64 residuals and Newton update:
    # converged to the same relative residual of 1e-8, the steady state is
    # the FP64 one
    with tempfile.TemporaryDirectory() as tmp:
        fp64 = _airfoil(tmp, 32, 12, False, cfl=20.0, max_iter=1500, ser=300.0)
        mixed = _airfoil(tmp, 32, 12, False, cfl=20.0, max_iter=1500, ser=300.0, precision=1)
    s = cc.Solver(mixed, reorder=True)
    try:
        rep = s.run(0)
        prim = s.get_state()
    finally:
        s.close()
    po, info, _ = restated.run_implicit(fp64, 0, ser_cfl_max=300.0)
    assert rep["converged"] and info["converged"]
    assert np.abs(prim[:, 0] - po[:, 0]).max() / np.abs(po[:, 0]).max() <= 1e-6
    assert abs(rep["cl"] - info["cl"]) <= 1e-6 and abs(rep["cd"] - info["cd"]) <= 1e-6


def test_mixed_batch_of_airfoils_converges_to_fp64_lift_and_drag():
    # three airfoil flows converged in one batch, FP64 and mixed precision
    flows = [(0.5, 2.0), (0.4, 1.0), (0.6, -1.0)]
    results = {}
    for precision in (0, 1):
        cases = []
        with tempfile.TemporaryDirectory() as tmp:
            for mach, alpha in flows:
                cases.append(_airfoil(tmp, 32, 12, False, cfl=20.0, max_iter=1500, ser=300.0, mach=mach,
                                      alpha=alpha, precision=precision))
        b = cc.Batch(0)
        members = [cc.Solver(c) for c in cases]
        try:
            for m in members:
                b.add(m, 0)
            while b.step(64):
                pass
            results[precision] = [b.report(m) for m in members]
        finally:
            b.close()
            for m in members:
                m.close()
    for r64, r32 in zip(results[0], results[1]):
        assert r64["converged"] and r32["converged"]
        assert abs(r64["cl"] - r32["cl"]) <= 1e-6 and abs(r64["cd"] - r32["cd"]) <= 1e-6
