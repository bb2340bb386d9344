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


def test_mixed_precision_blocks_are_fp32_roundings():
    with tempfile.TemporaryDirectory() as tmp:
        case = _airfoil(tmp, 32, 12, True, cfl=10.0, max_iter=5, precision=1)
    n = case.n_cells
    rng = np.random.default_rng(12)
    prim = case.prim0() * (1.0 + 0.05 * rng.uniform(-1.0, 1.0, (n, 4)))
    s = cc.Solver(case, reorder=True)
    try:
        s.set_state(prim)
        _, Di, O = s.build_matrix(0.0, 0.02)
    finally:
        s.close()
    _, _, Dir, Or = restated.build_matrix(case, prim, restated.residual(case, prim, 0.02), 0.0, 0.02)
    # D^-1: the FP64 inverse rounded once; off-diagonal blocks: the FP64
    # column rounded, then scaled by -dt and rounded again
    assert np.array_equal(Di, Dir.astype(np.float32).astype(np.float64))
    assert _rel(O, Or) <= 2.0 ** -22


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
