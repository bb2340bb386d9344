"""Batched stepping (ccfd_batch_*): every member's result equals the same
case stepped alone, bit for bit, whatever else is in the batch.

The batched stage kernel runs the same per-tile code as the single-instance
kernel, with the same operand order and the same per-cell summation order,
so an explicit member's state, time, time step and residual history are
identical alone and in any mix.  The mix below covers different meshes and
sizes, flux functions, orders, limiters, Euler and Navier-Stokes, FP64 and
mixed precision, different stop criteria, and members joining and leaving
while others run.
"""
import tempfile

import numpy as np
import pytest

import ccfd_b200 as cc
from tests.golden import cases as CASES

pytestmark = pytest.mark.gpu


def _specs():
    dmr = CASES._dmr_ini
    return {
        "dmr_hllc_vk": {"mesh": ("dmr", 24, 6), "ini": dmr(5, 2, 2, t_end=0.2), "eqn": "euler"},
        "dmr_roe_bj_short": {"mesh": ("dmr", 20, 5), "ini": dmr(2, 2, 1, t_end=0.004), "eqn": "euler"},
        "dmr_hllc_mixed": {"mesh": ("dmr", 30, 8),
                           "ini": dmr(5, 2, 2).replace("precision = 0", "precision = 1"), "eqn": "euler"},
        "zoo_ns_hllc_vk": {"mesh": None, "ini": CASES.zoo_ini(5, 2, 2, ns=True), "eqn": "navierstokes"},
        "zoo_stw_o1": {"mesh": None, "ini": CASES.zoo_ini(7, 1, 1), "eqn": "euler"},
        "zoo_ausmd_bj_rk4": {"mesh": None,
                             "ini": CASES.zoo_ini(9, 2, 1).replace("nRKstages = 3", "nRKstages = 4"),
                             "eqn": "euler"},
        # manufactured source term on a periodic mesh and on a mixed mesh
        # with the exact-solution boundary
        "sine_periodic_src": dict(CASES.run_cases()["sine_periodic_run"]),
        "sine_ns_src": dict(CASES.run_cases()["sine_ns_run"]),
    }


def _solver(spec, tmp):
    case, _, _ = CASES.load_case(spec, tmp)
    return cc.Solver(case, reorder=True)


def _alone(spec, steps):
    with tempfile.TemporaryDirectory() as tmp:
        s = _solver(spec, tmp)
    rep = s.run(steps)
    prim = s.get_state()
    s.close()
    return prim, rep


def _same(rep_a, rep_b):
    for k in ("iterations", "t", "dt", "residual", "finished", "converged"):
        assert rep_a[k] == rep_b[k], k


def test_batch_members_equal_alone():
    specs = _specs()
    steps = 21  # one 16-step graph and five single steps
    alone = {k: _alone(v, steps) for k, v in specs.items()}
    b = cc.Batch(0)
    solvers = {}
    with tempfile.TemporaryDirectory() as tmp:
        for k, v in specs.items():
            solvers[k] = _solver(v, tmp)
    for s in solvers.values():
        b.add(s, steps)
    running = b.step(steps)
    assert running == 0
    for k, s in solvers.items():
        prim, rep = alone[k]
        assert np.array_equal(s.get_state(), prim), k
        _same(b.report(s), rep)
    # the short case stopped at its tEnd long before the budget
    assert b.report(solvers["dmr_roe_bj_short"])["finished"]
    assert b.report(solvers["dmr_roe_bj_short"])["iterations"] < steps
    b.close()
    for s in solvers.values():
        s.close()


def test_batch_join_and_leave_mid_run():
    specs = _specs()
    a, c = specs["dmr_hllc_vk"], specs["zoo_ns_hllc_vk"]
    prim_a, rep_a = _alone(a, 12)
    prim_c, rep_c = _alone(c, 9)
    with tempfile.TemporaryDirectory() as tmp:
        sa = _solver(a, tmp)
        sc = _solver(c, tmp)
    b = cc.Batch(0)
    b.add(sa)            # no step budget: runs until removed
    b.step(3)
    b.add(sc, 9)         # joins after three steps of the first member
    b.step(5)
    b.remove(sa)         # leaves after 8 steps, continues alone
    with pytest.raises(cc.CcfdError):
        b.step(0)
    b.step(4)            # the second member finishes its budget (9)
    rep = sa.run(4)
    assert np.array_equal(sa.get_state(), prim_a)
    _same(rep, rep_a)
    assert np.array_equal(sc.get_state(), prim_c)
    _same(b.report(sc), rep_c)
    # a member cannot be stepped alone while the batch owns it
    with pytest.raises(cc.CcfdError):
        sc.run(1)
    b.close()
    sc.run(1)  # released by the batch
    sa.close()
    sc.close()


def test_implicit_members_in_lockstep_equal_alone():
    # uneven implicit members (sizes, Krylov dimensions, preconditioner on /
    # off, Euler / Navier-Stokes, FP64 / mixed) advance in lockstep Newton / GMRES /
    # LU-SGS launches; each must match its own run alone exactly
    imp = CASES.implicit_cases()
    specs = {
        "pc": (dict(imp["naca_euler_imp_pc"]), 4),
        "nopc": (dict(imp["naca_euler_imp_nopc"]), 4),
        "ns_pc": (dict(imp["naca_ns_imp_pc"]), 3),
        "pc_small": ({"mesh": ("naca", 24, 8, 101), "ini": imp["naca_euler_imp_pc"]["ini"],
                      "eqn": "euler"}, 5),
        "pc_mixed": ({"mesh": ("naca", 32, 12, 101),
                      "ini": imp["naca_euler_imp_pc"]["ini"].replace("precision = 0", "precision = 1"),
                      "eqn": "euler"}, 4),
    }
    alone = {}
    for k, (spec, steps) in specs.items():
        with tempfile.TemporaryDirectory() as tmp:
            s = _solver(spec, tmp)
        rep = s.run(steps)
        alone[k] = (s.get_state(), rep)
        s.close()
    b = cc.Batch(0)
    solvers = {}
    with tempfile.TemporaryDirectory() as tmp:
        for k, (spec, steps) in specs.items():
            solvers[k] = _solver(spec, tmp)
    for k, s in solvers.items():
        b.add(s, specs[k][1])
    assert b.step(10) == 0
    for k, s in solvers.items():
        prim, rep = alone[k]
        got = b.report(s)
        assert np.array_equal(s.get_state(), prim), k
        _same(got, rep)
        assert got["newton_iterations"] == rep["newton_iterations"], k
        assert got["gmres_iterations"] == rep["gmres_iterations"], k
        assert got["cl"] == rep["cl"] and got["cd"] == rep["cd"], k
    b.close()
    for s in solvers.values():
        s.close()
