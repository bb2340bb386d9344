"""Serving with continuous batching (ccfd_server_*): each request's result is
the same alone and in the mix, the device-memory budget holds at every
scheduling round, and requests that arrive while others run are admitted as
memory frees up.

Explicit requests are bit-identical alone and served (same kernels, same
operand and summation order).  Implicit requests are stepped by the same
Newton / GMRES / LU-SGS code alone and served, so they are identical too.
"""
import tempfile

import numpy as np
import pytest

import ccfd_b200 as cc
from ccfd_b200 import meshgen
from tests.golden import cases as CASES

pytestmark = pytest.mark.gpu


def _cases(tmp):
    dmr = CASES._dmr_ini
    out = {}
    specs = {
        "dmr_hllc_vk": ({"mesh": ("dmr", 24, 6), "ini": dmr(5, 2, 2, t_end=0.2)}, 30),
        "dmr_roe_bj_short": ({"mesh": ("dmr", 20, 5), "ini": dmr(2, 2, 1, t_end=0.004)}, 0),
        "zoo_ns": ({"mesh": None, "ini": CASES.zoo_ini(5, 2, 2, ns=True)}, 25),
        "zoo_o1": ({"mesh": None, "ini": CASES.zoo_ini(3, 1, 1)}, 40),
        "dmr_mixed": ({"mesh": ("dmr", 30, 8), "ini": dmr(5, 2, 2).replace("precision = 0", "precision = 1")}, 20),
        "naca_implicit": ({"mesh": ("naca", 32, 12, 101),
                           "ini": CASES.implicit_cases()["naca_euler_imp_pc"]["ini"]}, 3),
    }
    for k, (spec, steps) in specs.items():
        case, _, _ = CASES.load_case(spec, tmp)
        out[k] = (case, steps)
    # a 2-D Riemann problem of the served stream (four quadrant states)
    path = tmp + "/r2d.msh"
    meshgen.riemann2d_mesh(40).write_gmsh(path)
    rng = np.random.Generator(np.random.PCG64(20260005))
    states = [(rng.uniform(0.1, 2), rng.uniform(-1, 1), rng.uniform(-1, 1), rng.uniform(0.1, 2))
              for _ in range(4)]
    out["riemann2d"] = (cc.CaseData.from_text(meshgen.riemann2d_ini("r2d", states), tmp), 15)
    return out


def _alone(case, steps):
    s = cc.Solver(case, reorder=True)
    rep = s.run(steps)
    prim = s.get_state()
    s.close()
    return prim, rep


def _serve(cases, budget, steps_per_poll, stagger):
    srv = cc.Server(0, hbm_budget_bytes=budget, max_running=64)
    ids = {}
    results = {}
    max_used = 0
    pending = list(cases.items())
    polls = 0
    while pending or len(results) < len(cases):
        # new requests arrive while others are running
        for _ in range(stagger if pending else 0):
            if pending:
                k, (case, steps) = pending.pop(0)
                ids[k] = srv.submit(case, steps)
        q, r, d = srv.poll(steps_per_poll)
        used, _ = srv.memory()
        max_used = max(max_used, used)
        for k, rid in ids.items():
            if k not in results:
                got = srv.result(rid)
                if got is not None:
                    results[k] = got
        polls += 1
        assert polls < 10000
    srv.close()
    return results, max_used


@pytest.mark.parametrize("budget_kind", ["roomy", "tight"])
def test_served_results_equal_alone(budget_kind):
    with tempfile.TemporaryDirectory() as tmp:
        cases = _cases(tmp)
        alone = {k: _alone(c, n) for k, (c, n) in cases.items()}
        est = {k: cc.estimate_device_bytes(c) for k, (c, _) in cases.items()}
        # tight: the largest request alone fits, but not all of them at once
        budget = 10 * sum(est.values()) if budget_kind == "roomy" else int(1.05 * max(est.values()))
        results, max_used = _serve(cases, budget, steps_per_poll=4, stagger=2)
    assert max_used <= budget
    for k, (rep, prim, times) in results.items():
        want_prim, want_rep = alone[k]
        assert rep["status"] == 0, k
        assert np.array_equal(prim, want_prim), k
        for f in ("iterations", "t", "dt", "residual", "finished", "converged"):
            assert rep[f] == want_rep[f], (k, f)
        assert times[0] <= times[1] <= times[2]


def test_estimate_covers_actual_device_memory():
    with tempfile.TemporaryDirectory() as tmp:
        cases = _cases(tmp)
    for k, (case, _) in cases.items():
        s = cc.Solver(case, reorder=True)
        actual = s.device_bytes()
        s.close()
        est = cc.estimate_device_bytes(case)
        assert actual <= est <= 3 * actual + (8 << 20), (k, actual, est)


def test_request_beyond_budget_is_refused():
    with tempfile.TemporaryDirectory() as tmp:
        case, _ = _cases(tmp)["dmr_hllc_vk"]
    srv = cc.Server(0, hbm_budget_bytes=1 << 20, max_running=4)
    with pytest.raises(cc.CcfdError):
        srv.submit(case, 5)
    srv.close()
