"""Per-step history (the data of the reference's analyze: residual file,
CL / CD, record points) recorded on the device at every step end, against
the compiled reference's per-step residuals, alone and as a batch member,
explicit and implicit."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

import ccfd_b200 as cc
from ccfd_b200 import meshgen
from tests.golden import cases as CASES

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = os.path.join(ROOT, "ccfd_b200", "lib", "ccfd_run")


def _check_rows(rows, hist, rtol, t_rtol=1e-13):
    # rows: iteration, t, dt, residuals [6], CL, CD; hist: t, dt, residuals [6]
    assert np.array_equal(rows[:, 0], np.arange(1, len(hist) + 1))
    np.testing.assert_allclose(rows[:, 1:3], hist[:, 0:2], rtol=t_rtol, atol=0)
    np.testing.assert_allclose(rows[:, 3:7], hist[:, 2:6], rtol=rtol, atol=1e-300)


@pytest.mark.parametrize("key", ["dmr_hllc_vk_run", "zoo_ns_run", "sine_periodic_run"])
def test_explicit_history_matches_reference_residuals(ref_small, key):
    spec = CASES.run_cases()[key]
    with tempfile.TemporaryDirectory() as tmp:
        case, _, _ = CASES.load_case(spec, tmp)
        s = cc.Solver(case)
        s.set_history(64)  # smaller than the step count: drained per graph
        s.run(spec["steps"])
        rows = s.history()
        again = s.history()
        s.close()
    hist = ref_small[f"{key}/history"].reshape(-1, 8)
    assert len(rows) == len(hist) and len(again) == 0
    _check_rows(rows, hist, 1e-10)


def test_implicit_history_matches_reference_residuals_and_clcd(ref_small):
    key = "naca_euler_imp_pc"
    spec = CASES.implicit_cases()[key]
    with tempfile.TemporaryDirectory() as tmp:
        case, _, _ = CASES.load_case(spec, tmp)
        s = cc.Solver(case)
        s.set_history(64)
        rep = s.run(spec["steps"])
        rows = s.history()
        s.close()
    hist = ref_small[f"{key}/history"].reshape(-1, 8)
    _check_rows(rows, hist, 1e-6, t_rtol=1e-8)
    np.testing.assert_allclose(rows[:, 7:9], hist[:, 6:8], rtol=1e-6, atol=1e-12)  # CL / CD residuals
    assert rows[-1, 9] == rep["cl"] and rows[-1, 10] == rep["cd"]


def test_batch_member_history_equals_alone():
    with tempfile.TemporaryDirectory() as tmp:
        meshgen.dmr_mesh(40, 10).write_gmsh(os.path.join(tmp, "dmr.msh"))
        case = cc.CaseData.from_text(meshgen.dmr_ini("dmr", t_end=0.01), tmp)
        cells = [3, 117, 555]
        alone = cc.Solver(case)
        alone.set_history(64, cells)
        alone.run(0)
        want = alone.history()
        alone.close()
        a, b = cc.Solver(case), cc.Solver(case)
        a.set_history(64, cells)
        batch = cc.Batch()
        batch.add(a)
        batch.add(b)
        while batch.step(16):
            pass
        got = a.history()
        batch.close()
        state = a.get_state()
        a.close()
        b.close()
    assert np.array_equal(got, want)
    # the record cells' state after the last step
    assert np.array_equal(got[-1, 11:].reshape(-1, 4), state[cells])


def test_driver_writes_record_point_files():
    # record points (the reference's own initRecordPoints crashes on them, so
    # the files are checked against the solver's state): one row per step
    # with t + dt and the state of the cell the point lies in
    spec = CASES.output_cases()["out_sod_stationary_csv"]
    ini = spec["ini"] + CASES.RECORD_POINTS
    with tempfile.TemporaryDirectory() as tmp:
        with open(os.path.join(tmp, "case.ini"), "w") as f:
            f.write(ini)
        r = subprocess.run([DRIVER, "case.ini"], cwd=tmp, capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stdout + r.stderr
        files = [np.genfromtxt(os.path.join(tmp, f"sod_recordPoint_{k}.csv"), delimiter=",", skip_header=1)
                 for k in range(3)]
        with open(os.path.join(tmp, f"sod_recordPoint_0.csv")) as f:
            assert f.readline() == "Time, Density, VelocityX, VelocityY, Pressure\n"
        case = cc.CaseData.from_text(ini, tmp)
    xy, cells = case.record_points()
    s = cc.Solver(case)
    s.set_history(64)
    s.run(0)
    rows = s.history()
    prim = s.get_state()
    s.close()
    assert len(rows) == 12
    for k in range(3):
        assert files[k].shape == (12, 5)
        np.testing.assert_allclose(files[k][:, 0], rows[:, 1] + rows[:, 2], atol=1e-12)
        np.testing.assert_allclose(files[k][-1, 1:], prim[cells[k]], atol=1e-12)
