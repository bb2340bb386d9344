"""Solution output in the reference's CSV and curve formats (with the
exact-solution files) and the command-line driver.

The writer is checked on the CPU with the oracle's state of the reference's
own regression cases (check/*.ini): the written file must reproduce the
golden CSV within the reference's tolerance (Frobenius norm of the
differences of x, density and velocity <= 1e-5, check/check.py:33-42).  The
driver (ccfd_run) runs the same cases on the GPU.
"""
import json
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

import ccfd_b200 as cc
from oracle import restated
from tests.golden import cases as CASES

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = os.path.join(ROOT, "ccfd_b200", "lib", "ccfd_run")


def _frobenius_vs_golden(path, g):
    data = np.genfromtxt(path, skip_header=1, delimiter=",")
    gold = np.stack([g["x"], g["rho"], g["u"]], 1)
    return float(np.linalg.norm(data[:, 0:3] - gold))


def test_csv_writer_reproduces_golden_output(sod_check):
    for name in ("sod_FF02", "sod_SO2_VK", "sod_TO2_4RK"):
        g = sod_check[name]
        case = cc.CaseData.from_text(g["ini"])
        prim, info = restated.run_explicit(case)
        cwd = os.getcwd()
        with tempfile.TemporaryDirectory() as tmp:
            os.chdir(tmp)
            try:
                path = case.write_output(prim, info["t"], info["iterations"])
                assert path == g["target"]
                assert _frobenius_vs_golden(path, g) < 1e-5
            finally:
                os.chdir(cwd)


def test_writer_refuses_formats_it_does_not_build(sod_check):
    # CGNS (outputFormat = 1) needs the CGNS library
    g = sod_check["sod_FF02"]
    ini = re.sub(r"(?im)^(\s*outputformat\s*=\s*)3", r"\g<1>1", g["ini"])
    case = cc.CaseData.from_text(ini)
    assert case.c.output_format == 1
    cwd = os.getcwd()
    with tempfile.TemporaryDirectory() as tmp:
        os.chdir(tmp)
        try:
            with pytest.raises(cc.CcfdError):
                case.write_output(case.prim0(), 0.0, 0)
            assert os.listdir(tmp) == []
        finally:
            os.chdir(cwd)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["sod_FF05", "sod_SO2_BJ", "sod_TO2_3RK"])
def test_driver_runs_regression_case(sod_check, name):
    g = sod_check[name]
    with tempfile.TemporaryDirectory() as tmp:
        with open(os.path.join(tmp, "case.ini"), "w") as f:
            f.write(g["ini"])
        r = subprocess.run([DRIVER, "case.ini"], cwd=tmp, capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stdout + r.stderr
        assert f"wrote {g['target']}" in r.stdout
        assert _frobenius_vs_golden(os.path.join(tmp, g["target"]), g) < 1e-5


@pytest.fixture(scope="module")
def ref_output():
    with open(os.path.join(ROOT, "tests", "golden", "ref_output.json")) as f:
        return json.load(f)


def _numbers(text):
    return np.array([float(v) for v in re.findall(r"-?\d+\.\d+(?:e[+-]\d+)?", text)])


def _files_equal_to_printed_digits(got, want, name):
    if name.endswith(".dem"):
        assert got == want, name
        return
    assert got.splitlines()[0] == want.splitlines()[0], name
    assert len(got.splitlines()) == len(want.splitlines()), name
    a, b = _numbers(got), _numbers(want)
    assert a.shape == b.shape, name
    # the last printed digit, or 1e-7 relative where the run agrees to
    # rounding only (implicit iterates)
    np.testing.assert_allclose(a, b, rtol=1e-7, atol=2.1e-9, err_msg=name)


@pytest.mark.parametrize("key", sorted(CASES.output_cases()))
def test_writer_reproduces_reference_files_from_its_state(ref_output, key):
    # the reference's final state through the writer: the solution file must
    # be the reference's, byte for byte (same name, header, sort, format)
    g = ref_output[key]
    prim = np.array(g["pvar"]).reshape(-1, 4)
    cwd = os.getcwd()
    with tempfile.TemporaryDirectory() as tmp:
        case, _, _ = CASES.load_case(CASES.output_cases()[key], tmp)
        out_dir = os.path.join(tmp, "out")
        os.mkdir(out_dir)
        os.chdir(out_dir)
        try:
            path = case.write_output(prim, g["t"], g["iterations"])
            with open(path) as f:
                text = f.read()
        finally:
            os.chdir(cwd)
    assert path in g["files"]
    assert text == g["files"][path]


def test_history_writer_reproduces_reference_residual_file(ref_output):
    # the reference's per-step residuals as history rows: the residual file
    # and its gnuplot script must be the reference's, byte for byte
    g = ref_output["out_sod_stationary_csv"]
    case = cc.CaseData.from_text(CASES.output_cases()["out_sod_stationary_csv"]["ini"])
    h = np.array(g["history"]).reshape(-1, 8)  # t after the step, dt, residuals [6]
    rows = np.zeros((len(h), 11))
    rows[:, 0] = np.arange(1, len(h) + 1)
    rows[:, 1:9] = h
    cwd = os.getcwd()
    with tempfile.TemporaryDirectory() as tmp:
        os.chdir(tmp)
        try:
            case.write_history(rows)
            got = {n: open(n).read() for n in sorted(os.listdir(tmp))}
        finally:
            os.chdir(cwd)
    assert sorted(got) == ["sod_analysis.csv", "sod_residuals.dem"]
    for name, text in got.items():
        assert text == g["files"][name], name


@pytest.mark.gpu
@pytest.mark.parametrize("key", sorted(CASES.output_cases()))
def test_driver_writes_reference_solution_and_exact_files(ref_output, key):
    # ccfd_run on the same .ini: the same files (flow solution and exact
    # solution) as the reference's dataOutput, equal to their printed digits
    g = ref_output[key]
    with tempfile.TemporaryDirectory() as tmp:
        ini, _ = CASES.materialise(CASES.output_cases()[key], tmp)
        with open(os.path.join(tmp, "case.ini"), "w") as f:
            f.write(ini)
        r = subprocess.run([DRIVER, "case.ini"], cwd=tmp, capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stdout + r.stderr
        written = sorted(n for n in os.listdir(tmp)
                         if n.endswith((".csv", ".curve", ".dem")) and "_CP_" not in n)
        assert written == sorted(g["files"])
        for name in written:
            with open(os.path.join(tmp, name)) as f:
                _files_equal_to_printed_digits(f.read(), g["files"][name], name)


def test_history_writer_record_points_and_append(tmp_path):
    # record-point files (initRecordPoints / evalRecordPoints format) and
    # appending further rows without repeating the headers
    ini = CASES.output_cases()["out_sod_stationary_csv"]["ini"] + CASES.RECORD_POINTS
    case = cc.CaseData.from_text(ini)
    xy, cells = case.record_points()
    assert len(cells) == 3
    w = 11 + 4 * 3
    rows = np.zeros((2, w))
    rows[:, 0] = [1, 2]
    rows[:, 1] = [0.01, 0.02]
    rows[:, 2] = [0.01, 0.01]
    rows[:, 3:7] = 1e-3
    rows[:, 11:] = np.arange(12, dtype=float) / 10
    cwd = os.getcwd()
    os.chdir(tmp_path)
    try:
        case.write_history(rows)
        case.write_history(rows, append=True)
        rp = open("sod_recordPoint_2.csv").read().splitlines()
        an = open("sod_analysis.csv").read().splitlines()
    finally:
        os.chdir(cwd)
    assert rp[0] == "Time, Density, VelocityX, VelocityY, Pressure" and len(rp) == 5
    assert rp[1] == "%20.12f,%20.12f,%20.12f,%20.12f,%20.12f" % (0.02, 0.8, 0.9, 1.0, 1.1)
    assert an[0].startswith("Iter, Time, Residual(RHO)") and len(an) == 5
    assert an[3] == "%7d, %13.8f, %15.8e, %15.8e, %15.8e, %15.8e" % (1, 0.02, 1e-3, 1e-3, 1e-3, 1e-3)
