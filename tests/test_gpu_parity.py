"""Parity of the CUDA path (through the C ABI) with the oracle and with the
compiled reference's outputs.

Tolerances (stated by the task for FP64): residual evaluations agree to 1e-12
in max-norm relative to max|R| per variable; explicit runs agree to 1e-10 in
L1 and L-infinity.  Where no transcendental function is involved the FP64 path
is expected to be bit-identical, and a test asserts that too.
"""
import os
import tempfile

import numpy as np
import pytest

import ccfd_b200 as cc
from ccfd_b200 import meshgen
from oracle import refdump, restated
from tests.golden import cases as CASES
from tests.helpers import l1_linf, rel_max_err, sod_frobenius

pytestmark = pytest.mark.gpu

RES_TOL = 1e-12
RUN_TOL = 1e-10


@pytest.mark.parametrize("key", sorted(CASES.residual_cases()))
def test_residual_matches_oracle_and_reference(ref_small, key):
    spec = CASES.residual_cases()[key]
    with tempfile.TemporaryDirectory() as tmp:
        case, _, _ = CASES.load_case(spec, tmp)
        prim = ref_small[f"{key}/prim"].reshape(-1, 4)
        s = cc.Solver(case, reorder=True)
        s.set_state(prim)
        ut, gr = s.fv_time_derivative(spec["time"], with_grad=True)
        uo, go, _, _ = restated.residual(case, prim, spec["time"], with_extras=True)
        s.close()
    assert rel_max_err(ut, uo) <= RES_TOL
    assert rel_max_err(ut, ref_small[f"{key}/u_t"]) <= RES_TOL
    assert rel_max_err(gr[:, :4], go[:, :4]) <= RES_TOL
    assert rel_max_err(gr[:, 4:], go[:, 4:]) <= RES_TOL


@pytest.mark.parametrize("flux", [2, 3, 4, 5, 6, 7, 8, 9, 10, 11])
@pytest.mark.parametrize("order,limiter", [(1, 1), (2, 1), (2, 2)])
def test_residual_bit_identical_without_transcendentals(flux, order, limiter):
    # Euler zoo without the exact-solution boundary: every operation is
    # + - * / sqrt, correctly rounded on both sides
    ini = CASES.zoo_ini(flux, order, limiter).replace("meshBCtype = 601", "meshBCtype = 501")
    case = cc.CaseData.from_text(ini)
    rng = np.random.Generator(np.random.PCG64(flux * 10 + order + limiter))
    n = case.n_cells
    prim = np.stack([rng.uniform(0.5, 2, n), rng.uniform(-1.5, 1.5, n),
                     rng.uniform(-1.5, 1.5, n), rng.uniform(0.5, 2, n)], 1)
    s = cc.Solver(case)
    s.set_state(prim)
    ut = s.fv_time_derivative(0.0)
    s.close()
    uo = restated.residual(case, prim, 0.0)
    assert np.array_equal(ut, uo)


@pytest.mark.parametrize("name", ["sod_FF01", "sod_FF02", "sod_FF03", "sod_FF04", "sod_FF05",
                                  "sod_FF06", "sod_FF07", "sod_FF09", "sod_FF11", "sod_SO2_BJ",
                                  "sod_SO2_VK", "sod_TO2_3RK", "sod_TO2_4RK", "sod_TO2_5RK"])
def test_reference_regression_suite_on_gpu(sod_check, name):
    g = sod_check[name]
    case = cc.CaseData.from_text(g["ini"])
    s = cc.Solver(case)
    rep = s.run(0)
    prim = s.get_state()
    s.close()
    assert rep["finished"] and abs(rep["t"] - 0.25) < 1e-12
    assert sod_frobenius(case, prim, g) < 1e-5
    po, info = restated.run_explicit(case)
    assert rep["iterations"] == info["iterations"]
    l1, linf = l1_linf(prim, po)
    assert l1 <= RUN_TOL and linf <= RUN_TOL


@pytest.mark.parametrize("key", sorted(CASES.run_cases()))
def test_explicit_run_matches_reference_fixture(ref_small, key):
    spec = CASES.run_cases()[key]
    with tempfile.TemporaryDirectory() as tmp:
        case, _, _ = CASES.load_case(spec, tmp)
        s = cc.Solver(case, reorder=True)
        rep = s.run(spec["steps"])
        prim = s.get_state()
        s.close()
    ref = ref_small[f"{key}/pvar"].reshape(-1, 4)
    info = ref_small[f"{key}/info"]
    hist = ref_small[f"{key}/history"].reshape(-1, 8)
    assert rep["iterations"] == int(info[1])
    assert abs(rep["t"] - info[0]) <= 1e-14
    l1, linf = l1_linf(prim, ref)
    assert l1 <= RUN_TOL and linf <= RUN_TOL
    # global residual of the last step (src/analyze.c:521-539)
    np.testing.assert_allclose(rep["residual"][:4], hist[-1, 2:6], rtol=1e-10, atol=1e-300)


def test_results_independent_of_ordering_and_repeatable():
    with tempfile.TemporaryDirectory() as tmp:
        meshgen.dmr_mesh(40, 10).write_gmsh(os.path.join(tmp, "dmr.msh"))
        case = cc.CaseData.from_text(meshgen.dmr_ini("dmr", t_end=0.01), tmp)
        out = []
        for reorder in (1, 0, 1, 2):  # Hilbert, reference numbering, Hilbert, reverse Cuthill-McKee
            s = cc.Solver(case, reorder=reorder)
            rep = s.run(0)
            out.append((s.get_state(), rep["residual"][:4]))
            s.close()
    assert all(np.array_equal(out[0][0], o[0]) for o in out[1:])
    assert out[0][1] == out[2][1]


def test_full_size_dmr_residual_matches_oracle():
    """Double Mach reflection at its benchmark size (1000 x 250 quads split
    into 500,000 triangles): one residual at the initial state and after two
    RK3 steps, against the oracle."""
    with tempfile.TemporaryDirectory() as tmp:
        meshgen.dmr_mesh(1000, 250).write_gmsh(os.path.join(tmp, "dmr.msh"))
        case = cc.CaseData.from_text(meshgen.dmr_ini("dmr"), tmp)
    s = cc.Solver(case, reorder=True)
    ut = s.fv_time_derivative(0.0)
    uo = restated.residual(case, case.prim0(), 0.0)
    assert rel_max_err(ut, uo) <= RES_TOL
    rep = s.run(2)
    prim = s.get_state()
    s.close()
    po, info = restated.run_explicit(case, nsteps=2)
    assert rep["iterations"] == 2 == info["iterations"]
    l1, linf = l1_linf(prim, po)
    assert l1 <= RUN_TOL and linf <= RUN_TOL
    assert np.all(prim[:, 0] > 0) and np.all(prim[:, 3] > 0)


def test_nonfinite_time_step_is_reported_not_fatal():
    case = cc.CaseData.from_text(meshgen.sod_ini(40, 2, t_end=0.01))
    s = cc.Solver(case)
    prim = case.prim0()
    prim[7, 0] = np.nan
    s.set_state(prim)
    with pytest.raises(cc.CcfdError) as e:
        s.run(0)
    assert e.value.status == 4  # CCFD_ERR_DT, "Convective Time Step NaN"
    # the context stays usable
    s.set_state(case.prim0())
    s.time = 0.0
    rep = s.run(3)
    assert rep["iterations"] >= 3
    s.close()


SINE_RUNS = ["sine_euler_run", "sine_ns_run", "sine_cart_o1_run", "sine_periodic_run",
             "sine_periodic_ns_cart_run"]


@pytest.mark.parametrize("key", SINE_RUNS)
def test_error_norms_match_oracle_and_reference(ref_small, key):
    # manufactured solution with the source term, then calcErrors
    # (ccfd_errors) against the oracle on the same state and against the
    # norms the reference printed
    spec = CASES.run_cases()[key]
    with tempfile.TemporaryDirectory() as tmp:
        case, _, _ = CASES.load_case(spec, tmp)
        s = cc.Solver(case, reorder=True)
        rep = s.run(spec["steps"])
        prim = s.get_state()
        e = s.errors()
        s.close()
        eo = restated.errors(case, prim, rep["t"])
    for k in ("L1", "L2", "Linf"):
        np.testing.assert_allclose(e[k], eo[k], rtol=1e-12, atol=0)
    printed = ref_small[f"{key}/errors_printed"]
    got = np.stack([e["L1"], e["L2"], e["Linf"]])
    np.testing.assert_allclose(got, printed, rtol=6e-6, atol=0)


def test_driver_prints_error_analysis():
    import re
    import subprocess
    driver = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                          "ccfd_b200", "lib", "ccfd_run")
    with tempfile.TemporaryDirectory() as tmp:
        meshgen.sinewave_mesh(16).write_gmsh(os.path.join(tmp, "sine.msh"))
        ini = os.path.join(tmp, "sine.ini")
        with open(ini, "w") as f:
            f.write(meshgen.sinewave_ini("sine", order=2, limiter=2, t_end=0.2))
        r = subprocess.run([driver, ini, "--no-output"], capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stdout + r.stderr
        case = cc.CaseData.from_text(open(ini).read(), tmp)
        s = cc.Solver(case)
        s.run(0)
        e = s.errors()
        s.close()
    rows = {m.group(1): [float(v) for v in m.group(2).split()]
            for m in re.finditer(r"^\| (L1  |L2  |Linf):\s+(.*)$", r.stdout, re.M)}
    assert set(rows) == {"L1  ", "L2  ", "Linf"}
    np.testing.assert_allclose(rows["L1  "], e["L1"], rtol=6e-6)
    np.testing.assert_allclose(rows["Linf"], e["Linf"], rtol=6e-6)


@pytest.mark.parametrize("shape", ["one_triangle", "one_quad", "two_cells"])
def test_tiny_meshes_match_oracle(shape):
    # degenerate sizes: a single cell (every face a boundary face, a tile
    # without rings) and two cells sharing one face
    nodes = np.array([[0.0, 0.0], [1.0, 0.0], [1.0, 1.0], [0.0, 1.0]])
    if shape == "one_triangle":
        mesh = meshgen.RawMesh(nodes[:3], tria=[[0, 1, 2, 1]], bc=[[0, 1, 301], [1, 2, 401], [2, 0, 101]])
    elif shape == "one_quad":
        mesh = meshgen.RawMesh(nodes, quad=[[0, 1, 2, 3, 1]],
                               bc=[[0, 1, 101], [1, 2, 401], [2, 3, 101], [3, 0, 301]])
    else:
        mesh = meshgen.RawMesh(nodes, tria=[[0, 1, 2, 1], [0, 2, 3, 1]],
                               bc=[[0, 1, 101], [1, 2, 401], [2, 3, 101], [3, 0, 301]])
    ini = """meshType = 0
meshFormat = .msh
meshFile = tiny
nBC = 3
BCtype = 101
BCtype = 301
rho = 1.2
mach = 0.4
alpha = 10.0
pressure = 1.1
BCtype = 401
icType = 1
nDomains = 1
domainID = 1
rho = 1.0
mach = 0.3
alpha = 20.0
pressure = 1.0
fluxFunction = 5
spatialOrder = 2
limiter = 2
venk_k = 5.0
timeOrder = 2
nRKstages = 3
CFL = 0.5
stationary = F
tEnd = 10.0
maxIter = 100000
fileName = tiny
IOtimeInterval = 10.0
IOiterInterval = 100000000
outputFormat = 3
"""
    with tempfile.TemporaryDirectory() as tmp:
        mesh.write_gmsh(os.path.join(tmp, "tiny.msh"))
        case = cc.CaseData.from_text(ini, tmp)
    s = cc.Solver(case)
    ut = s.fv_time_derivative(0.0)
    uo = restated.residual(case, case.prim0(), 0.0)
    assert rel_max_err(ut, uo) <= RES_TOL
    rep = s.run(5)
    prim = s.get_state()
    s.close()
    po, info = restated.run_explicit(case, nsteps=5)
    assert rep["iterations"] == info["iterations"] == 5
    l1, linf = l1_linf(prim, po)
    assert l1 <= RUN_TOL and linf <= RUN_TOL


def test_state_transfers_roundtrip_in_reference_order():
    # the state moves in the caller's (reference) cell order and is permuted
    # and converted on the device: primitive and conservative round trips,
    # into a new array and into a caller-provided one
    with tempfile.TemporaryDirectory() as tmp:
        meshgen.dmr_mesh(40, 10).write_gmsh(os.path.join(tmp, "dmr.msh"))
        case = cc.CaseData.from_text(meshgen.dmr_ini("dmr"), tmp)
    s = cc.Solver(case, reorder=True)
    rng = np.random.Generator(np.random.PCG64(11))
    n = case.n_cells
    prim = np.stack([rng.uniform(0.5, 2, n), rng.uniform(-1, 1, n), rng.uniform(-1, 1, n),
                     rng.uniform(0.5, 2, n)], 1)
    s.set_state(prim)
    assert np.array_equal(s.get_state(), prim)
    out = np.full((n, 4), np.nan)
    assert s.get_state(out=out) is out and np.array_equal(out, prim)
    cons = s.get_state(cc.CONSERVATIVE)
    assert np.allclose(cons[:, 1], prim[:, 1] * prim[:, 0], rtol=1e-15)
    s.set_state(cons, cc.CONSERVATIVE)
    np.testing.assert_allclose(s.get_state(), prim, rtol=1e-14)
    with pytest.raises(ValueError):
        s.get_state(out=np.empty((n, 3)))
    s.close()


def test_state_upload_returns_after_its_copy():
    # ccfd_set_state returns once the caller's array is copied and lets the
    # conversion run on in the context's stream: overwriting a pinned array
    # right after the call leaves the uploaded state intact, and a run that
    # follows the upload at once equals one after a synchronising read
    import torch

    with tempfile.TemporaryDirectory() as tmp:
        meshgen.dmr_mesh(400, 100).write_gmsh(os.path.join(tmp, "dmr.msh"))
        case = cc.CaseData.from_text(meshgen.dmr_ini("dmr"), tmp)
    a = cc.Solver(case, reorder=True)
    b = cc.Solver(case, reorder=True)
    n = case.n_cells
    a.run(2)
    prim = a.get_state()
    host = torch.empty((n, 4), dtype=torch.float64, pin_memory=True).numpy()
    for _ in range(3):
        host[:] = prim
        a.set_state(host)
        host[:] = np.nan
        assert np.array_equal(a.get_state(), prim)
    host[:] = prim
    a.set_state(host)
    host[:] = np.nan
    a.run(3)
    b.run(2)
    b.set_state(prim)
    assert np.array_equal(b.get_state(), prim)
    b.run(3)
    assert np.array_equal(a.get_state(), b.get_state())
    a.close()
    b.close()


@pytest.mark.skipif(not refdump.have_ref(), reason="compiled reference not built")
def test_sod_400x20_to_t_end_matches_compiled_reference():
    """The small plain configuration: Sod shock tube on [0,1]x[0,0.05],
    400 x 20 Cartesian quads (the reference's own generator), Roe, second
    order least squares with Barth-Jespersen, 3-stage RK (timeOrder 2),
    CFL 0.5, to t_end = 0.2, against the compiled reference run live."""
    ini = meshgen.sod_ini(400, 20, t_end=0.2, flux=2, order=2, limiter=1, cfl=0.5)
    case = cc.CaseData.from_text(ini)
    assert case.n_cells == 8000
    s = cc.Solver(case, reorder=True)
    rep = s.run(0)
    prim = s.get_state()
    s.close()
    d = refdump.run_ref(ini, "run", 0, threads=8)
    ref = d["pvar"].reshape(-1, 4)
    assert rep["finished"] and abs(rep["t"] - 0.2) <= 1e-14
    assert rep["iterations"] == int(d["run_info"][1])
    l1, linf = l1_linf(prim, ref)
    assert l1 <= RUN_TOL and linf <= RUN_TOL
