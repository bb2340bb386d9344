"""The CPU oracle (C restatement of the reference path) pinned against the
reference's own regression suite and against the compiled reference."""
import os
import tempfile

import numpy as np
import pytest

import ccfd_b200 as cc
from oracle import refdump, restated
from tests.golden import cases as CASES
from tests.helpers import rel_max_err, sod_frobenius


@pytest.mark.parametrize("name", ["sod_FF01", "sod_FF02", "sod_FF03", "sod_FF04", "sod_FF05",
                                  "sod_FF06", "sod_FF07", "sod_FF09", "sod_FF11", "sod_SO2_BJ",
                                  "sod_SO2_VK", "sod_TO2_3RK", "sod_TO2_4RK", "sod_TO2_5RK"])
def test_oracle_reproduces_reference_regression_suite(sod_check, name):
    g = sod_check[name]
    case = cc.CaseData.from_text(g["ini"])
    prim, info = restated.run_explicit(case)
    assert info["finished"] and abs(info["t"] - 0.25) < 1e-12
    # check/check.py:38-43: "ok" below 1e-5
    assert sod_frobenius(case, prim, g) < 1e-5


@pytest.mark.parametrize("key", sorted(CASES.residual_cases()))
def test_oracle_residual_matches_reference_fixture(ref_small, key):
    spec = CASES.residual_cases()[key]
    with tempfile.TemporaryDirectory() as tmp:
        case, _, _ = CASES.load_case(spec, tmp)
        prim = ref_small[f"{key}/prim"].reshape(-1, 4)
        ut, gr, _, _ = restated.residual(case, prim, spec["time"], with_extras=True)
    # bit-identical arithmetic except libm transcendental functions (pow /
    # tanh of the Godunov flux and the exact-solution boundary) whose last
    # bits can depend on the CPU's libm code path
    assert rel_max_err(ut, ref_small[f"{key}/u_t"]) <= 1e-13
    assert rel_max_err(gr[:, :4], ref_small[f"{key}/u_x"]) <= 1e-13


@pytest.mark.parametrize("key", sorted(CASES.run_cases()))
def test_oracle_explicit_run_matches_reference_fixture(ref_small, key):
    spec = CASES.run_cases()[key]
    if spec["eqn"] != "euler":
        pytest.skip("explicit oracle loop compared on Euler cases; NS via residual cases")
    with tempfile.TemporaryDirectory() as tmp:
        case, _, _ = CASES.load_case(spec, tmp)
        prim, info = restated.run_explicit(case, nsteps=spec["steps"])
    ref = ref_small[f"{key}/pvar"].reshape(-1, 4)
    assert info["iterations"] == int(ref_small[f"{key}/info"][1])
    assert np.abs(prim - ref).max() <= 1e-10 * np.abs(ref).max()


@pytest.mark.skipif(not refdump.have_ref(), reason="compiled reference not built")
@pytest.mark.parametrize("key", ["dmr_f02_vk", "dmr_f05_bj", "zoo_euler_vk", "dmr_f10_o1"])
def test_oracle_bit_identical_to_live_reference(key):
    spec = CASES.residual_cases()[key]
    with tempfile.TemporaryDirectory() as tmp:
        case, ini, files = CASES.load_case(spec, tmp)
        prim = CASES.random_state(spec, tmp)
        d = refdump.run_ref(ini, "residual", spec["time"], state=prim, files=files)
        ut = restated.residual(case, prim, spec["time"])
    assert np.array_equal(ut.ravel(), d["u_t"])


@pytest.mark.skipif(not refdump.have_ref(), reason="compiled reference not built")
@pytest.mark.parametrize("kind", ["dmr", "periodic_gmsh", "periodic_cartesian", "periodic_gmsh4", "dmr_gmsh4",
                                  "sine_emc2", "riemann_emc2"])
def test_mesh_builder_bit_identical_to_reference(kind):
    from ccfd_b200 import meshgen
    with tempfile.TemporaryDirectory() as tmp:
        files = {}
        if kind == "dmr":
            meshgen.dmr_mesh(30, 8, seed=5).write_gmsh(os.path.join(tmp, "dmr.msh"))
            ini = meshgen.dmr_ini("dmr")
            files = {"dmr.msh": os.path.join(tmp, "dmr.msh")}
        elif kind == "periodic_gmsh":
            # connectPeriodicBC: matched boundary faces become interior faces
            meshgen.sinewave_mesh(7, periodic=True).write_gmsh(os.path.join(tmp, "sine.msh"))
            ini = meshgen.sinewave_ini("sine", periodic=True)
            files = {"sine.msh": os.path.join(tmp, "sine.msh")}
        elif kind == "periodic_gmsh4":
            # gmsh 4 (readGmsh, src/mesh.c:743-983): BC codes from the
            # curves' physical tags
            meshgen.write_gmsh4(meshgen.sinewave_mesh(7, periodic=True), os.path.join(tmp, "sine.msh4"))
            ini = meshgen.sinewave_ini("sine", periodic=True).replace("meshFormat = .msh\n",
                                                                     "meshFormat = .msh4\n")
            files = {"sine.msh4": os.path.join(tmp, "sine.msh4")}
        elif kind == "dmr_gmsh4":
            meshgen.write_gmsh4(meshgen.dmr_mesh(30, 8, seed=5), os.path.join(tmp, "dmr.msh4"))
            ini = meshgen.dmr_ini("dmr").replace("meshFormat = .msh\n", "meshFormat = .msh4\n")
            files = {"dmr.msh4": os.path.join(tmp, "dmr.msh4")}
        elif kind == "sine_emc2":
            # EMC2 (readEMC2, src/mesh.c:1004-1139), with interior edges of
            # reference 0 that the reader drops
            meshgen.write_emc2(meshgen.sinewave_mesh(7, periodic=True), os.path.join(tmp, "sine.mesh"),
                               interior_edges=5)
            ini = meshgen.sinewave_ini("sine", periodic=True).replace("meshFormat = .msh\n",
                                                                     "meshFormat = .mesh\n")
            files = {"sine.mesh": os.path.join(tmp, "sine.mesh")}
        elif kind == "riemann_emc2":
            # four quadrant domains from the element references
            meshgen.write_emc2(meshgen.riemann2d_mesh(12), os.path.join(tmp, "rm.mesh"))
            states = [(1.0, 0.1, 0.0, 1.0), (0.5, 0.0, 0.2, 0.4), (0.8, -0.3, 0.0, 0.6), (1.2, 0.0, -0.1, 1.1)]
            ini = meshgen.riemann2d_ini("rm", states).replace("meshFormat = .msh\n", "meshFormat = .mesh\n")
            files = {"rm.mesh": os.path.join(tmp, "rm.mesh")}
        else:
            ini = meshgen.sinewave_ini(None, n=9, periodic=True)
        case = cc.CaseData.from_text(ini, tmp)
        d = refdump.run_ref(ini, "mesh", files=files)
    M = case.mesh()
    if kind.startswith("periodic"):
        assert M["n_bc"] == 0 and M["n_faces"] == len(d["face_sides"]) // 4
    hs = d["hs_geo"].reshape(-1, 12)
    fs = d["face_sides"].reshape(-1, 4)
    fg = d["face_geo"].reshape(-1, 3)
    assert np.array_equal(M["cell_bary"].ravel(), d["elem_bary"])
    assert np.array_equal(M["cell_geo"], d["elem_geo"].reshape(-1, 5)[:, :4])
    assert np.array_equal(M["hs_gp"], hs[:, 0:2]) and np.array_equal(M["hs_w"], hs[:, 2:4])
    assert np.array_equal(np.where(M["hs_nb"] >= 0, M["hs_nb"], -1), d["hs_conn_elem"])
    assert np.array_equal(M["face_cells"][:, 0], fs[:, 1])
    assert np.array_equal(M["face_n"], fg[:, :2]) and np.array_equal(M["face_len"], fg[:, 2])
    assert (M["total_area_q"], M["dx_ref"]) == tuple(d["mesh_scalars"][:2])
    assert np.array_equal(case.prim0().ravel(), d["pvar"])


SINE_RUNS = ["sine_euler_run", "sine_ns_run", "sine_cart_o1_run", "sine_periodic_run",
             "sine_periodic_ns_cart_run"]


@pytest.mark.parametrize("key", SINE_RUNS)
def test_oracle_error_norms_match_reference(ref_small, key):
    # calcErrors restated on the reference's final state: its printed norms
    # (%7.5e) and, at full precision, the same sums formed from the
    # gradients the reference reconstructed for them
    spec = CASES.run_cases()[key]
    info = ref_small[f"{key}/info"]
    prim = ref_small[f"{key}/pvar"].reshape(-1, 4)
    with tempfile.TemporaryDirectory() as tmp:
        case, _, _ = CASES.load_case(spec, tmp)
        assert case.c.params.source_func == 1 and case.c.params.exact_solution == 1
        assert case.c.exact_func == 3
        e = restated.errors(case, prim, float(info[0]))
        if case.c.params.spatial_order == 2:
            _, gr, _, _ = restated.residual(case, prim, float(info[0]), with_extras=True)
            assert np.array_equal(gr[:, :4].ravel(), ref_small[f"{key}/err_u_x"])
            assert np.array_equal(gr[:, 4:].ravel(), ref_small[f"{key}/err_u_y"])
    printed = ref_small[f"{key}/errors_printed"]
    got = np.stack([e["L1"], e["L2"], e["Linf"]])
    np.testing.assert_allclose(got, printed, rtol=6e-6, atol=0)


@pytest.mark.skipif(not refdump.have_ref(), reason="compiled reference not built")
@pytest.mark.parametrize("key", ["sine_euler_bj", "sine_ns_vk"])
def test_oracle_source_term_bit_identical_to_live_reference(key):
    spec = CASES.residual_cases()[key]
    with tempfile.TemporaryDirectory() as tmp:
        case, ini, files = CASES.load_case(spec, tmp)
        prim = CASES.random_state(spec, tmp)
        d = refdump.run_ref(ini, "residual", spec["time"], state=prim, eqn=spec["eqn"], files=files)
        ut = restated.residual(case, prim, spec["time"])
        # the same state without the source term: the source is what differs
        case0 = cc.CaseData.from_text(ini.replace("calcSource = T", "calcSource = F"), tmp)
        ut0 = restated.residual(case0, prim, spec["time"])
    assert np.array_equal(ut.ravel(), d["u_t"])
    assert np.abs(ut - ut0).max() > 1e-3
