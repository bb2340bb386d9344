"""Host layer: library loading / exported C ABI, .ini semantics, mesh errors."""
import ctypes as C
import os
import re
import tempfile

import numpy as np
import pytest

import ccfd_b200 as cc
from ccfd_b200 import _native as N
from ccfd_b200 import meshgen

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_library_exports_every_declared_symbol():
    with open(os.path.join(ROOT, "include", "ccfd_b200.h")) as f:
        hdr = f.read()
    hdr = re.sub(r"/\*.*?\*/", "", hdr, flags=re.S)
    names = set(re.findall(r"\b(ccfd_[a-z0-9_]+)\s*\(", hdr))
    assert len(names) > 20
    lib = C.CDLL(N.LIB_PATH)
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


def test_strerror_covers_statuses():
    for s in range(0, 16):
        assert N.lib.ccfd_strerror(s).decode() != "unknown status"


SOD = """meshType = 1
nElemsX = 10
nElemsY = 2
X0 = (/0.0, 0.0/)
Xmax = (/1.0, 0.1/)
nBCsegments = (/1, 1, 1, 1/)
meshBCtype = 101 ! bottom
MeshBCType = 401
meshbctype = 101
meshBCtype = 401
icType = 2
exactFunc = 5
StateLeft = (/1.0, 0.0, 0.0, 1.0/)
StateRight = (/0.125, 0.0, 0.0, 0.1/)
nBC = 2
BCtype = 101
BCtype = 401
FluxFunction = 3
fileName = t
tEnd = 0.1
IOtimeInterval = 0.1
IOiterInterval = 10
"""


def test_ini_semantics_defaults_and_case_insensitive_keys():
    case = cc.CaseData.from_text(SOD)
    p = case.params
    # defaults of the reference (src/*.c getX(..., "default"))
    assert p.gamma == 1.4 and p.cfl == 0.9 and p.spatial_order == 1
    assert p.n_rk_stages == 1 and p.time_order == 1 and p.stationary == 1
    assert p.flux == 3 and p.max_iter == 100000
    assert case.n_cells == 20
    prim = case.prim0()
    x = case.mesh()["cell_bary"][:, 0]
    assert np.all(prim[x <= 0.5, 0] == 1.0) and np.all(prim[x > 0.5, 0] == 0.125)


def test_ini_missing_mandatory_key_is_an_error():
    bad = SOD.replace("FluxFunction    = 3", "").replace("FluxFunction = 3", "")
    with pytest.raises(cc.CcfdError) as e:
        cc.CaseData.from_text(bad)
    assert e.value.status == 9


def test_ini_repeated_keys_are_consumed_in_order():
    txt = SOD.replace("meshBCtype = 101 ! bottom", "meshBCtype = 401 ! bottom")
    case = cc.CaseData.from_text(txt)
    m = case.mesh()
    codes = np.array([case.c.bc_table[i].type * 100 + case.c.bc_table[i].id for i in m["bc_index"]])
    # bottom (first 10 BC edges) now outflow
    assert (codes == 401).sum() == 10 + 2 + 2


def test_undefined_bc_code_is_a_mesh_error():
    bad = SOD.replace("BCtype = 401", "BCtype = 501\nrho=1\nmach=0.1\nalpha=0\npressure=1")
    with pytest.raises(cc.CcfdError) as e:
        cc.CaseData.from_text(bad)
    assert e.value.status == 10


def test_mesh_build_rejects_inconsistent_boundary(tmp_path):
    m = meshgen.dmr_mesh(4, 2)
    m.bc = m.bc[:-1]  # drop one boundary edge: odd side count
    m.write_gmsh(str(tmp_path / "dmr.msh"))
    with pytest.raises(cc.CcfdError) as e:
        cc.CaseData.from_text(meshgen.dmr_ini("dmr"), str(tmp_path))
    assert e.value.status == 10


def test_gmsh_roundtrip(tmp_path):
    m = meshgen.dmr_mesh(6, 3)
    m.write_gmsh(str(tmp_path / "a.msh"))
    case = cc.CaseData.from_text(meshgen.dmr_ini("a"), str(tmp_path))
    assert case.n_cells == 36
    mm = case.mesh()
    assert mm["n_bc"] == 18 and mm["n_faces"] == (3 * 36 + 18) // 2
    # cell areas sum to the domain area
    assert abs(mm["cell_geo"][:, 0].sum() - 4.0) < 1e-12


def test_source_term_keys_and_quadrature_points():
    # calcSource / sourceFunction (src/equation.c:120-123): the function is
    # mandatory once the source is on; the reference knows function 1 only
    src = SOD + "calcSource = T\nsourceFunction = 1\nexactSolution = T\n"
    case = cc.CaseData.from_text(src)
    assert case.params.source_func == 1 and case.params.exact_solution == 1
    with pytest.raises(cc.CcfdError) as e:
        cc.CaseData.from_text(SOD + "calcSource = T\n")
    assert e.value.status == 9
    with pytest.raises(cc.CcfdError):
        cc.CaseData.from_text(SOD + "calcSource = T\nsourceFunction = 2\n")
    assert cc.CaseData.from_text(SOD).params.source_func == 0
    # fifth quadrature point of a quad: midpoint of its nodes 0 and 2
    # (src/mesh.c:157-160); triangles carry their barycentre
    m = meshgen.sinewave_mesh(4)
    with tempfile.TemporaryDirectory() as tmp:
        m.write_gmsh(os.path.join(tmp, "sine.msh"))
        sc = cc.CaseData.from_text(meshgen.sinewave_ini("sine"), tmp)
        mesh = sc.c.mesh
        n = sc.n_cells
        gp5 = np.ctypeslib.as_array(mesh.cell_gp5, shape=(n * 2,)).reshape(n, 2)
        bary = sc.mesh()["cell_bary"]
        ctype = np.ctypeslib.as_array(mesh.cell_type, shape=(n,))
    assert set(np.unique(ctype)) == {3, 4}
    tri = ctype == 3
    assert np.array_equal(gp5[tri], bary[tri])
    assert np.abs(gp5[~tri] - bary[~tri]).max() > 1e-4  # jittered quads


def test_record_point_location_follows_reference_rule():
    # initRecordPoints (src/analyze.c:43-82): first cell in element order
    # with no edge having the point strictly outside; the edge normal is
    # scaled by sqrt(2 u_x^2), so edges with u_x = 0 (horizontal) exclude
    # nothing.  Restated here with numpy on a Sod Cartesian mesh.
    ini = meshgen.sod_ini(50, 2, t_end=0.1) + "nRecordPoints = 3\npointCoords = (/0.47, 0.02/)\n" \
        "pointCoords = (/0.51, 0.04/)\npointCoords = (/0.905, 0.013/)\n"
    case = cc.CaseData.from_text(ini)
    xy, cells = case.record_points()
    m = case.c.mesh
    n = case.n_cells
    nodes = np.ctypeslib.as_array(m.node_xy, shape=(m.n_nodes * 2,)).reshape(-1, 2)
    en = np.ctypeslib.as_array(m.cell_nodes, shape=(n * 4,)).reshape(n, 4)
    ctype = np.ctypeslib.as_array(m.cell_type, shape=(n,))
    want = []
    with np.errstate(divide="ignore", invalid="ignore"):
        for p in xy:
            for e in range(n):
                t = ctype[e]
                inside = True
                for i in range(t):
                    x1, x2 = nodes[en[e, i]], nodes[en[e, (i + 1) % t]]
                    u = np.array([x2[1] - x1[1], x1[0] - x2[0]])
                    u = u / np.sqrt(u[0] * u[0] + u[0] * u[0])
                    if u[0] * (p[0] - x1[0]) + u[1] * (p[1] - x1[1]) > 0.0:
                        inside = False
                if inside:
                    want.append(e)
                    break
    assert list(cells) == want
    assert np.allclose(xy, [[0.47, 0.02], [0.51, 0.04], [0.905, 0.013]])
    with pytest.raises(cc.CcfdError) as e:
        cc.CaseData.from_text(meshgen.sod_ini(50, 2) + "nRecordPoints = 1\npointCoords = (/1.5, 0.02/)\n")
    assert e.value.status == 10  # "Record Point # is not in Domain"


def test_degenerate_mesh_files_are_errors(tmp_path):
    # a gmsh file without cells, an EMC2 file without vertices and a gmsh 4
    # file without physical curves: mesh errors, no crash
    (tmp_path / "empty.msh").write_text("$MeshFormat\n2.2 0 8\n$EndMeshFormat\n$Nodes\n3\n"
                                        "1 0 0 0\n2 1 0 0\n3 0 1 0\n$EndNodes\n$Elements\n1\n"
                                        "1 1 2 101 101 1 2\n$EndElements\n")
    (tmp_path / "empty.mesh").write_text("MeshVersionFormatted 1\nDimension 2\nEnd\n")
    (tmp_path / "nocurves.msh4").write_text("$MeshFormat\n4.1 0 8\n$EndMeshFormat\n$Entities\n0 0 1 0\n"
                                            "1 0 0 0 0 0 0 0 0\n$EndEntities\n")
    base = meshgen.dmr_ini("empty")
    for fmt, name in ((".msh", "empty"), (".mesh", "empty"), (".msh4", "nocurves")):
        ini = base.replace("meshFormat = .msh\n", f"meshFormat = {fmt}\n").replace(
            "meshFile = empty", f"meshFile = {name}")
        with pytest.raises(cc.CcfdError) as e:
            cc.CaseData.from_text(ini, str(tmp_path))
        assert e.value.status == 10, fmt
