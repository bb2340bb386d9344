"""The benchmark's reference arm: its input is written without this
library (the timed reference process and the Python process that drives it
map no native code of the package), and the Python mesh writer it uses gives
the same bytes as the library's writer."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROBE = r"""
import json, os, sys, tempfile
sys.path.insert(0, {root!r})
import bench
bench.NX, bench.NY = 40, 10
with tempfile.TemporaryDirectory() as tmp:
    ini, path, n, faces = bench.reference_arm_inputs(tmp)
    size = os.path.getsize(path)
maps = open("/proc/self/maps").read()
print(json.dumps({{
    "package_loaded": any(k == "ccfd_b200" or k.startswith("ccfd_b200.") for k in sys.modules),
    "native_mapped": "libccfd_b200" in maps,
    "n": n, "faces": faces, "size": size, "meshfile": "meshFile = dmr" in ini}}))
"""


def test_reference_arm_inputs_load_no_repo_library():
    r = subprocess.run([sys.executable, "-c", PROBE.format(root=ROOT)], capture_output=True,
                       text=True, timeout=300, cwd=ROOT)
    assert r.returncode == 0, r.stderr
    got = json.loads(r.stdout.strip().splitlines()[-1])
    assert not got["package_loaded"]
    assert not got["native_mapped"]
    assert got["n"] == 2 * 40 * 10
    # triangles: every interior edge shared by two cells, boundary edges once
    assert got["faces"] == (3 * 800 + 2 * (40 + 10)) // 2
    assert got["size"] > 0 and got["meshfile"]


@pytest.mark.parametrize("kind", ["dmr", "airfoil", "riemann"])
def test_python_gmsh_writer_equals_library_writer(tmp_path, kind):
    from ccfd_b200 import meshgen
    if kind == "dmr":
        m = meshgen.dmr_mesh(30, 9, seed=11)
    elif kind == "airfoil":
        m = meshgen.naca_ogrid(0.02, 0.4, 0.12, 32, 16)
    else:
        m = meshgen.riemann2d_mesh(12)
    a, b = str(tmp_path / "a.msh"), str(tmp_path / "b.msh")
    m.write_gmsh(a)
    m.write_gmsh_text(b)
    with open(a, "rb") as fa, open(b, "rb") as fb:
        assert fa.read() == fb.read()


def test_host_cpu_reports_physical_cores():
    import bench
    c = bench.host_cpu()
    assert 1 <= c["physical_cores"] <= c["logical_cpus"]
    assert isinstance(c["model"], str) and c["model"]
