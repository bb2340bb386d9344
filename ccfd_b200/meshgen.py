"""Synthetic meshes and ``.ini`` cases for the benchmark configurations.

Meshes are produced as raw arrays (nodes, triangles, quads, BC edges) and
written as gmsh 2.2 ASCII -- the format the reference reads
(src/mesh.c:498-742) -- so the reference solver and this library read
byte-identical input.  All randomness uses numpy's PCG64 generator with the
seed stated per function.

Physical-group conventions of the reference's gmsh reader: a line element
whose physical group is > 100 is a boundary edge with that BC code
(type * 100 + id); triangles / quads carry their physical group as the
initial-condition domain.
"""
from __future__ import annotations

import ctypes as C
import math
import os

import numpy as np


class RawMesh:
    def __init__(self, nodes, tria=None, quad=None, bc=None):
        self.nodes = np.ascontiguousarray(nodes, dtype=np.float64).reshape(-1, 2)
        self.tria = np.ascontiguousarray(tria if tria is not None else np.zeros((0, 4)),
                                         dtype=np.int64).reshape(-1, 4)
        self.quad = np.ascontiguousarray(quad if quad is not None else np.zeros((0, 5)),
                                         dtype=np.int64).reshape(-1, 5)
        self.bc = np.ascontiguousarray(bc if bc is not None else np.zeros((0, 3)),
                                       dtype=np.int64).reshape(-1, 3)

    @property
    def n_cells(self) -> int:
        return len(self.tria) + len(self.quad)

    def write_gmsh(self, path: str) -> str:
        """Write the mesh as gmsh 2.2 ASCII through the library's writer
        (``ccfd_write_gmsh2``)."""
        from . import _native as N
        lp = lambda a: a.ctypes.data_as(C.POINTER(C.c_long))
        st = N.lib.ccfd_write_gmsh2(os.fsencode(path),
                                    self.nodes.ctypes.data_as(C.POINTER(C.c_double)),
                                    len(self.nodes), lp(self.tria), len(self.tria),
                                    lp(self.quad), len(self.quad), lp(self.bc), len(self.bc))
        if st != 0:
            raise OSError(f"writing {path} failed ({st})")
        return path

    def write_gmsh_text(self, path: str) -> str:
        """The same gmsh 2.2 file as ``write_gmsh``, byte for byte, written
        in Python: for callers that must not load the native library (the
        timed reference arm of the benchmark reads its mesh from here).
        The module has no import of the package, so it can be loaded by
        file path on its own."""
        out = ["$MeshFormat\n2.2 0 8\n$EndMeshFormat\n$Nodes\n%d\n" % len(self.nodes)]
        out += ["%d %.17g %.17g 0\n" % (i + 1, x, y) for i, (x, y) in enumerate(self.nodes.tolist())]
        out.append("$EndNodes\n$Elements\n%d\n" % (len(self.bc) + len(self.tria) + len(self.quad)))
        k = 1
        for a, b, c in self.bc.tolist():
            out.append("%d 1 2 %d %d %d %d\n" % (k, c, c, a + 1, b + 1))
            k += 1
        for a, b, c, dom in self.tria.tolist():
            out.append("%d 2 2 %d %d %d %d %d\n" % (k, dom, dom, a + 1, b + 1, c + 1))
            k += 1
        for a, b, c, d, dom in self.quad.tolist():
            out.append("%d 3 2 %d %d %d %d %d %d\n" % (k, dom, dom, a + 1, b + 1, c + 1, d + 1))
            k += 1
        out.append("$EndElements\n")
        with open(path, "w") as f:
            f.write("".join(out))
        return path

    @property
    def n_faces(self) -> int:
        """Unique faces of the mesh: every interior edge is shared by two
        cells, every boundary edge belongs to one."""
        return (3 * len(self.tria) + 4 * len(self.quad) + len(self.bc)) // 2


def write_gmsh4(mesh: "RawMesh", path: str) -> str:
    """Write a mesh as gmsh 4.1 ASCII in the layout the reference's gmsh 4
    reader expects (src/mesh.c:743-983): one curve entity per boundary code
    with that code as its physical tag, the boundary line blocks first and
    in the same order, then one triangle and one quadrilateral block (the
    reference gives cells domain 1 in this format)."""
    codes = sorted(set(int(c) for c in mesh.bc[:, 2]))
    nv = len(mesh.nodes)
    blocks = [(1, k + 1, 1, mesh.bc[mesh.bc[:, 2] == c][:, :2]) for k, c in enumerate(codes)]
    if len(mesh.tria):
        blocks.append((2, 1, 2, mesh.tria[:, :3]))
    if len(mesh.quad):
        blocks.append((2, 1, 3, mesh.quad[:, :4]))
    n_el = sum(len(b[3]) for b in blocks)
    out = ["$MeshFormat", "4.1 0 8", "$EndMeshFormat", "$Entities", f"0 {len(codes)} 1 0"]
    for k, c in enumerate(codes):
        out.append(f"{k + 1} 0 0 0 0 0 0 1 {c} 0")
    out.append("1 0 0 0 0 0 0 0 0")
    out += ["$EndEntities", "$Nodes", f"1 {nv} 1 {nv}", f"2 1 0 {nv}"]
    out += [str(i + 1) for i in range(nv)]
    out += [f"{x!r} {y!r} 0" for x, y in mesh.nodes.tolist()]
    out += ["$EndNodes", "$Elements", f"{len(blocks)} {n_el} 1 {n_el}"]
    tag = 1
    for dim, ent, typ, conn in blocks:
        out.append(f"{dim} {ent} {typ} {len(conn)}")
        for row in conn.tolist():
            out.append(" ".join([str(tag)] + [str(v + 1) for v in row]))
            tag += 1
    out += ["$EndElements", ""]
    with open(path, "w") as f:
        f.write("\n".join(out))
    return path


def write_emc2(mesh: "RawMesh", path: str, interior_edges: int = 0) -> str:
    """Write a mesh in the EMC2 format the reference reads (readEMC2,
    src/mesh.c:1004-1139): boundary edges carry their BC code, elements
    their domain; ``interior_edges`` edges of the first triangles are added
    with reference 0 (not boundary edges, dropped by the reader)."""
    out = ["MeshVersionFormatted 1", "", "Dimension 2", "", "Vertices", str(len(mesh.nodes))]
    out += [f"{x!r} {y!r} 0" for x, y in mesh.nodes.tolist()]
    extra = [(int(t[0]), int(t[1])) for t in mesh.tria[:interior_edges]]
    out += ["", "Edges", str(len(mesh.bc) + len(extra))]
    out += [f"{a + 1} {b + 1} {c}" for a, b, c in mesh.bc.tolist()]
    out += [f"{a + 1} {b + 1} 0" for a, b in extra]
    if len(mesh.tria):
        out += ["", "Triangles", str(len(mesh.tria))]
        out += [" ".join(str(v + 1) for v in row[:3]) + f" {row[3]}" for row in mesh.tria.tolist()]
    if len(mesh.quad):
        out += ["", "Quadrangles", str(len(mesh.quad))]
        out += [" ".join(str(v + 1) for v in row[:4]) + f" {row[4]}" for row in mesh.quad.tolist()]
    out += ["", "End", ""]
    with open(path, "w") as f:
        f.write("\n".join(out))
    return path


def _grid_nodes(nx, ny, x0, x1, y0, y1):
    xs = np.linspace(x0, x1, nx + 1)
    ys = np.linspace(y0, y1, ny + 1)
    X, Y = np.meshgrid(xs, ys)  # row-major in j
    return np.stack([X.ravel(), Y.ravel()], axis=1)


def _quad_conn(nx, ny):
    j, i = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
    a = (j * (nx + 1) + i).ravel()
    return a, a + 1, a + 1 + (nx + 1), a + (nx + 1)


def dmr_mesh(nx: int = 1000, ny: int = 250, jitter: float = 0.2,
             seed: int = 20260001) -> RawMesh:
    """Double Mach reflection domain [0,4]x[0,1]: nx*ny quads, each split
    along its (i,j)-(i+1,j+1) diagonal into two triangles; interior nodes are
    moved by U(-jitter, jitter) * (dx, dy) (PCG64, ``seed``), boundary nodes
    stay fixed.  BCs: bottom faces with midpoint x < 1/6 -> 401 (outflow),
    others -> 101 (slip wall); right -> 401; top and left -> 601 (exact DMR
    solution)."""
    nodes = _grid_nodes(nx, ny, 0.0, 4.0, 0.0, 1.0)
    rng = np.random.Generator(np.random.PCG64(seed))
    dx, dy = 4.0 / nx, 1.0 / ny
    jj, ii = np.meshgrid(np.arange(ny + 1), np.arange(nx + 1), indexing="ij")
    interior = ((ii > 0) & (ii < nx) & (jj > 0) & (jj < ny)).ravel()
    d = rng.uniform(-jitter, jitter, size=(int(interior.sum()), 2))
    nodes[interior, 0] += d[:, 0] * dx
    nodes[interior, 1] += d[:, 1] * dy
    a, b, c, dd = _quad_conn(nx, ny)
    t1 = np.stack([a, b, c, np.ones_like(a)], axis=1)
    t2 = np.stack([a, c, dd, np.ones_like(a)], axis=1)
    tria = np.empty((2 * len(a), 4), dtype=np.int64)
    tria[0::2] = t1
    tria[1::2] = t2
    bc = []
    for i in range(nx):  # bottom
        xm = 0.5 * (nodes[i, 0] + nodes[i + 1, 0])
        bc.append((i, i + 1, 401 if xm < 1.0 / 6.0 else 101))
    for j in range(ny):  # right
        bc.append(((j + 1) * (nx + 1) - 1, (j + 2) * (nx + 1) - 1, 401))
    for i in range(nx):  # top
        k = ny * (nx + 1) + i
        bc.append((k, k + 1, 601))
    for j in range(ny):  # left
        bc.append((j * (nx + 1), (j + 1) * (nx + 1), 601))
    return RawMesh(nodes, tria=tria, bc=np.array(bc))


def dmr_ini(mesh_file: str, flux: int = 5, limiter: int = 2, venk_k: float = 5.0,
            cfl: float = 0.8, t_end: float = 0.2, precision: int = 0,
            max_iter: int = 1000000) -> str:
    base = mesh_file[:-4] if mesh_file.endswith(".msh") else mesh_file
    return f"""! double Mach reflection on a jittered triangle mesh
meshType = 0
meshFormat = .msh
meshFile = {base}
nBC = 3
BCtype = 101
BCtype = 401
BCtype = 601
BCexactFunc = 4
icType = 2
exactFunc = 4
fluxFunction = {flux}
spatialOrder = 2
limiter = {limiter}
venk_k = {venk_k}
timeOrder = 2
nRKstages = 3
CFL = {cfl}
stationary = F
tEnd = {t_end}
maxIter = {max_iter}
fileName = dmr
IOtimeInterval = {t_end}
IOiterInterval = 100000000
outputFormat = 3
precision = {precision}
"""


def sod_ini(nx: int = 400, ny: int = 20, t_end: float = 0.2, flux: int = 2,
            order: int = 2, limiter: int = 1, cfl: float = 0.5) -> str:
    """Sod shock tube [0,1]x[0,0.05] (Cartesian generator of the reference)."""
    return f"""! Sod shock tube
meshType = 1
nElemsX = {nx}
nElemsY = {ny}
X0 = (/0.0, 0.0/)
Xmax = (/1.0, 0.05/)
nBCsegments = (/1, 1, 1, 1/)
meshBCtype = 101
meshBCtype = 401
meshBCtype = 101
meshBCtype = 401
icType = 2
exactFunc = 5
RP_1D_interface = 0.5
StateLeft = (/1.0, 0.0, 0.0, 1.0/)
StateRight = (/0.125, 0.0, 0.0, 0.1/)
nBC = 2
BCtype = 101
BCtype = 401
timeStep1D = F
stationary = F
fluxFunction = {flux}
spatialOrder = {order}
limiter = {limiter}
timeOrder = 2
nRKstages = 3
CFL = {cfl}
fileName = sod
tEnd = {t_end}
maxIter = 1000000
IOtimeInterval = {t_end}
IOiterInterval = 100000000
outputFormat = 3
"""


def sinewave_mesh(n: int, jitter: float = 0.15, seed: int = 20260005,
                  periodic: bool = False) -> RawMesh:
    """Square [-1,1]^2 for the manufactured sine-wave solution: n x n cells,
    interior nodes moved by U(-jitter, jitter) * h (PCG64, ``seed``) so that
    the quads are general quadrilaterals, every cell whose (i + j) is odd
    split along its diagonal into two triangles (both quadrature rules in one
    mesh); all boundary faces 601 (exact solution), or with ``periodic``
    the periodic pairs bottom 701 / top 702 and right 711 / left 712."""
    nodes = _grid_nodes(n, n, -1.0, 1.0, -1.0, 1.0)
    rng = np.random.Generator(np.random.PCG64(seed))
    h = 2.0 / n
    jj, ii = np.meshgrid(np.arange(n + 1), np.arange(n + 1), indexing="ij")
    interior = ((ii > 0) & (ii < n) & (jj > 0) & (jj < n)).ravel()
    d = rng.uniform(-jitter, jitter, size=(int(interior.sum()), 2))
    nodes[interior] += d * h
    a, b, c, dd = _quad_conn(n, n)
    j, i = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    odd = ((i + j).ravel() % 2) == 1
    one = np.ones(int((~odd).sum()), dtype=np.int64)
    quad = np.stack([a[~odd], b[~odd], c[~odd], dd[~odd], one], axis=1)
    t1 = np.stack([a[odd], b[odd], c[odd], np.ones_like(a[odd])], axis=1)
    t2 = np.stack([a[odd], c[odd], dd[odd], np.ones_like(a[odd])], axis=1)
    tria = np.concatenate([t1, t2])
    codes = (701, 711, 702, 712) if periodic else (601, 601, 601, 601)
    bc = []
    for k in range(n):
        bc.append((k, k + 1, codes[0]))
        bc.append(((k + 1) * (n + 1) - 1, (k + 2) * (n + 1) - 1, codes[1]))
        bc.append((n * (n + 1) + k, n * (n + 1) + k + 1, codes[2]))
        bc.append((k * (n + 1), (k + 1) * (n + 1), codes[3]))
    return RawMesh(nodes, tria=tria, quad=quad, bc=np.array(bc))


def sinewave_ini(mesh_file: str | None, n: int = 16, order: int = 2, limiter: int = 1,
                 flux: int = 2, navier_stokes: bool = False, mu: float = 0.01,
                 source: bool = True, t_end: float = 0.05, cfl: float = 0.9,
                 time_order: int = 2, rk_stages: int = 3, periodic: bool = False,
                 implicit: bool = False) -> str:
    """Manufactured sine-wave solution (exact function 3 with source
    function 1), the convergence case of the reference's calc/sinewave.
    ``mesh_file`` None: the reference's own Cartesian n x n mesh on
    [-1,1]^2.  ``periodic``: periodic boundaries (pairs 701 / 702 bottom to
    top, 711 / 712 right to left, as in calc/sinewave/sinewave_1D.ini)
    instead of the exact solution.  ``implicit``: backward Euler with
    JFNK-GMRES and LU-SGS (time-accurate, fixed CFL)."""
    codes = ("701", "711", "702", "712") if periodic else ("601",) * 4
    if mesh_file is None:
        mesh = f"""meshType = 1
nElemsX = {n}
nElemsY = {n}
X0 = (/-1.0, -1.0/)
Xmax = (/1.0, 1.0/)
nBCsegments = (/1, 1, 1, 1/)
meshBCtype = {codes[0]}
meshBCtype = {codes[1]}
meshBCtype = {codes[2]}
meshBCtype = {codes[3]}
"""
    else:
        base = mesh_file[:-4] if mesh_file.endswith(".msh") else mesh_file
        mesh = f"meshType = 0\nmeshFormat = .msh\nmeshFile = {base}\n"
    ns = f"navierStokes = T\nmu = {mu}\nPr = 0.72\n" if navier_stokes else ""
    src = "calcSource = T\nsourceFunction = 1\n" if source else "calcSource = F\n"
    if periodic:
        bcs = """nBC = 4
BCtype = 701
connection = (/0.0, 2.0/)
BCtype = 711
connection = (/-2.0, 0.0/)
BCtype = 702
connection = (/0.0, -2.0/)
BCtype = 712
connection = (/2.0, 0.0/)
"""
    else:
        bcs = "nBC = 1\nBCtype = 601\nBCexactFunc = 3\n"
    imp = ("implicit = T\nprecond = T\nnKdim = 10\nnNewtonIter = 100\nepsNewton = 0.001\n"
           "epsGMRES = 0.001\n") if implicit else ""
    return f"""! manufactured sine-wave solution
{ns}{mesh}{bcs}{imp}icType = 2
exactFunc = 3
{src}exactSolution = T
fluxFunction = {flux}
spatialOrder = {order}
limiter = {limiter}
venk_k = 5.0
timeOrder = {time_order}
nRKstages = {rk_stages}
CFL = {cfl}
stationary = F
tEnd = {t_end}
maxIter = 1000000
fileName = sinewave
IOtimeInterval = {t_end}
IOiterInterval = 100000000
outputFormat = 3
"""


def riemann2d_mesh(n: int) -> RawMesh:
    """Unit square, n x n quads, four quadrant domains (physical groups 1..4
    counter-clockwise from the upper right), outflow (401) on all sides."""
    nodes = _grid_nodes(n, n, 0.0, 1.0, 0.0, 1.0)
    a, b, c, d = _quad_conn(n, n)
    j, i = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    right, top = (i.ravel() >= n // 2), (j.ravel() >= n // 2)
    dom = np.where(top, np.where(right, 1, 2), np.where(right, 4, 3))
    quad = np.stack([a, b, c, d, dom], axis=1)
    bc = []
    for k in range(n):
        bc.append((k, k + 1, 401))
        bc.append(((k + 1) * (n + 1) - 1, (k + 2) * (n + 1) - 1, 401))
        bc.append((n * (n + 1) + k, n * (n + 1) + k + 1, 401))
        bc.append((k * (n + 1), (k + 1) * (n + 1), 401))
    return RawMesh(nodes, quad=quad, bc=np.array(bc))


def riemann2d_ini(mesh_file: str, states, steps: int = 200, flux: int = 5,
                  gamma: float = 1.4) -> str:
    """Four-quadrant Riemann problem; ``states`` is 4 x (rho, u, v, p) for
    domains 1..4, encoded as the reference's (rho, mach, alpha, pressure)."""
    base = mesh_file[:-4] if mesh_file.endswith(".msh") else mesh_file
    lines = [f"""! 2-D Riemann problem
meshType = 0
meshFormat = .msh
meshFile = {base}
nBC = 1
BCtype = 401
icType = 1
nDomains = 4"""]
    for k, (r, u, v, p) in enumerate(states):
        c = math.sqrt(gamma * p / r)
        mach = math.hypot(u, v) / c
        alpha = math.degrees(math.atan2(v, u))
        lines.append(f"domainID = {k + 1}\nrho = {r!r}\nmach = {mach!r}\nalpha = {alpha!r}\n"
                     f"pressure = {p!r}")
    lines.append(f"""fluxFunction = {flux}
spatialOrder = 2
limiter = 2
venk_k = 5
timeOrder = 2
nRKstages = 3
CFL = 0.8
stationary = F
tEnd = 1e10
maxIter = {steps}
fileName = riemann
IOtimeInterval = 1e10
IOiterInterval = 100000000
outputFormat = 3
""")
    return "\n".join(lines)


def naca_thickness(x, t):
    """NACA 4-digit half thickness with the closed trailing edge
    (coefficient -0.1036 on x^4)."""
    return 5.0 * t * (0.2969 * np.sqrt(x) - 0.1260 * x - 0.3516 * x**2 + 0.2843 * x**3
                      - 0.1036 * x**4)


def naca_surface(m: float, p: float, t: float, ni: int):
    """ni points around a NACA mpxx airfoil (cosine clustering, closed trailing
    edge), counter-clockwise from the trailing edge over the lower surface."""
    beta = np.linspace(0.0, 2.0 * np.pi, ni, endpoint=False)
    xc = 0.5 * (1.0 + np.cos(beta))          # 1 -> 0 -> 1
    yt = naca_thickness(xc, t)
    if m > 0.0 and p > 0.0:
        yc = np.where(xc < p, m / p**2 * (2 * p * xc - xc**2),
                      m / (1 - p)**2 * ((1 - 2 * p) + 2 * p * xc - xc**2))
        dyc = np.where(xc < p, 2 * m / p**2 * (p - xc), 2 * m / (1 - p)**2 * (p - xc))
    else:
        yc = np.zeros_like(xc)
        dyc = np.zeros_like(xc)
    th = np.arctan(dyc)
    lower = beta < np.pi  # first half: lower surface from TE to LE
    sgn = np.where(lower, -1.0, 1.0)
    x = xc - sgn * yt * np.sin(th)
    y = yc + sgn * yt * np.cos(th)
    return np.stack([x, y], axis=1)


def naca_ogrid(m: float = 0.0, p: float = 0.0, t: float = 0.12, ni: int = 256, nj: int = 128,
               r_far: float = 20.0, h0: float = 1e-4, wall_code: int = 201,
               far_code: int = 501) -> RawMesh:
    """O-grid of ni (circumferential) x nj (radial) quads around a NACA
    4-digit airfoil; far field circle of radius r_far chords about the
    mid-chord; first cell height h0 with geometric radial stretching (ratio
    solved by bisection)."""
    surf = naca_surface(m, p, t, ni)
    centre = np.array([0.5, 0.0])
    ang = np.arctan2(surf[:, 1] - centre[1], surf[:, 0] - centre[0])
    far = centre + r_far * np.stack([np.cos(ang), np.sin(ang)], axis=1)
    dist = np.linalg.norm(far - surf, axis=1).mean()
    lo, hi = 1.0 + 1e-9, 2.0
    for _ in range(200):  # sum_{k<nj} h0 q^k = dist
        q = 0.5 * (lo + hi)
        s = h0 * (q**nj - 1.0) / (q - 1.0)
        lo, hi = (q, hi) if s < dist else (lo, q)
    q = 0.5 * (lo + hi)
    s = np.concatenate([[0.0], np.cumsum(h0 * q ** np.arange(nj))])
    s /= s[-1]
    nodes = np.empty(((nj + 1) * ni, 2))
    for j in range(nj + 1):
        nodes[j * ni:(j + 1) * ni] = surf + s[j] * (far - surf)
    quad = []
    for j in range(nj):
        for i in range(ni):
            i1 = (i + 1) % ni
            quad.append((j * ni + i, j * ni + i1, (j + 1) * ni + i1, (j + 1) * ni + i, 1))
    bc = [(i, (i + 1) % ni, wall_code) for i in range(ni)]
    bc += [(nj * ni + i, nj * ni + (i + 1) % ni, far_code) for i in range(ni)]
    return RawMesh(nodes, quad=np.array(quad), bc=np.array(bc))


def airfoil_ini(mesh_file: str, mach: float = 0.5, alpha: float = 1.0, navier_stokes: bool = False,
                reynolds: float = 5000.0, flux: int = 2, implicit: bool = True,
                precond: bool = True, n_kdim: int = 30, rel_res: float = 1e-8,
                cfl: float = 1e3, max_iter: int = 100000, precision: int = 0,
                wall_code: int | None = None, venk_k: float = 5.0, dfl: float | None = None,
                ser_cfl_max: float | None = None) -> str:
    """Steady airfoil case: far field 501 (characteristic) with rho = p = 1,
    wall 101 (Euler) or 201 (adiabatic no-slip, Navier-Stokes).  ``dfl``:
    viscous time-step number (DFL; the reference's default otherwise);
    ``ser_cfl_max``: CFL ramp by switched evolution relaxation up to this
    value (extension key serCFLmax)."""
    base = mesh_file[:-4] if mesh_file.endswith(".msh") else mesh_file
    wall = wall_code if wall_code is not None else (201 if navier_stokes else 101)
    gam = 1.4
    c_inf = math.sqrt(gam * 1.0 / 1.0)
    mu = 1.0 * mach * c_inf * 1.0 / reynolds
    ns = f"navierStokes = T\nmu = {mu!r}\nPr = 0.72\n" if navier_stokes else ""
    wall_keys = "adiabaticWall = T\n" if wall // 100 == 2 else ""
    return f"""! steady airfoil
meshType = 0
meshFormat = .msh
meshFile = {base}
{ns}nBC = 2
BCtype = {wall}
{wall_keys}BCtype = 501
rho = 1.0
mach = {mach!r}
alpha = {alpha!r}
pressure = 1.0
icType = 1
nDomains = 1
domainID = 1
rho = 1.0
mach = {mach!r}
alpha = {alpha!r}
pressure = 1.0
fluxFunction = {flux}
spatialOrder = 2
limiter = 2
venk_k = {venk_k}
timeOrder = 1
nRKstages = 1
CFL = {cfl}
{f"DFL = {dfl!r}" + chr(10) if dfl is not None else ""}{f"serCFLmax = {ser_cfl_max!r}" + chr(10) if ser_cfl_max else ""}implicit = {'T' if implicit else 'F'}
precond = {'T' if precond else 'F'}
nKdim = {n_kdim}
nNewtonIter = 100
epsNewton = 0.001
epsGMRES = 0.001
stationary = T
abortResidual = 0.0
relAbortResidual = {rel_res}
tEnd = 1e10
maxIter = {max_iter}
fileName = airfoil
IOtimeInterval = 1e10
IOiterInterval = 100000000
outputFormat = 3
calcWing = T
wall_id = {wall}
precision = {precision}
"""


def cylinder_mesh(n_theta: int = 128, n_r: int = 64, r0: float = 0.5, r_far: float = 20.0,
                  wall_code: int = 201, far_code: int = 501) -> RawMesh:
    """Triangle mesh around a circular cylinder of diameter 1: an O-grid with
    geometric radial stretching, each quad split into two triangles."""
    th = np.linspace(0.0, 2.0 * np.pi, n_theta, endpoint=False)
    q = (r_far / r0) ** (1.0 / n_r)
    r = r0 * q ** np.arange(n_r + 1)
    nodes = np.concatenate([np.stack([rj * np.cos(th), rj * np.sin(th)], 1) for rj in r])
    tri = []
    for j in range(n_r):
        for i in range(n_theta):
            i1 = (i + 1) % n_theta
            a, b = j * n_theta + i, j * n_theta + i1
            c, d = (j + 1) * n_theta + i1, (j + 1) * n_theta + i
            tri.append((a, b, c, 1))
            tri.append((a, c, d, 1))
    bc = [(i, (i + 1) % n_theta, wall_code) for i in range(n_theta)]
    bc += [(n_r * n_theta + i, n_r * n_theta + (i + 1) % n_theta, far_code) for i in range(n_theta)]
    return RawMesh(nodes, tria=np.array(tri), bc=np.array(bc))


def cylinder_ini(mesh_file: str, reynolds: float = 100.0, mach: float = 0.2, steps: int = 1000,
                 flux: int = 2, cfl: float = 0.8, wall_code: int = 201) -> str:
    """Viscous flow past the cylinder of cylinder_mesh (diameter 1): far field
    501 with rho = p = 1 at the given Mach number, adiabatic no-slip wall,
    mu from the Reynolds number on the diameter; a window of `steps` RK3
    steps."""
    base = mesh_file[:-4] if mesh_file.endswith(".msh") else mesh_file
    c_inf = math.sqrt(1.4 * 1.0 / 1.0)
    mu = 1.0 * mach * c_inf * 1.0 / reynolds
    return f"""! cylinder wake
navierStokes = T
mu = {mu!r}
Pr = 0.72
meshType = 0
meshFormat = .msh
meshFile = {base}
nBC = 2
BCtype = {wall_code}
adiabaticWall = T
BCtype = 501
rho = 1.0
mach = {mach!r}
alpha = 0.0
pressure = 1.0
icType = 1
nDomains = 1
domainID = 1
rho = 1.0
mach = {mach!r}
alpha = 0.0
pressure = 1.0
fluxFunction = {flux}
spatialOrder = 2
limiter = 2
venk_k = 5.0
timeOrder = 2
nRKstages = 3
CFL = {cfl}
stationary = F
tEnd = 1e10
maxIter = {steps}
fileName = cylinder
IOtimeInterval = 1e10
IOiterInterval = 100000000
outputFormat = 3
"""
