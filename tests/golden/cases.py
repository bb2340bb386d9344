"""Small parity cases shared by the fixture generator and the tests.

Each case is a mesh generator (seeded), an ``.ini`` text in the reference's
format and, for residual checks, a seeded random primitive state that makes
every branch of the fluxes and limiters active (densities / pressures in
[0.5, 2], velocities in [-1.5, 1.5], i.e. sub- and supersonic faces mixed).
"""
from __future__ import annotations

import os

import numpy as np

from ccfd_b200 import meshgen

FLUX_IDS = list(range(1, 12))

ZOO_MESH = """meshType = 1
nElemsX = 12
nElemsY = 8
X0 = (/0.0, 0.0/)
Xmax = (/1.0, 0.6/)
nBCsegments = (/3, 1, 2, 1/)
meshBCtype = {b1}
BCstart = 1
BCend = 4
meshBCtype = 301
BCstart = 5
BCend = 8
meshBCtype = 801
BCstart = 9
BCend = 12
meshBCtype = 401
meshBCtype = 501
BCstart = 1
BCend = 6
meshBCtype = 601
BCstart = 7
BCend = 12
meshBCtype = 301
"""

ZOO_BCS = """nBC = 6
BCtype = {b1}
{wall}BCtype = 301
rho = 1.2
mach = 0.6
alpha = 10.0
pressure = 1.1
BCtype = 401
BCtype = 501
rho = 1.0
mach = 0.4
alpha = -5.0
pressure = 1.0
BCtype = 601
BCexactFunc = 4
BCtype = 801
pressure = 0.9
"""

COMMON_TAIL = """icType = 1
nDomains = 1
domainID = 1
rho = 1.0
mach = 0.5
alpha = 30.0
pressure = 1.0
fluxFunction = {flux}
spatialOrder = {order}
limiter = {limiter}
venk_k = 5.0
timeOrder = 2
nRKstages = 3
CFL = 0.5
stationary = F
tEnd = 10.0
maxIter = 100000
fileName = zoo
IOtimeInterval = 10.0
IOiterInterval = 100000000
outputFormat = 3
"""


def zoo_ini(flux=2, order=2, limiter=2, ns=False, mu=0.01):
    b1 = 201 if ns else 101
    wall = "adiabaticWall = T\n" if ns else ""
    head = f"navierStokes = T\nmu = {mu}\nPr = 0.72\n" if ns else ""
    return (head + ZOO_MESH.format(b1=b1) + ZOO_BCS.format(b1=b1, wall=wall)
            + COMMON_TAIL.format(flux=flux, order=order, limiter=limiter))


def _dmr_ini(flux, order, limiter, t_end=0.2):
    s = meshgen.dmr_ini("dmr", flux=flux, limiter=limiter if order == 2 else 1, t_end=t_end)
    return s.replace("spatialOrder = 2", f"spatialOrder = {order}")


def residual_cases() -> dict:
    cases = {}
    for flux in FLUX_IDS:
        for tag, order, lim in (("o1", 1, 1), ("bj", 2, 1), ("vk", 2, 2)):
            cases[f"dmr_f{flux:02d}_{tag}"] = {
                "mesh": ("dmr", 24, 6), "ini": _dmr_ini(flux, order, lim), "eqn": "euler",
                "time": 0.01, "seed": 1000 + 10 * flux + order + lim}
    for tag, order, lim in (("o1", 1, 1), ("bj", 2, 1), ("vk", 2, 2)):
        cases[f"zoo_euler_{tag}"] = {"mesh": None, "ini": zoo_ini(2, order, lim),
                                     "eqn": "euler", "time": 0.02, "seed": 77 + order + lim}
        cases[f"zoo_ns_{tag}"] = {"mesh": None, "ini": zoo_ini(5, order, lim, ns=True),
                                  "eqn": "navierstokes", "time": 0.02, "seed": 88 + order + lim}
    # manufactured sine-wave solution with the source term (triangles and
    # general quads in one mesh)
    cases["sine_euler_bj"] = {"mesh": ("sine", 12), "ini": meshgen.sinewave_ini("sine", order=2, limiter=1),
                              "eqn": "euler", "time": 0.13, "seed": 515}
    cases["sine_ns_vk"] = {"mesh": ("sine", 12),
                           "ini": meshgen.sinewave_ini("sine", order=2, limiter=2, flux=5, navier_stokes=True),
                           "eqn": "navierstokes", "time": 0.37, "seed": 516}
    cases["sine_periodic_vk"] = {"mesh": ("sine_periodic", 12),
                                 "ini": meshgen.sinewave_ini("sine", order=2, limiter=2, flux=5, periodic=True),
                                 "eqn": "euler", "time": 0.21, "seed": 517}
    cases["naca_ns_vk"] = {
        "mesh": ("naca", 32, 12),
        "ini": meshgen.airfoil_ini("naca", navier_stokes=True, reynolds=500.0, implicit=False,
                                   precond=False, cfl=0.5),
        "eqn": "navierstokes", "time": 0.0, "seed": 4242, "mild": True}
    return cases


def run_cases() -> dict:
    return {
        "dmr_hllc_vk_run": {"mesh": ("dmr", 24, 6), "ini": _dmr_ini(5, 2, 2, t_end=0.02),
                            "eqn": "euler", "steps": 0},
        "dmr_roe_bj_run": {"mesh": ("dmr", 24, 6), "ini": _dmr_ini(2, 2, 1, t_end=0.01),
                           "eqn": "euler", "steps": 0},
        "zoo_euler_run": {"mesh": None, "ini": zoo_ini(3, 2, 2).replace("tEnd = 10.0", "tEnd = 0.05"),
                          "eqn": "euler", "steps": 0},
        "zoo_ns_run": {"mesh": None, "ini": zoo_ini(2, 2, 1, ns=True).replace("tEnd = 10.0", "tEnd = 0.02"),
                       "eqn": "navierstokes", "steps": 0},
        # manufactured solution runs ending with the error analysis
        "sine_euler_run": {"mesh": ("sine", 16), "ini": meshgen.sinewave_ini("sine", order=2, limiter=2,
                                                                             t_end=0.2),
                           "eqn": "euler", "steps": 0},
        "sine_ns_run": {"mesh": ("sine", 16), "ini": meshgen.sinewave_ini("sine", order=2, limiter=1, flux=5,
                                                                          navier_stokes=True, t_end=0.2),
                        "eqn": "navierstokes", "steps": 0},
        "sine_periodic_run": {"mesh": ("sine_periodic", 16),
                              "ini": meshgen.sinewave_ini("sine", order=2, limiter=1, periodic=True, t_end=0.2),
                              "eqn": "euler", "steps": 0},
        "sine_periodic_ns_cart_run": {"mesh": None,
                                      "ini": meshgen.sinewave_ini(None, n=16, order=2, limiter=2, flux=3,
                                                                  navier_stokes=True, periodic=True, t_end=0.2),
                                      "eqn": "navierstokes", "steps": 0},
        "sine_cart_o1_run": {"mesh": None, "ini": meshgen.sinewave_ini(None, n=16, order=1, time_order=1,
                                                                       rk_stages=1, t_end=0.2),
                             "eqn": "euler", "steps": 0},
    }


def implicit_cases() -> dict:
    """Short implicit runs on a small NACA 0012 O-grid (32 x 12 quads), where
    the reference's dense Jacobian ((4N)^2 doubles) is still affordable."""
    def ini(ns=False, precond=True, cfl=20.0, kdim=10, steps=4):
        s = meshgen.airfoil_ini("naca", mach=0.5, alpha=2.0, navier_stokes=ns, reynolds=500.0,
                                flux=2, implicit=True, precond=precond, n_kdim=kdim, cfl=cfl,
                                max_iter=steps)
        return s
    return {
        "naca_euler_imp_pc": {"mesh": ("naca", 32, 12, 101), "ini": ini(), "eqn": "euler", "steps": 4},
        "naca_euler_imp_nopc": {"mesh": ("naca", 32, 12, 101), "ini": ini(precond=False, kdim=20),
                                "eqn": "euler", "steps": 4},
        "naca_ns_imp_pc": {"mesh": ("naca", 32, 12), "ini": ini(ns=True, cfl=10.0), "eqn": "navierstokes",
                           "steps": 3},
        # a long run towards the steady state (relative residual 1.7e-2 after
        # 200 steps; the reference's fixed-CFL backward Euler converges
        # slowly, so 1e-8 is out of reach of the dense reference Jacobian)
        "naca_euler_imp_pc_long": {"mesh": ("naca", 32, 12, 101), "ini": ini(steps=200), "eqn": "euler",
                                   "steps": 200},
        # steady run to a relative residual of 0.3 (relAbortResidual; the
        # reference driver stops at the same relative drop)
        "naca_euler_imp_rel": {"mesh": ("naca", 32, 12, 101),
                               "ini": meshgen.airfoil_ini("naca", mach=0.5, alpha=2.0, flux=2, implicit=True,
                                                          precond=True, n_kdim=10, cfl=20.0, max_iter=200,
                                                          rel_res=0.3),
                               "eqn": "euler", "steps": 0, "rel_abort": 0.3},
        # time-accurate implicit steps of the sine wave on a periodic mesh
        # (with the source term or the exact-solution boundary the
        # reference's Newton iteration stalls at a relative residual of
        # 0.5-0.9 in its first step, at CFL 0.5 to 4)
        "sine_periodic_imp": {"mesh": ("sine_periodic", 8),
                              "ini": meshgen.sinewave_ini("sine", order=2, limiter=2, periodic=True, implicit=True,
                                                          cfl=4.0, t_end=1.0, source=False),
                              "eqn": "euler", "steps": 5},
    }


def make_mesh(spec):
    kind = spec.get("mesh")
    if kind is None:
        return None
    if kind[0] == "dmr":
        return "dmr", meshgen.dmr_mesh(kind[1], kind[2])
    if kind[0] == "sine":
        return "sine", meshgen.sinewave_mesh(kind[1])
    if kind[0] == "sine_periodic":
        return "sine", meshgen.sinewave_mesh(kind[1], periodic=True)
    if kind[0] == "naca":
        wall = kind[3] if len(kind) > 3 else 201
        return "naca", meshgen.naca_ogrid(0.0, 0.0, 0.12, kind[1], kind[2], r_far=5.0, h0=1e-2,
                                          wall_code=wall)
    raise ValueError(kind)


def materialise(spec, tmpdir):
    """Write the case's mesh into tmpdir; returns (ini text, {name: path})."""
    mm = make_mesh(spec)
    if mm is None:
        return spec["ini"], {}
    name, mesh = mm
    path = os.path.join(tmpdir, name + ".msh")
    mesh.write_gmsh(path)
    return spec["ini"], {name + ".msh": path}


def random_state(spec, tmpdir):
    """Seeded random primitive state for the case's cell count."""
    import ccfd_b200 as cc
    ini, files = materialise(spec, tmpdir)
    case = cc.CaseData.from_text(ini, tmpdir)
    rng = np.random.Generator(np.random.PCG64(spec["seed"]))
    n = case.n_cells
    if spec.get("mild"):
        # +-10 % around the initial state (far-field boundaries stay
        # physical: the characteristic ghost state of wild states overflows)
        return case.prim0() * (1.0 + 0.1 * rng.uniform(-1.0, 1.0, (n, 4)))
    prim = np.empty((n, 4))
    prim[:, 0] = rng.uniform(0.5, 2.0, n)
    prim[:, 1] = rng.uniform(-1.5, 1.5, n)
    prim[:, 2] = rng.uniform(-1.5, 1.5, n)
    prim[:, 3] = rng.uniform(0.5, 2.0, n)
    return prim


def load_case(spec, tmpdir):
    import ccfd_b200 as cc
    ini, files = materialise(spec, tmpdir)
    return cc.CaseData.from_text(ini, tmpdir), ini, files


def output_cases() -> dict:
    """Final-solution files of dataOutput (src/output.c:334-398) in the
    formats that are built: curve and CSV, transient (time in the name) and
    stationary (iteration in the name), with the exact-solution file."""
    sod = meshgen.sod_ini(50, 2, t_end=0.1)
    return {
        "out_sod_curve": {"ini": sod.replace("outputFormat = 3", "outputFormat = 2\nexactSolution = T"),
                          "eqn": "euler"},
        "out_sod_stationary_csv": {"ini": sod.replace("stationary = F", "stationary = T")
                                   .replace("maxIter = 1000000", "maxIter = 12")
                                   .replace("outputFormat = 3", "outputFormat = 3\nexactSolution = T"),
                                   "eqn": "euler"},
        "out_sine_periodic_csv": {"ini": meshgen.sinewave_ini(None, n=8, periodic=True, t_end=0.1),
                                  "eqn": "euler"},
        # residual file with CL / CD (and the CL / CD gnuplot script)
        "out_naca_wing_imp": {"mesh": ("naca", 32, 12, 101),
                              "ini": meshgen.airfoil_ini("naca", mach=0.5, alpha=2.0, flux=2, implicit=True,
                                                         precond=True, n_kdim=10, cfl=20.0, max_iter=3),
                              "eqn": "euler"},
    }


# Record points (nRecordPoints / pointCoords) are not among the output cases:
# the reference crashes on them (initRecordPoints stores into
# recordPoint.elem / recordPoint.ioFile, src/analyze.c:72 and 87, which are
# never allocated), so no reference file exists to compare with.
RECORD_POINTS = "nRecordPoints = 3\npointCoords = (/0.47, 0.02/)\npointCoords = (/0.51, 0.04/)\n" \
                "pointCoords = (/0.905, 0.013/)\n"
