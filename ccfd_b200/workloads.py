"""Synthetic cases of the batched and served workloads (meshes in gmsh 2.2,
cases in the reference's .ini format), drawn from seeded PCG64 streams.

* Batched airfoils: NACA 4-digit airfoils with camber m ~ U[0, 0.06],
  camber position p ~ U[0.2, 0.6], thickness t ~ U[0.08, 0.18],
  Mach ~ U[0.3, 0.75], angle of attack ~ U[-2, 4] degrees, O-grids of
  (128..512) x (64..256) quads; steady Euler, Roe flux, second order with the
  Venkatakrishnan limiter, implicit backward Euler with JFNK-GMRES (Krylov
  dimension 30) and the LU-SGS preconditioner.
* Served stream: 2-D Riemann problems (four random quadrant states,
  rho, p ~ U[0.1, 2], u, v ~ U[-1, 1], HLLC, 200 RK3 steps), cylinder-wake
  Navier-Stokes windows (Re 100, Mach 0.2, 1000 RK3 steps) and airfoils of
  the batched distribution, in random order.
"""
from __future__ import annotations

import os

import numpy as np

from . import meshgen


def airfoil_specs(n: int, seed: int = 20260004) -> list[dict]:
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for _ in range(n):
        out.append({"m": rng.uniform(0.0, 0.06), "p": rng.uniform(0.2, 0.6),
                    "t": rng.uniform(0.08, 0.18), "mach": rng.uniform(0.3, 0.75),
                    "alpha": rng.uniform(-2.0, 4.0), "ni": int(rng.integers(128, 513)),
                    "nj": int(rng.integers(64, 257))})
    return out


def airfoil_ini(spec: dict, mesh_name: str, cfl: float, precision: int = 0) -> str:
    ini = meshgen.airfoil_ini(mesh_name, mach=spec["mach"], alpha=spec["alpha"], cfl=cfl,
                              max_iter=100000, precision=precision)
    # the reference's preconditioned examples: nNewtonIter 55, epsNewton 0.1
    return ini.replace("nNewtonIter = 100", "nNewtonIter = 55").replace("epsNewton = 0.001",
                                                                          "epsNewton = 0.1")


def airfoil_case(spec: dict, tmpdir: str, name: str, cfl: float = 1.0, h0: float = 2e-3,
                 precision: int = 0):
    import ccfd_b200 as cc
    path = os.path.join(tmpdir, name + ".msh")
    if not os.path.exists(path):
        meshgen.naca_ogrid(spec["m"], spec["p"], spec["t"], spec["ni"], spec["nj"], h0=h0,
                           wall_code=101).write_gmsh(path)
    return cc.CaseData.from_text(airfoil_ini(spec, name, cfl, precision), tmpdir)


def stream_specs(n: int, seed: int = 20260005, riemann_n=(256, 2048), cylinder_cells=(50_000, 400_000),
                 airfoil_steps: int = 5) -> list[dict]:
    """Request mix of the served stream (kinds in equal shares, random order)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    af = airfoil_specs(n, seed + 1)
    out = []
    for k in range(n):
        kind = ("riemann", "cylinder", "airfoil")[int(rng.integers(0, 3))]
        if kind == "riemann":
            states = [(rng.uniform(0.1, 2.0), rng.uniform(-1.0, 1.0), rng.uniform(-1.0, 1.0),
                       rng.uniform(0.1, 2.0)) for _ in range(4)]
            nn = int(rng.integers(riemann_n[0], riemann_n[1] + 1))
            out.append({"kind": kind, "n": nn, "states": states, "steps": 200})
        elif kind == "cylinder":
            cells = int(rng.integers(cylinder_cells[0], cylinder_cells[1] + 1))
            n_theta = int(round(np.sqrt(cells)))       # cells = 2 n_theta n_r
            n_r = max(8, cells // (2 * n_theta))
            out.append({"kind": kind, "n_theta": n_theta, "n_r": n_r, "steps": 1000})
        else:
            out.append({"kind": kind, "airfoil": af[k], "steps": airfoil_steps})
    return out


def stream_case(req: dict, tmpdir: str, name: str):
    import ccfd_b200 as cc
    if req["kind"] == "riemann":
        meshgen.riemann2d_mesh(req["n"]).write_gmsh(os.path.join(tmpdir, name + ".msh"))
        return cc.CaseData.from_text(meshgen.riemann2d_ini(name, req["states"], steps=req["steps"]), tmpdir)
    if req["kind"] == "cylinder":
        meshgen.cylinder_mesh(req["n_theta"], req["n_r"]).write_gmsh(os.path.join(tmpdir, name + ".msh"))
        return cc.CaseData.from_text(meshgen.cylinder_ini(name, steps=req["steps"]), tmpdir)
    return airfoil_case(req["airfoil"], tmpdir, name)


def _main(argv=None) -> int:
    """python -m ccfd_b200.workloads airfoil NI NJ STEPS [CFL]: one steady
    airfoil (m 0.02, p 0.4, t 0.12, Mach 0.5, 1 degree) through the implicit
    solver on device 0; prints cells, steps, Newton / GMRES iterations and
    device milliseconds.
    python -m ccfd_b200.workloads batch N STEPS [CFL] [PRECISION]: the first
    N airfoils of the batched distribution stepped together in one batch
    (PRECISION 0: FP64, 1: mixed); prints the total cells, Newton / GMRES
    iterations and batch device milliseconds."""
    import sys
    import tempfile

    import ccfd_b200 as cc
    args = sys.argv[1:] if argv is None else argv
    if len(args) >= 3 and args[0] == "batch":
        n, steps = int(args[1]), int(args[2])
        cfl = float(args[3]) if len(args) > 3 else 1.0
        prec = int(args[4]) if len(args) > 4 else 0
        cc.set_device(0)
        with tempfile.TemporaryDirectory() as tmp:
            cases = [airfoil_case(sp, tmp, f"af{k}", cfl=cfl, precision=prec)
                     for k, sp in enumerate(airfoil_specs(n))]
        b = cc.Batch(0)
        members = [cc.Solver(c) for c in cases]
        for s in members:
            b.add(s, steps)
        b.step(steps)
        reps = [b.report(s) for s in members]
        print(sum(c.n_cells for c in cases), sum(r["newton_iterations"] for r in reps),
              sum(r["gmres_iterations"] for r in reps), f"{reps[0]['device_ms']:.3f}")
        b.close()
        return 0
    if len(args) < 4 or args[0] != "airfoil":
        print(_main.__doc__)
        return 2
    ni, nj, steps = int(args[1]), int(args[2]), int(args[3])
    cfl = float(args[4]) if len(args) > 4 else 10.0
    spec = {"m": 0.02, "p": 0.4, "t": 0.12, "mach": 0.5, "alpha": 1.0, "ni": ni, "nj": nj}
    cc.set_device(0)
    with tempfile.TemporaryDirectory() as tmp:
        case = airfoil_case(spec, tmp, "af", cfl=cfl)
    s = cc.Solver(case)
    rep = s.run(steps)
    s.close()
    print(case.n_cells, rep["iterations"], rep["newton_iterations"], rep["gmres_iterations"],
          f"{rep['device_ms']:.3f}")
    return 0


if __name__ == "__main__":
    raise SystemExit(_main())
