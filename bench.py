"""Benchmark of the residual-and-update path (one JSON line on rank 0).

Workload (one "step" = one explicit time step): double Mach reflection on a
jittered triangle mesh, 1000 x 250 quads split into 500,000 triangles, HLLC
flux, second order with the Venkatakrishnan limiter (K = 5), 3-stage RK,
CFL 0.8, FP64.  Metric unit: cell-updates/s = cells x RK stages x steps / s.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun each rank runs an independent replica on its own GPU (the path
does not shard: replicas only, weak scaling); time is the max over ranks of
the device time measured with CUDA events on the solver's stream.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "served solves/s & p50/p99 vs plain GPU loop @1e-8 res; cell-updates/s vs HBM"
UNIT = "cell-updates/s"
NX, NY = 1000, 250
L2_BYTES = 126 * 1024 * 1024


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "20"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            # the timed region is short: wait for the first sample so that
            # the samples cover it
            t0 = time.perf_counter()
            while not self.lines and time.perf_counter() - t0 < 3.0 and self.proc.poll() is None:
                time.sleep(0.005)
            self.skip = len(self.lines)
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines[getattr(self, "skip", 0):]:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def workload_config(n: int, faces: int, world: int) -> dict:
    """The `config` object of the JSON line (both arms)."""
    return {
        "workload": f"double Mach reflection, {n} jittered triangles ({NX}x{NY} quads "
                    "split, seed 20260001), HLLC, Venkatakrishnan K=5, RK3 (timeOrder 2), "
                    "CFL 0.8, FP64",
        "cells": n, "faces": faces, "rk_stages": 3,
        "parallelism": f"replicas x{world}",
        "l2": "inputs larger than L2 (working set > 126 MB), no flush",
    }


def max_over_ranks(x: float, dist) -> float:
    """The largest value of x over the ranks (the job's time is its slowest
    rank's); a plain return without a process group."""
    if dist is None:
        return float(x)
    import torch
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], device=dev, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(world: int, cells: int, stages: int, steps: int, seconds: float) -> float:
    """Whole-job cell-updates/s of `world` independent replicas that each
    ran `steps` steps of `stages` stages over `cells` cells, timed by the
    slowest rank."""
    return world * cells * stages * steps / seconds


def algorithmic_bytes_per_stage(m: dict, venk: bool) -> int:
    """Compulsory HBM traffic of one residual evaluation + RK stage of the
    fused scheme (gradients and face fluxes never leave the chip), each array
    touched once: per cell the primitive state read (32 B) and written (32),
    the stage-start conservative state read (32), 1/area (8) and, with the
    Venkatakrishnan limiter, eps^2 (8); per half-side the neighbour index
    (4), the face / sign code of the flux sum (4), the least-squares weights
    (16) and the face-midpoint offset (16); per face the normal (16), the
    length (8) and the two cell indices (8)."""
    n, h, f = m["n_cells"], m["n_half_sides"], m["n_faces"]
    per_cell = 32 + 32 + 32 + 8 + (8 if venk else 0)
    return n * per_cell + h * (4 + 4 + 16 + 16) + f * (16 + 8 + 8)


# Algorithmic bytes per residual evaluation and cell of the two-pass
# scheme (gradient pass, then face pass, each array touched once), FP64:
# triangles 356 B (Barth-Jespersen) / 364 B (Venkatakrishnan), quads 408 /
# 416 B.  The roofline's `achieved` uses these per-cell figures.
ROOFLINE_BYTES_PER_CELL = {("tri", False): 356, ("tri", True): 364,
                           ("quad", False): 408, ("quad", True): 416}


def roofline_bytes_per_residual(n_tri: int, n_quad: int, venk: bool) -> int:
    return (n_tri * ROOFLINE_BYTES_PER_CELL[("tri", venk)]
            + n_quad * ROOFLINE_BYTES_PER_CELL[("quad", venk)])


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) per launch of the
# stage kernel on this workload from one ncu capture, valid only for the
# kernel sources whose digest is recorded beside it (STAGE_SOURCES); for
# other sources the line reports no traffic.
STAGE_TRAFFIC = {"bytes": 149.260e6 + 8.613e6,
                 "sha256": "c4f694ad24ef324a"}
STAGE_SOURCES = ("ccfd_b200/csrc/stage_impl.cuh", "ccfd_b200/csrc/physics.cuh",
                 "ccfd_b200/csrc/kernels.cuh", "ccfd_b200/csrc/stage_flux.inc",
                 "ccfd_b200/csrc/stage_f05.cu", "ccfd_b200/csrc/tiles.cpp")


def stage_sources_digest() -> str:
    import hashlib
    h = hashlib.sha256()
    for rel in STAGE_SOURCES:
        with open(os.path.join(ROOT, rel), "rb") as f:
            h.update(f.read())
    return h.hexdigest()[:16]


def stage_traffic():
    """(bytes, note): the recorded ncu traffic if it was measured on the
    current stage-kernel sources, else (None, why)."""
    dig = stage_sources_digest()
    if (NX, NY) != (1000, 250):
        return None, "recorded for the 1000x250 workload only"
    if STAGE_TRAFFIC["sha256"] != dig:
        return None, f"no ncu capture of this kernel revision (sources {dig})"
    return STAGE_TRAFFIC["bytes"], f"ncu dram__bytes_read.sum + dram__bytes_write.sum, sources {dig}"


def make_case(tmpdir: str, precision: int = 0):
    import ccfd_b200 as cc
    from ccfd_b200 import meshgen
    path = os.path.join(tmpdir, "dmr.msh")
    if not os.path.exists(path):
        meshgen.dmr_mesh(NX, NY).write_gmsh(path)
    ini = meshgen.dmr_ini("dmr", precision=precision)
    return cc.CaseData.from_text(ini, tmpdir), ini, path


def run_mixed(tmpdir: str, steps: int, warmup: int, prim_fp64, nrk: int, bytes_stage: int,
              oracle_steps: int = 0):
    """The same workload with FP32 reconstruction / face fluxes and FP64
    accumulation and state: throughput, stage-kernel time and the state's
    deviation from the FP64 run after the same steps."""
    import ccfd_b200 as cc
    case, _, _ = make_case(tmpdir, precision=1)
    n = case.n_cells
    s = cc.Solver(case, reorder=True)
    s.set_profiling(True)
    s.run(warmup)
    s.profile(reset=True)
    rep = s.run(steps)
    res_ms, res_cnt = s.profile(reset=True)
    s.set_profiling(False)
    prim = s.get_state()
    s.close()
    done = rep["iterations"] - warmup
    avg = res_ms / max(res_cnt, 1)
    scale = np.abs(prim_fp64).max(axis=0)
    d = np.abs(prim - prim_fp64) / scale
    out = {"value": n * nrk * done / (rep["device_ms"] / 1e3), "unit": UNIT,
           "ms_per_step": rep["device_ms"] / max(done, 1), "dtype": "f32 flux / f64 accumulation",
           "stage_avg_ms": avg, "stage_achieved_gbs": bytes_stage / (avg / 1e3) / 1e9,
           "state_vs_fp64": {"l1": float(d.mean()), "linf": float(d.max()),
                             "after_steps": int(rep["iterations"]),
                             "norm": "per variable, relative to max|U_fp64|"}}
    if oracle_steps > 0:
        # against the FP64 oracle (C restatement, pinned bit for bit to the
        # compiled reference) after the same steps from the initial state
        from oracle import restated
        s = cc.Solver(case, reorder=True)
        s.run(oracle_steps)
        pm = s.get_state()
        s.close()
        po, _ = restated.run_explicit(case, nsteps=oracle_steps)
        e = np.abs(pm - po) / np.abs(po).max(axis=0)
        out["state_vs_oracle"] = {"l1": float(e.mean()), "linf": float(e.max()), "after_steps": oracle_steps,
                                  "norm": "per variable, relative to max|U_oracle|"}
    return out


def run_sod_c1(threads: int) -> dict:
    """The small plain configuration: Sod shock tube, 400 x 20 quads, Roe,
    second order Barth-Jespersen, RK3, CFL 0.5, to t_end = 0.2: device time
    of the run against the compiled reference on the host cores (its own
    time loop), and the final state's deviation from it."""
    import ccfd_b200 as cc
    from ccfd_b200 import meshgen
    from oracle import refdump
    ini = meshgen.sod_ini(400, 20, t_end=0.2, flux=2, order=2, limiter=1, cfl=0.5)
    case = cc.CaseData.from_text(ini)
    s = cc.Solver(case, reorder=True)
    s.run(3)  # warm-up (graph capture); the timed run starts again from t = 0
    s.close()
    s = cc.Solver(case, reorder=True)
    rep = s.run(0)
    prim = s.get_state()
    s.close()
    n, steps = case.n_cells, int(rep["iterations"])
    out = {"workload": "Sod shock tube, 400x20 quads (8,000 cells), Roe, 2nd order Barth-Jespersen, RK3, "
                       "CFL 0.5, t_end 0.2, FP64",
           "cells": n, "steps": steps, "gpu_ms": rep["device_ms"],
           "gpu_cell_updates_per_s": n * 3 * steps / (rep["device_ms"] / 1e3),
           "note": "8,000 cells fit in L2: launch-bound, not a roofline workload"}
    if refdump.have_ref("euler", fast=True):
        os.environ["OMP_PROC_BIND"] = "close"
        os.environ["OMP_PLACES"] = "cores"
        d = refdump.run_ref(ini, "run", 0, fast=True, threads=threads)
        wall = float(d["step_wall"][-1])
        ref = d["pvar"].reshape(-1, 4)
        out["reference"] = {"wall_s": wall, "cell_updates_per_s": n * 3 * int(d["run_info"][1]) / wall,
                            "threads": threads, "steps": int(d["run_info"][1])}
        out["state_vs_reference_linf"] = float(np.abs(prim - ref).max())
    return out


def run_airfoil_c3(steps: int = 3) -> dict:
    """The implicit Navier-Stokes configuration's mesh and physics (NACA
    0012 O-grid 256 x 128 quads, first cell 1e-4 chord, far field 20 chords,
    Mach 0.5, Re 5,000, AoA 1 deg, Roe, VK K=5, JFNK-GMRES Krylov 30 with
    LU-SGS, CFL 10): `steps` implicit steps on the GPU against the restated
    oracle (block-sparse buildMatrix / LU-SGS; the reference's dense Jacobian
    would need 137 GB) timed on one host core."""
    import ccfd_b200 as cc
    from ccfd_b200 import meshgen
    from oracle import restated
    with tempfile.TemporaryDirectory() as tmp:
        meshgen.naca_ogrid(0.0, 0.0, 0.12, 256, 128, r_far=20.0, h0=1e-4, wall_code=201).write_gmsh(
            os.path.join(tmp, "c3.msh"))
        ini = meshgen.airfoil_ini("c3", mach=0.5, alpha=1.0, navier_stokes=True, reynolds=5000.0, flux=2,
                                  implicit=True, precond=True, n_kdim=30, cfl=10.0, max_iter=100)
        case = cc.CaseData.from_text(ini, tmp)
    s = cc.Solver(case, reorder=True)
    s.run(1)  # warm-up (set-up of the lockstep set)
    s.close()
    s = cc.Solver(case, reorder=True)
    rep = s.run(steps)
    prim = s.get_state()
    s.close()
    t0 = time.perf_counter()
    po, info, _ = restated.run_implicit(case, steps)
    cpu_s = time.perf_counter() - t0
    n = case.n_cells
    return {"workload": "NACA 0012 O-grid 256x128 (32,768 cells), Navier-Stokes Re 5000, Mach 0.5, AoA 1 deg, "
                        f"Roe, VK K=5, JFNK-GMRES(30) + LU-SGS, CFL 10, {steps} implicit steps",
            "cells": n, "newton_iterations": rep["newton_iterations"], "gmres_iterations": rep["gmres_iterations"],
            "gpu_ms_per_step": rep["device_ms"] / steps,
            "restated_cpu": {"s_per_step": cpu_s / steps, "cores": 1, "kind": "restated",
                             "newton_iterations": info["newton_iterations"],
                             "gmres_iterations": info["gmres_iterations"]},
            "speedup_vs_restated_cpu": (cpu_s / steps) / (rep["device_ms"] / 1e3 / steps),
            "state_vs_restated": float((np.abs(prim - po).max(axis=0) / np.abs(po).max(axis=0)).max()),
            "cl_cd_vs_restated": [abs(rep["cl"] - info["cl"]), abs(rep["cd"] - info["cd"])]}


def run_batched_airfoils(n_cases: int, steps: int, cfl: float) -> dict:
    """Steady-Euler airfoils of the batched distribution: the plain FP64 GPU
    solver looping over the cases one at a time vs all cases in one batch
    (lockstep Newton / GMRES / LU-SGS sets over all members), in FP64 and in
    mixed precision (FP32 Krylov basis and LU-SGS).  A solve is `steps`
    implicit time steps of one airfoil.  The FP64 batch gives states
    bit-identical to the loop (checked); the mixed batch states its error
    against the FP64 loop."""
    import ccfd_b200 as cc
    from ccfd_b200 import workloads
    specs = workloads.airfoil_specs(n_cases)
    with tempfile.TemporaryDirectory() as tmp:
        cases = [workloads.airfoil_case(sp, tmp, f"af{k}", cfl=cfl) for k, sp in enumerate(specs)]
        mixed = [workloads.airfoil_case(sp, tmp, f"af{k}", cfl=cfl, precision=1) for k, sp in enumerate(specs)]
    cells = [c.n_cells for c in cases]
    loop_ms, loop_states, loop_reps, t0 = 0.0, [], [], time.perf_counter()
    for c in cases:
        s = cc.Solver(c)
        rep = s.run(steps)
        loop_ms += rep["device_ms"]
        loop_states.append(s.get_state())
        loop_reps.append(rep)
        s.close()
    loop_wall = time.perf_counter() - t0

    def batched(cs):
        b = cc.Batch(0)
        members = [cc.Solver(c) for c in cs]
        for s in members:
            b.add(s, steps)
        t1 = time.perf_counter()
        b.step(steps)
        wall = time.perf_counter() - t1
        reps = [b.report(s) for s in members]
        states = [s.get_state() for s in members]
        b.close()
        for s in members:
            s.close()
        return reps, states, reps[0]["device_ms"], wall

    reps, states, batch_ms, batch_wall = batched(cases)
    diff = max(float(np.abs(st - ls).max()) for st, ls in zip(states, loop_states))
    mreps, mstates, mixed_ms, mixed_wall = batched(mixed)
    merr = max(float((np.abs(st - ls).max(axis=0) / np.abs(ls).max(axis=0)).max())
               for st, ls in zip(mstates, loop_states))
    mcl = max(abs(a["cl"] - b["cl"]) for a, b in zip(mreps, loop_reps))
    mcd = max(abs(a["cd"] - b["cd"]) for a, b in zip(mreps, loop_reps))
    return {
        "workload": f"{n_cases} NACA airfoils of the batched distribution (seed 20260004), O-grids "
                    f"{min(cells)}..{max(cells)} cells, steady Euler, Roe, 2nd order VK K=5, JFNK-GMRES "
                    f"(Krylov 30) + LU-SGS, CFL {cfl}, {steps} implicit steps per solve",
        "cells_total": int(sum(cells)), "solves": n_cases,
        "loop_fp64": {"device_s": loop_ms / 1e3, "wall_s": loop_wall,
                      "solves_per_s": n_cases / (loop_ms / 1e3)},
        "batched_fp64": {"device_s": batch_ms / 1e3, "wall_s": batch_wall,
                         "solves_per_s": n_cases / (batch_ms / 1e3),
                         "max_state_diff_vs_loop": diff},
        "batched_mixed": {"device_s": mixed_ms / 1e3, "wall_s": mixed_wall,
                          "solves_per_s": n_cases / (mixed_ms / 1e3),
                          "state_rel_err_vs_fp64_loop": merr, "cl_err": mcl, "cd_err": mcd,
                          "gmres_iterations": sum(r["gmres_iterations"] for r in mreps)},
        "speedup_batched_fp64": loop_ms / batch_ms,
        "speedup_batched_mixed": loop_ms / mixed_ms,
        "newton_iterations": sum(r["newton_iterations"] for r in reps),
        "gmres_iterations": sum(r["gmres_iterations"] for r in reps),
        "failed": sum(1 for r in reps + mreps if r["status"] != 0),
    }


def run_serving(n_req: int, load: float, budget: int, seed: int = 20260005) -> dict:
    """Served mixed stream: Riemann problems, cylinder-wake windows and
    airfoils.  (1) Each request alone through the plain loop gives its
    service time; (2) all requests submitted at once give the server's
    capacity; (3) Poisson arrivals at `load` x capacity are served with
    continuous batching in real time; the plain loop is scored on the same
    arrival times (first come, first served, measured service times)."""
    import ccfd_b200 as cc
    from ccfd_b200 import workloads
    reqs = workloads.stream_specs(n_req, seed, riemann_n=(256, 2048), cylinder_cells=(50_000, 400_000))
    with tempfile.TemporaryDirectory() as tmp:
        cases = [workloads.stream_case(r, tmp, f"q{k}") for k, r in enumerate(reqs)]
    # plain loop: per request upload, run, read the result back, release
    service, service_dev, ref_states = [], [], []
    for c, r in zip(cases, reqs):
        t0 = time.perf_counter()
        s = cc.Solver(c)
        rep = s.run(r["steps"])
        ref_states.append(s.get_state())
        s.close()
        service.append(time.perf_counter() - t0)
        service_dev.append(rep["device_ms"] / 1e3)

    def serve(arrivals, budget=budget):
        srv = cc.Server(0, hbm_budget_bytes=budget, max_running=4096)
        ids, done, lat = {}, {}, {}
        order = np.argsort(arrivals, kind="stable")
        k = 0
        t0 = time.perf_counter()
        max_used = 0
        while len(done) < len(cases):
            now = time.perf_counter() - t0
            while k < len(order) and arrivals[order[k]] <= now:
                j = int(order[k])
                ids[j] = srv.submit(cases[j], reqs[j]["steps"])
                k += 1
            if len(ids) == len(done):
                time.sleep(max(0.0, min(0.002, arrivals[order[k]] - now)) if k < len(order) else 0)
                continue
            srv.poll(16)
            max_used = max(max_used, srv.memory()[0])
            for j, rid in ids.items():
                if j in done:
                    continue
                got = srv.result(rid)
                if got is not None:
                    done[j] = got
                    lat[j] = got[2][2] - got[2][0]
        makespan = time.perf_counter() - t0
        host = srv.times()
        srv.close()
        return done, lat, makespan, max_used, host

    done, _, makespan_all, max_used_all, host_all = serve(np.zeros(len(cases)))
    capacity = len(cases) / makespan_all
    # admission under pressure: the closed loop again with a budget of 1.5x
    # the largest request's estimate, so requests wait for memory to free up
    est = [cc.estimate_device_bytes(c) for c in cases]
    tight = int(1.5 * max(est))
    done_t, _, makespan_t, max_used_t, _ = serve(np.zeros(len(cases)), budget=tight)
    same_t = all(np.array_equal(done_t[j][1], done[j][1]) for j in range(len(cases)))
    rate = load * capacity
    rng = np.random.Generator(np.random.PCG64(seed + 7))
    arrivals = np.cumsum(rng.exponential(1.0 / rate, len(cases)))
    arrivals -= arrivals[0]
    done, lat, makespan, max_used, host_open = serve(arrivals)
    same = all(np.array_equal(done[j][1], ref_states[j]) for j in range(len(cases)))
    # the plain loop on the same arrivals: first come, first served
    t_free, lat_loop = 0.0, []
    for j in np.argsort(arrivals, kind="stable"):
        start = max(t_free, arrivals[j])
        t_free = start + service[j]
        lat_loop.append(t_free - arrivals[j])
    lat_s = np.array([lat[j] for j in range(len(cases))])
    cells = [c.n_cells for c in cases]
    kinds = [r["kind"] for r in reqs]
    return {
        "workload": f"{n_req} requests (seed {seed}): " + ", ".join(
            f"{kinds.count(k)} {k}" for k in ("riemann", "cylinder", "airfoil"))
            + "; Riemann 256^2..2048^2 quads HLLC 200 RK3 steps, cylinder NS Re 100 M 0.2 50k..400k "
              "triangles 1000 RK3 steps, airfoils 5 implicit steps (JFNK + LU-SGS, CFL 1)",
        "cells_total": int(sum(cells)), "hbm_budget_bytes": budget, "max_resident_bytes": int(max_used),
        "max_resident_bytes_closed_loop": int(max_used_all),
        "tight_budget": {"hbm_budget_bytes": tight, "largest_request_estimate": int(max(est)),
                         "sum_of_estimates": int(sum(est)), "max_resident_bytes": int(max_used_t),
                         "capacity_solves_per_s": len(cases) / makespan_t, "results_equal": bool(same_t)},
        "capacity_solves_per_s": capacity, "arrival_rate_per_s": rate, "load": load,
        "served": {"solves_per_s": len(cases) / makespan, "p50_s": float(np.percentile(lat_s, 50)),
                   "p99_s": float(np.percentile(lat_s, 99))},
        "server_host_s": {"closed_loop": {"admit": host_all[0], "step": host_all[1], "retire": host_all[2],
                                          "makespan": makespan_all},
                          "open_loop": {"admit": host_open[0], "step": host_open[1], "retire": host_open[2],
                                        "makespan": makespan}},
        "plain_loop": {"solves_per_s": len(cases) / max(t_free, 1e-12),
                       "capacity_solves_per_s": len(cases) / sum(service),
                       "device_s": sum(service_dev), "wall_s": sum(service),
                       "p50_s": float(np.percentile(lat_loop, 50)),
                       "p99_s": float(np.percentile(lat_loop, 99))},
        "results_equal_alone": bool(same),
    }


def host_cpu() -> dict:
    """Host CPU of this process: model name, the logical CPUs it may run on
    and the physical cores behind them (distinct package / core ids)."""
    try:
        allowed = sorted(os.sched_getaffinity(0))
    except AttributeError:
        allowed = list(range(os.cpu_count() or 1))
    cores = set()
    for c in allowed:
        base = f"/sys/devices/system/cpu/cpu{c}/topology/"
        try:
            with open(base + "physical_package_id") as f:
                pkg = f.read().strip()
            with open(base + "core_id") as f:
                core = f.read().strip()
            cores.add((pkg, core))
        except OSError:
            cores.add(("?", str(c)))
    model = "unknown"
    try:
        with open("/proc/cpuinfo") as f:
            for ln in f:
                if ln.startswith("model name"):
                    model = ln.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return {"model": model, "logical_cpus": len(allowed), "physical_cores": len(cores)}


def cpu_reference_sample(ini: str, mesh_path: str, steps: int, threads: int):
    """Time the reference (compiled from its sources, oracle/_ref) on the
    host cores for `steps` time steps, `threads` OpenMP threads bound one per
    physical core (OMP_PROC_BIND=close, OMP_PLACES=cores): returns the wall
    clock (seconds, omp_get_wtime since the start of its time loop) at the
    end of each step and the whole dump of the run."""
    from oracle import refdump
    os.environ["OMP_PROC_BIND"] = "close"
    os.environ["OMP_PLACES"] = "cores"
    d = refdump.run_ref(ini, "run", steps, fast=True, threads=threads,
                        files={"dmr.msh": mesh_path}, timeout=1800)
    return d["step_wall"], d


def step_seconds(wall, first: int, last: int) -> float:
    """Wall time of steps first+1..last from the per-step clock of the
    reference's time loop (wall[k] = time at the end of step k+1)."""
    return wall[last - 1] - (wall[first - 1] if first > 0 else 0.0)


def load_meshgen_standalone():
    """The mesh generator module loaded by file path, without the package:
    the reference arm writes its input with it and must not load this
    library's native code."""
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "ccfd_meshgen_standalone", os.path.join(ROOT, "ccfd_b200", "meshgen.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def reference_arm_inputs(tmpdir: str):
    """Mesh file, .ini text, cell and face counts of the benchmark workload
    for the reference arm, made without importing the ccfd_b200 package."""
    mg = load_meshgen_standalone()
    mesh = mg.dmr_mesh(NX, NY)
    path = os.path.join(tmpdir, "dmr.msh")
    mesh.write_gmsh_text(path)
    return mg.dmr_ini("dmr"), path, mesh.n_cells, mesh.n_faces


def run_reference_arm(args, rank: int, world: int) -> None:
    if rank != 0:
        return
    from oracle import refdump
    cpu = host_cpu()
    threads = cpu["physical_cores"]
    with tempfile.TemporaryDirectory() as tmp:
        ini, path, n, faces = reference_arm_inputs(tmp)
        one = None
        if refdump.have_ref("euler", fast=True):
            kind = "reference"
            wall, _ = cpu_reference_sample(ini, path, args.warmup + args.steps, threads)
            t = step_seconds(wall, args.warmup, args.warmup + args.steps)
            cores = threads
            w1, _ = cpu_reference_sample(ini, path, 2, 1)
            one = n * 3 / step_seconds(w1, 1, 2)
        else:
            from oracle import restated
            import ccfd_b200 as cc  # the restatement reads the library's mesh arrays
            case = cc.CaseData.from_text(ini, tmp)
            kind = "port"
            cores = 1
            t0 = time.perf_counter()
            restated.run_explicit(case, nsteps=args.warmup + args.steps)
            t = (time.perf_counter() - t0) * args.steps / (args.warmup + args.steps)
    value = n * 3 * args.steps / t
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * t / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(n, faces, world),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": kind,
                             "cpu": cpu, "omp": "OMP_PROC_BIND=close OMP_PLACES=cores",
                             "one_thread_value": one,
                             "sample": f"{args.warmup} warm-up + {args.steps} timed RK3 steps of the "
                                       "full 500k-cell workload (reference's own time loop, "
                                       "omp_get_wtime per step); one_thread_value: step 2 of a "
                                       "2-step run on one thread"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main() -> int:
    global NX, NY
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--e2e-steps", type=int, default=20)
    ap.add_argument("--cpu-steps", type=int, default=3)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed-precision run")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-airfoil comparison")
    ap.add_argument("--no-serve", action="store_true", help="skip the served stream")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the Sod 400x20 and the 32k-cell Navier-Stokes airfoil legs")
    ap.add_argument("--airfoils", type=int, default=256,
                    help="airfoils of the batched set (the configuration's 256 by default)")
    ap.add_argument("--airfoil-steps", type=int, default=5)
    ap.add_argument("--requests", type=int, default=24)
    ap.add_argument("--nx", type=int, default=NX)
    ap.add_argument("--ny", type=int, default=NY)
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    NX, NY = args.nx, args.ny

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    import torch
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    if args.impl == "reference":
        run_reference_arm(args, rank, world)
        if dist is not None:
            dist.destroy_process_group()
        return 0

    torch.cuda.set_device(local)
    import ccfd_b200 as cc
    cc.set_device(local)
    hbm_peak, peak_src = _peaks()
    with tempfile.TemporaryDirectory() as tmp:
        case, ini, mesh_path = make_case(tmp)
        m = case.mesh()
        n = m["n_cells"]
        nrk = 3
        s = cc.Solver(case, reorder=True)
        s.set_profiling(True)
        # clocks are sampled from the start of the warm-up to the end of the
        # timed steps (the timed region alone can be shorter than a sample
        # period)
        clocks = ClockSampler(local)
        clocks.start()
        s.run(args.warmup)
        s.profile(reset=True)
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        rep = s.run(args.steps)
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        clk = clocks.stop()
        clk["window"] = "FP64 leg: warm-up and timed steps"
        res_ms, res_cnt = s.profile(reset=True)
        prim_fp64 = s.get_state()
        t_ms = max_over_ranks(rep["device_ms"], dist)
        steps_done = rep["iterations"] - args.warmup
        value = replica_throughput(world, n, nrk, steps_done, t_ms / 1e3)
        s.set_profiling(False)

        # end to end through the public API with host buffers: every step
        # uploads the state from pinned host memory and reads it back
        host = torch.empty((n, 4), dtype=torch.float64, pin_memory=True).numpy()
        host[:] = s.get_state()
        if dist is not None:
            dist.barrier()
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            s.set_state(host)
            s.run(1)
            s.get_state(out=host)
        t_e2e = time.perf_counter() - t0
        e2e_value = replica_throughput(world, n, nrk, args.e2e_steps, max_over_ranks(t_e2e, dist))
        s.close()

        n_tri = int((m["cell_type"] == 3).sum())
        bytes_stage = roofline_bytes_per_residual(n_tri, n - n_tri, venk=True)
        bytes_fused = algorithmic_bytes_per_stage(m, venk=True)
        mixed = None
        if not args.no_mixed:
            mixed = run_mixed(tmp, args.steps, args.warmup, prim_fp64, nrk, bytes_stage,
                              oracle_steps=0 if args.no_cpu else 2)
        batched = serving = sod = c3 = None
        if rank == 0 or world > 1:
            if not args.no_batch:
                batched = run_batched_airfoils(args.airfoils, args.airfoil_steps, cfl=1.0)
            if not args.no_serve:
                serving = run_serving(args.requests, load=0.8, budget=150 * 10**9)
            if not args.no_configs:
                sod = run_sod_c1(host_cpu()["physical_cores"])
                c3 = None if args.no_cpu else run_airfoil_c3()
        avg_res_ms = res_ms / max(res_cnt, 1)
        achieved = bytes_stage / (avg_res_ms / 1e3) / 1e9
        traffic, traffic_note = stage_traffic()

        cpu = None
        if rank == 0 and world == 1 and not args.no_cpu:
            from oracle import refdump
            hc = host_cpu()
            threads = hc["physical_cores"]
            if refdump.have_ref("euler", fast=True):
                wall, _ = cpu_reference_sample(ini, mesh_path, args.cpu_steps, threads)
                first = 1 if len(wall) > 1 else 0  # the first step is untimed
                st_cpu = len(wall) - first
                t_cpu = step_seconds(wall, first, len(wall))
                w1, _ = cpu_reference_sample(ini, mesh_path, 2, 1)
                cpu = {"value": n * nrk * st_cpu / t_cpu, "unit": UNIT, "cores": threads,
                       "kind": "reference", "cpu": hc,
                       "omp": "OMP_PROC_BIND=close OMP_PLACES=cores",
                       "one_thread_value": n * nrk / step_seconds(w1, 1, 2),
                       "sample": f"{args.cpu_steps} RK3 steps of the same 500k-cell workload "
                                 "(first step untimed), reference compiled from its sources "
                                 "(-O3 -march=x86-64-v3, OpenMP, one thread per physical core); "
                                 "one_thread_value: step 2 of a 2-step run on one thread"}
            else:
                from oracle import restated
                t0 = time.perf_counter()
                restated.residual(case, case.prim0(), 0.0)
                t_cpu = time.perf_counter() - t0
                cpu = {"value": n / t_cpu, "unit": UNIT, "cores": 1, "kind": "port", "cpu": hc,
                       "sample": "one residual evaluation of the 500k-cell workload (C restatement)"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t_ms / max(steps_done, 1), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(n, m["n_faces"], world),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm_peak,
                         "unit": "GB/s", "frac": achieved / hbm_peak,
                         "traffic": traffic, "traffic_source": traffic_note,
                         "kernel": "k_stage: fused residual evaluation + RK stage",
                         "bytes_per_launch": bytes_stage,
                         "bytes_per_cell": "364 (two-pass scheme, triangles, Venkatakrishnan)",
                         "fused_bytes_per_launch": bytes_fused, "avg_ms": avg_res_ms,
                         "peak_source": peak_src},
            "e2e": {"value": e2e_value, "unit": UNIT,
                    "h2d_bytes_per_step": n * 4 * 8, "d2h_bytes_per_step": n * 4 * 8},
            "gpu_launches": int(steps_done * nrk + 2),
            "clocks": clk,
            "cpu_baseline": cpu,
            "mixed_precision": mixed,
            "batched_airfoils": batched,
            "serving": serving,
            "sod_400x20": sod,
            "airfoil_ns_32k": c3,
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
