"""Python access to the C restatement of the reference path (oracle/ccfd_oracle.c).

TEST INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py as the checker.  The product never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_ROOT = os.path.dirname(_HERE)
SRC = os.path.join(_HERE, "ccfd_oracle.c")
LIB = os.path.join(_HERE, "_build", "libccfd_oracle.so")


def build(force: bool = False) -> str:
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    hdr = os.path.join(_ROOT, "include", "ccfd_b200.h")
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(
            os.path.getmtime(SRC), os.path.getmtime(hdr)):
        cmd = ["gcc", "-O2", "-std=c99", "-fPIC", "-shared", "-ffp-contract=off", "-Wall",
               "-I", os.path.join(_ROOT, "include"), SRC, "-o", LIB, "-lm"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("oracle build failed:\n" + r.stderr)
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB)
        dp = C.POINTER(C.c_double)
        L.oracle_residual.restype = C.c_int
        L.oracle_residual.argtypes = [C.c_void_p, dp, C.c_double, dp, dp, dp, dp]
        L.oracle_time_step.restype = C.c_int
        L.oracle_time_step.argtypes = [C.c_void_p, dp, C.c_double, C.c_double, dp]
        L.oracle_run_explicit.restype = C.c_int
        L.oracle_run_explicit.argtypes = [C.c_void_p, dp, C.c_long, dp]
        L.oracle_errors.restype = C.c_int
        L.oracle_errors.argtypes = [C.c_void_p, dp, C.c_double, C.c_int, dp]
        L.oracle_build_matrix.restype = C.c_int
        L.oracle_build_matrix.argtypes = [C.c_void_p, dp, dp, C.c_double, C.c_double, C.c_int,
                                          dp, dp, dp]
        L.oracle_lusgs.restype = None
        L.oracle_lusgs.argtypes = [C.c_void_p, dp, dp, dp, dp, dp]
        L.oracle_run_implicit.restype = C.c_int
        L.oracle_run_implicit.argtypes = [C.c_void_p, dp, C.c_long, C.c_double, C.c_int, dp, dp]
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double)) if a is not None else None


def _case_ptr(case):
    return C.cast(case._ptr, C.c_void_p)


def residual(case, prim: np.ndarray, time: float = 0.0, with_extras: bool = False):
    """fvTimeDerivative restated: returns u_t [N,4] (and grad [N,8], face flux
    [F,4], boundary-face interior pressure [B])."""
    n = case.n_cells
    m = case.c.mesh
    prim = np.ascontiguousarray(prim, dtype=np.float64).reshape(n, 4)
    ut = np.zeros((n, 4))
    gr = np.zeros((n, 8)) if with_extras else None
    ff = np.zeros((m.n_faces, 4)) if with_extras else None
    wp = np.zeros(max(m.n_bc, 1)) if with_extras else None
    st = lib().oracle_residual(_case_ptr(case), _dp(prim), float(time), _dp(ut), _dp(gr),
                               _dp(ff), _dp(wp))
    if st != 0:
        raise RuntimeError(f"oracle_residual status {st}")
    return (ut, gr, ff, wp[:m.n_bc]) if with_extras else ut


def errors(case, prim: np.ndarray, time: float, exact_func: int | None = None) -> dict:
    """calcErrors restated: L1, L2, Linf of the primitive variables."""
    which = case.c.exact_func if exact_func is None else exact_func
    prim = np.ascontiguousarray(prim, dtype=np.float64).reshape(case.n_cells, 4)
    e = np.zeros(12)
    st = lib().oracle_errors(_case_ptr(case), _dp(prim), float(time), int(which), _dp(e))
    if st != 0:
        raise RuntimeError(f"oracle_errors status {st}")
    return {"L1": e[0:4], "L2": e[4:8], "Linf": e[8:12]}


def time_step(case, prim: np.ndarray, t: float, print_time: float) -> float:
    dt = C.c_double()
    prim = np.ascontiguousarray(prim, dtype=np.float64)
    st = lib().oracle_time_step(_case_ptr(case), _dp(prim), float(t), float(print_time),
                                C.byref(dt))
    if st != 0:
        raise RuntimeError(f"oracle_time_step status {st}")
    return dt.value


def run_explicit(case, prim: np.ndarray | None = None, nsteps: int = 0):
    """Explicit time loop restated; returns (prim [N,4], info dict)."""
    p = np.array(case.prim0() if prim is None else prim, dtype=np.float64, copy=True)
    info = np.zeros(8)
    st = lib().oracle_run_explicit(_case_ptr(case), _dp(p), int(nsteps), _dp(info))
    if st != 0:
        raise RuntimeError(f"oracle_run_explicit status {st}")
    return p, {"t": info[0], "iterations": int(info[1]), "residual": info[2:6].tolist(),
               "finished": bool(info[6]), "converged": bool(info[7])}


def build_matrix(case, prim: np.ndarray, r_xk: np.ndarray, time: float, dt: float,
                 in_place: bool = True):
    """buildMatrix + calcDinv restated in block-sparse form.  Returns the
    state after the column evaluations (perturbed and restored in place like
    the reference when in_place), D and Dinv [N,4,4] and the off-diagonal
    block of every half-side [H,4,4] (row cell of the half-side, column cell
    across it; zero at boundary sides)."""
    n = case.n_cells
    h = case.c.mesh.n_half_sides
    p = np.array(prim, dtype=np.float64).reshape(n, 4).copy()
    r = np.ascontiguousarray(r_xk, dtype=np.float64).reshape(n, 4)
    D = np.zeros((n, 4, 4))
    Di = np.zeros((n, 4, 4))
    O = np.zeros((h, 4, 4))
    st = lib().oracle_build_matrix(_case_ptr(case), _dp(p), _dp(r), float(time), float(dt),
                                   int(bool(in_place)), _dp(D), _dp(Di), _dp(O))
    if st != 0:
        raise RuntimeError(f"oracle_build_matrix status {st}")
    return p, D, Di, O


def lusgs(case, Dinv: np.ndarray, O: np.ndarray, b: np.ndarray) -> np.ndarray:
    """LUSGS restated: the preconditioned vector M^-1 b [N,4]."""
    n = case.n_cells
    Di = np.ascontiguousarray(Dinv, dtype=np.float64)
    Oc = np.ascontiguousarray(O, dtype=np.float64)
    bb = np.ascontiguousarray(b, dtype=np.float64).reshape(n, 4)
    x = np.zeros((n, 4))
    xs = np.zeros((n, 4))
    lib().oracle_lusgs(_case_ptr(case), _dp(Di), _dp(Oc), _dp(bb), _dp(x), _dp(xs))
    return x


def run_implicit(case, nsteps: int, prim: np.ndarray | None = None, ser_cfl_max: float = 0.0,
                 in_place: bool = True):
    """The implicit time loop restated (implicitTimeStep with GMRES_M and,
    with precond, the restated buildMatrix / LUSGS).  Returns the final
    primitive state, an info dict and the per-step history rows
    (t, dt, res[4], cl, cd)."""
    n = case.n_cells
    p = np.array(case.prim0() if prim is None else prim, dtype=np.float64).reshape(n, 4).copy()
    info = np.zeros(12)
    cap = nsteps if nsteps > 0 else int(case.params.max_iter)
    hist = np.zeros((max(cap, 1), 8))
    st = lib().oracle_run_implicit(_case_ptr(case), _dp(p), int(nsteps), float(ser_cfl_max),
                                   int(bool(in_place)), _dp(info), _dp(hist))
    k = int(info[1])
    return p, {"status": st, "t": info[0], "iterations": k, "res": info[2:6].copy(),
               "finished": bool(info[6]), "converged": bool(info[7]),
               "newton_iterations": int(info[8]), "gmres_iterations": int(info[9]),
               "cl": info[10], "cd": info[11]}, hist[:k].copy()
