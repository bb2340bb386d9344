"""ccfd_b200: the residual-and-update path of the 2-D finite-volume solver ccfd
(hheinzer/ccfd) on NVIDIA B200, behind a C ABI (include/ccfd_b200.h).

The Python layer mirrors the reference's interface for this path:

* :class:`CaseData` -- a case read from a reference ``.ini`` file with the
  reference's parser semantics (main's init sequence, src/main.c:53-118).
* :class:`Solver`   -- device state of one case: ``fv_time_derivative``
  (fvTimeDerivative, src/finiteVolume.c:78), ``calc_time_step``
  (calcTimeStep, src/timeDiscretization.c:249), ``run`` (the time loop of
  timeDisc with explicitTimeStepRK / implicitTimeStep), ``global_residual``
  (src/analyze.c:521) and ``clcd`` (calcCoef, src/analyze.c:292).

Every call goes to the CUDA kernels in ``lib/libccfd_b200.so``; there is no
CPU implementation behind this package.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import _native as N

__all__ = ["CaseData", "Solver", "Batch", "Server", "estimate_device_bytes", "set_device", "CcfdError", "mesh_arrays", "PRIMITIVE", "CONSERVATIVE"]

PRIMITIVE, CONSERVATIVE = N.PRIMITIVE, N.CONSERVATIVE

FLUX_NAMES = {1: "Godunov", 2: "Roe", 3: "HLL", 4: "HLLE", 5: "HLLC", 6: "Lax-Friedrichs",
              7: "Steger-Warming", 8: "central", 9: "AUSMD", 10: "AUSMDV", 11: "van Leer"}


class CcfdError(RuntimeError):
    def __init__(self, status: int, where: str):
        msg = N.lib.ccfd_strerror(status).decode()
        super().__init__(f"{where}: {msg} (status {status})")
        self.status = status


def _check(st: int, where: str) -> None:
    if st != 0:
        raise CcfdError(st, where)


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _lptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_long))


def _arr(ptr, shape, dtype):
    n = int(np.prod(shape))
    if n == 0:
        return np.zeros(shape, dtype=dtype)
    return np.ctypeslib.as_array(ptr, shape=(n,)).astype(dtype, copy=True).reshape(shape)


def mesh_arrays(m: N.Mesh) -> dict:
    """Copy a ccfd_mesh into numpy arrays (reference element / face order)."""
    n, f, b, h = m.n_cells, m.n_faces, m.n_bc, m.n_half_sides
    return {
        "n_cells": n, "n_faces": f, "n_bc": b, "n_half_sides": h,
        "cell_type": _arr(m.cell_type, (n,), np.int32),
        "cell_domain": _arr(m.cell_domain, (n,), np.int32),
        "cell_bary": _arr(m.cell_bary, (n, 2), np.float64),
        "cell_geo": _arr(m.cell_geo, (n, 4), np.float64),
        "hs_offset": _arr(m.hs_offset, (n + 1,), np.int64),
        "hs_face": _arr(m.hs_face, (h,), np.int64),
        "hs_sign": _arr(m.hs_sign, (h,), np.int32),
        "hs_nb": _arr(m.hs_nb, (h,), np.int64),
        "hs_gp": _arr(m.hs_gp, (h, 2), np.float64),
        "hs_w": _arr(m.hs_w, (h, 2), np.float64),
        "face_cells": _arr(m.face_cells, (f, 2), np.int64),
        "face_hs": _arr(m.face_hs, (f, 2), np.int64),
        "face_n": _arr(m.face_n, (f, 2), np.float64),
        "face_len": _arr(m.face_len, (f,), np.float64),
        "face_bb": _arr(m.face_bb, (f, 3), np.float64),
        "ghost_gp": _arr(m.ghost_gp, (b, 2), np.float64),
        "bc_face": _arr(m.bc_face, (b,), np.int64),
        "bc_index": _arr(m.bc_index, (b,), np.int32),
        "bc_ghost_bary": _arr(m.bc_ghost_bary, (b, 2), np.float64),
        "bc_x": _arr(m.bc_x, (b, 2), np.float64),
        "total_area_q": m.total_area_q, "dx_ref": m.dx_ref,
        "x_min": m.x_min, "x_max": m.x_max, "y_min": m.y_min, "y_max": m.y_max,
    }


def colour_cells(hs_offset: np.ndarray, hs_nb: np.ndarray, budget: int = -1) -> tuple[np.ndarray, int]:
    """Distance-3 colouring of the face-neighbour graph that groups the
    columns of the block-sparse buildMatrix (``ccfd_colour_cells``); budget 0:
    greedy only, negative: the solver's default tabu-search budget."""
    off = np.ascontiguousarray(hs_offset, dtype=np.int64)
    nb = np.ascontiguousarray(hs_nb, dtype=np.int64)
    n = len(off) - 1
    color = np.zeros(max(n, 1), dtype=np.int32)
    nc = C.c_int(0)
    _check(N.lib.ccfd_colour_cells(n, _lptr(off), _lptr(nb), int(budget),
                                   color.ctypes.data_as(C.POINTER(C.c_int)), C.byref(nc)), "colour_cells")
    return color[:n], nc.value


class CaseData:
    """A case built by the C host layer from a reference ``.ini`` file."""

    def __init__(self, ptr):
        self._ptr = ptr

    @classmethod
    def from_ini(cls, path: str) -> "CaseData":
        p = C.POINTER(N.Case)()
        _check(N.lib.ccfd_case_load(os.fsencode(path), C.byref(p)), f"load {path}")
        return cls(p)

    @classmethod
    def from_text(cls, text: str, base_dir: str | None = None) -> "CaseData":
        p = C.POINTER(N.Case)()
        bd = os.fsencode(base_dir) if base_dir else None
        _check(N.lib.ccfd_case_load_text(text.encode(), bd, C.byref(p)), "load ini text")
        return cls(p)

    def __del__(self):
        if getattr(self, "_ptr", None):
            try:
                N.lib.ccfd_case_free(self._ptr)
            except Exception:  # interpreter shutdown: the module is gone
                pass
            self._ptr = None

    @property
    def c(self) -> N.Case:
        return self._ptr.contents

    @property
    def params(self) -> N.Params:
        return self.c.params

    @property
    def n_cells(self) -> int:
        return self.c.mesh.n_cells

    def mesh(self) -> dict:
        return mesh_arrays(self.c.mesh)

    def prim0(self) -> np.ndarray:
        return _arr(self.c.prim0, (self.n_cells, 4), np.float64)

    def venk_eps2(self, venk_k: float | None = None) -> np.ndarray:
        k = self.params.venk_k if venk_k is None else venk_k
        out = np.zeros(self.n_cells)
        N.lib.ccfd_venk_eps2(C.byref(self.c.mesh), k, _dptr(out))
        return out

    @property
    def file_name(self) -> str:
        return self.c.file_name.decode()

    def record_points(self) -> tuple[np.ndarray, np.ndarray]:
        """(pointCoords [n, 2], containing cell [n]) of the case."""
        c = self.c
        xy = np.array([[c.record_xy[k][0], c.record_xy[k][1]] for k in range(c.n_record)]).reshape(-1, 2)
        return xy, np.array([c.record_cell[k] for k in range(c.n_record)], dtype=np.int64)

    def write_history(self, rows: np.ndarray, append: bool = False) -> None:
        """analyze's files (residual file, record points) from history rows,
        into the current directory."""
        r = np.ascontiguousarray(rows, dtype=np.float64)
        _check(N.lib.ccfd_write_history(self._ptr, _dptr(r), r.shape[0], r.shape[1] if r.ndim == 2 else 0,
                                        int(append)), "ccfd_write_history")

    def write_output(self, prim: np.ndarray, time: float, iteration: int, exact: bool = False) -> str:
        """Write the state in the reference's output format (CSV or curve)
        into the current directory; ``exact``: the exact-solution file
        (<fileName>_ex_...) of a state from Solver.exact_state.  Returns the
        file name."""
        p = np.ascontiguousarray(prim, dtype=np.float64).reshape(self.n_cells, 4)
        buf = C.create_string_buffer(600)
        fn = N.lib.ccfd_write_exact_output if exact else N.lib.ccfd_write_output
        _check(fn(self._ptr, _dptr(p), float(time), int(iteration), buf, 600), "ccfd_write_output")
        return buf.value.decode()


def set_device(device: int) -> None:
    """Bind the calling thread's next contexts to a CUDA device."""
    _check(N.lib.ccfd_set_device(int(device)), "ccfd_set_device")


class Solver:
    """One case resident on the current CUDA device."""

    def __init__(self, case: CaseData, reorder: int = 1, params: N.Params | None = None):
        """Upload a case; ``reorder`` is the device cell order (0 the
        reference's numbering, 1 Hilbert curve, 2 reverse Cuthill-McKee)."""
        self.case = case
        self._ctx = C.c_void_p()
        prm = params if params is not None else case.params
        _check(N.lib.ccfd_create(C.byref(prm), C.byref(self._ctx)), "ccfd_create")
        c = case.c
        _check(N.lib.ccfd_upload_case(self._ctx, C.byref(c.mesh), c.bc_table, c.n_bc_table,
                                      C.byref(c.exact), int(reorder)), "ccfd_upload_case")
        self.n = case.n_cells
        self.set_state(case.prim0(), PRIMITIVE)

    def close(self):
        if self._ctx:
            N.lib.ccfd_destroy(self._ctx)
            self._ctx = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_state(self, state: np.ndarray, kind: int = PRIMITIVE) -> None:
        s = np.ascontiguousarray(state, dtype=np.float64).reshape(self.n, 4)
        _check(N.lib.ccfd_set_state(self._ctx, _dptr(s), kind), "ccfd_set_state")

    def get_state(self, kind: int = PRIMITIVE, out: np.ndarray | None = None) -> np.ndarray:
        """The state [N, 4] in reference cell order; `out` (C-contiguous
        float64, e.g. pinned host memory) receives it without a new array."""
        if out is None:
            out = np.empty((self.n, 4))
        elif out.dtype != np.float64 or not out.flags.c_contiguous or out.size != 4 * self.n:
            raise ValueError("out must be a C-contiguous float64 array of n_cells x 4")
        _check(N.lib.ccfd_get_state(self._ctx, _dptr(out), kind), "ccfd_get_state")
        return out

    @property
    def time(self) -> float:
        t = C.c_double()
        _check(N.lib.ccfd_get_time(self._ctx, C.byref(t)), "ccfd_get_time")
        return t.value

    @time.setter
    def time(self, t: float) -> None:
        _check(N.lib.ccfd_set_time(self._ctx, float(t)), "ccfd_set_time")

    def fv_time_derivative(self, time: float = 0.0, with_grad: bool = False):
        """R(U) of the current state; [N, 4] (and [N, 8] limited gradients)."""
        ut = np.empty((self.n, 4))
        gr = np.empty((self.n, 8)) if with_grad else None
        _check(N.lib.ccfd_residual(self._ctx, float(time), _dptr(ut),
                                   _dptr(gr) if with_grad else None), "ccfd_residual")
        return (ut, gr) if with_grad else ut

    def calc_time_step(self) -> float:
        dt = C.c_double()
        _check(N.lib.ccfd_time_step(self._ctx, C.byref(dt)), "ccfd_time_step")
        return dt.value

    def global_residual(self) -> np.ndarray:
        r = np.zeros(4)
        _check(N.lib.ccfd_global_residual(self._ctx, _dptr(r)), "ccfd_global_residual")
        return r

    def run(self, nsteps: int = 0) -> dict:
        """Time steps (explicit or implicit per the case); nsteps <= 0: to the end."""
        rep = N.Report()
        fn = N.lib.ccfd_run_implicit if self.case.params.implicit else N.lib.ccfd_run_explicit
        _check(fn(self._ctx, int(nsteps), C.byref(rep)), "ccfd_run")
        return report_dict(rep)

    def set_profiling(self, on: bool) -> None:
        _check(N.lib.ccfd_set_profiling(self._ctx, int(on)), "ccfd_set_profiling")

    def profile(self, reset: bool = True):
        """(accumulated residual-evaluation device ms, count) inside step graphs."""
        ms, cnt = C.c_double(), C.c_long()
        _check(N.lib.ccfd_get_profile(self._ctx, C.byref(ms), C.byref(cnt), int(reset)),
               "ccfd_get_profile")
        return ms.value, cnt.value

    def autotune(self, state: np.ndarray | None = None) -> dict:
        """Pick the stage kernel's tile size, cell ordering and CTA size by
        timing (ccfd_autotune); the solver keeps the fastest and `state`
        (default: the case's initial state)."""
        c = self.case.c
        prim = np.ascontiguousarray(self.case.prim0() if state is None else state,
                                    dtype=np.float64).reshape(self.n, 4)
        tc, ro, th, ms = C.c_int(), C.c_int(), C.c_int(), C.c_double()
        _check(N.lib.ccfd_autotune(self._ctx, C.byref(c.mesh), c.bc_table, c.n_bc_table,
                                   C.byref(c.exact), _dptr(prim), C.byref(tc), C.byref(ro),
                                   C.byref(th), C.byref(ms)), "ccfd_autotune")
        return {"tile_cells": tc.value, "hilbert_order": bool(ro.value), "threads": th.value,
                "ms_per_residual": ms.value}

    def device_bytes(self) -> int:
        b = C.c_size_t()
        _check(N.lib.ccfd_device_bytes(self._ctx, C.byref(b)), "ccfd_device_bytes")
        return b.value

    def wall_cp(self):
        """(x, y, cp, n_pressure_side) along the wing (ccfd_wall_cp)."""
        n, npres = C.c_int(), C.c_int()
        _check(N.lib.ccfd_wall_cp(self._ctx, None, None, None, C.byref(n), C.byref(npres)), "ccfd_wall_cp")
        x, y, cp = np.empty(n.value), np.empty(n.value), np.empty(n.value)
        _check(N.lib.ccfd_wall_cp(self._ctx, _dptr(x), _dptr(y), _dptr(cp), C.byref(n), C.byref(npres)),
               "ccfd_wall_cp")
        return x, y, cp, npres.value

    def write_cp(self, base: str) -> None:
        """The reference's CP files <base>_CP_pressureSide.csv / _CP_suctionSide.csv."""
        _check(N.lib.ccfd_write_cp(self._ctx, os.fsencode(base)), "ccfd_write_cp")

    def errors(self, exact_func: int | None = None) -> dict:
        """calcErrors at the current time (ccfd_errors): L1, L2 and Linf of
        the primitive variables against the case's exact function."""
        which = self.case.c.exact_func if exact_func is None else exact_func
        e = np.empty(12)
        _check(N.lib.ccfd_errors(self._ctx, int(which), _dptr(e)), "ccfd_errors")
        return {"L1": e[0:4].copy(), "L2": e[4:8].copy(), "Linf": e[8:12].copy()}

    def set_history(self, capacity: int = 4096, record_cells=None) -> None:
        """Record one row per step from now on (ccfd_set_history): residuals,
        CL / CD and the state of the record cells (default: the case's
        record points).  capacity <= 0 switches it off."""
        if record_cells is None:
            c = self.case.c
            record_cells = [c.record_cell[k] for k in range(c.n_record)]
        cells = np.ascontiguousarray(record_cells, dtype=np.int64)
        _check(N.lib.ccfd_set_history(self._ctx, int(capacity), _lptr(cells), len(cells)),
               "ccfd_set_history")

    def history(self) -> np.ndarray:
        """Rows recorded since the last call, [n, 11 + 4 * n_record]:
        iteration, t, dt, residuals [6], CL, CD, (rho, vx, vy, p) per record
        cell."""
        n, w = C.c_long(), C.c_int()
        _check(N.lib.ccfd_get_history(self._ctx, None, 0, C.byref(n), C.byref(w)), "ccfd_get_history")
        out = np.empty((n.value, w.value))
        _check(N.lib.ccfd_get_history(self._ctx, _dptr(out), n.value, C.byref(n), C.byref(w)),
               "ccfd_get_history")
        return out[:n.value]

    def exact_state(self, time: float | None = None, exact_func: int | None = None) -> np.ndarray:
        """Exact function at the cell barycentres (ccfd_exact_state), at the
        solver's current time by default; [N, 4] primitive."""
        which = self.case.c.exact_func if exact_func is None else exact_func
        t = self.time if time is None else time
        out = np.empty((self.n, 4))
        _check(N.lib.ccfd_exact_state(self._ctx, int(which), float(t), _dptr(out)), "ccfd_exact_state")
        return out

    def clcd(self):
        cl, cd = C.c_double(), C.c_double()
        _check(N.lib.ccfd_clcd(self._ctx, C.byref(cl), C.byref(cd)), "ccfd_clcd")
        return cl.value, cd.value

    def build_matrix(self, time: float, dt: float):
        """buildMatrix + calcDinv at the current state (first Newton
        iteration of a step from `time` with step `dt`): D, Dinv [N,4,4] and
        the off-diagonal block of every half-side [H,4,4], reference order."""
        n = self.case.n_cells
        h = self.case.c.mesh.n_half_sides
        D = np.zeros((n, 4, 4))
        Di = np.zeros((n, 4, 4))
        O = np.zeros((h, 4, 4))
        dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
        _check(N.lib.ccfd_build_matrix(self._ctx, float(time), float(dt), dp(D), dp(Di), dp(O)),
               "ccfd_build_matrix")
        return D, Di, O

    def lusgs(self, b: np.ndarray) -> np.ndarray:
        """LUSGS of b [N,4] with the blocks of the last build_matrix."""
        n = self.case.n_cells
        bb = np.ascontiguousarray(b, dtype=np.float64).reshape(n, 4)
        x = np.zeros((n, 4))
        dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
        _check(N.lib.ccfd_lusgs(self._ctx, dp(bb), dp(x)), "ccfd_lusgs")
        return x


class Batch:
    """Many solvers stepped together on one device (see ccfd_batch_* in the
    C header).  A solver in a batch is stepped only by the batch; its state
    and report stay readable."""

    def __init__(self, device: int = 0):
        self._b = C.c_void_p()
        _check(N.lib.ccfd_batch_create(int(device), C.byref(self._b)), "ccfd_batch_create")
        self.members: list[Solver] = []

    def add(self, solver: "Solver", nsteps: int = 0) -> None:
        _check(N.lib.ccfd_batch_add(self._b, solver._ctx, int(nsteps)), "ccfd_batch_add")
        self.members.append(solver)

    def remove(self, solver: "Solver") -> None:
        _check(N.lib.ccfd_batch_remove(self._b, solver._ctx), "ccfd_batch_remove")
        self.members.remove(solver)

    def step(self, steps: int = 1) -> int:
        """Advance every running member by up to ``steps`` time steps;
        returns how many members can still step."""
        n = C.c_int()
        _check(N.lib.ccfd_batch_step(self._b, int(steps), C.byref(n)), "ccfd_batch_step")
        return n.value

    def report(self, solver: "Solver") -> dict:
        rep = N.Report()
        _check(N.lib.ccfd_batch_report(self._b, solver._ctx, C.byref(rep)), "ccfd_batch_report")
        return report_dict(rep)

    def close(self) -> None:
        if self._b:
            N.lib.ccfd_batch_destroy(self._b)
            self._b = C.c_void_p()
            self.members = []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Request loop with continuous batching (see ccfd_server_* in the C
    header): cases queue in arrival order, are admitted by a device-memory
    budget, run together and are retired when they stop."""

    def __init__(self, device: int = 0, hbm_budget_bytes: int = 150 * 10**9, max_running: int = 4096):
        self._s = C.c_void_p()
        _check(N.lib.ccfd_server_create(int(device), int(hbm_budget_bytes), int(max_running),
                                        C.byref(self._s)), "ccfd_server_create")
        self._cases: dict[int, CaseData] = {}

    def submit(self, case: "CaseData", nsteps: int = 0) -> int:
        rid = C.c_long()
        _check(N.lib.ccfd_server_submit(self._s, case._ptr, int(nsteps), C.byref(rid)),
               "ccfd_server_submit")
        self._cases[rid.value] = case  # the server reads the case until it finishes
        return rid.value

    def poll(self, steps: int = 16) -> tuple[int, int, int]:
        """(queued, running, finished-not-fetched) after one scheduling round."""
        q, r, d = C.c_int(), C.c_int(), C.c_int()
        _check(N.lib.ccfd_server_poll(self._s, int(steps), C.byref(q), C.byref(r), C.byref(d)),
               "ccfd_server_poll")
        return q.value, r.value, d.value

    def result(self, rid: int, with_state: bool = True):
        """(report, final primitive state or None, (t_submit, t_admit, t_done)),
        or None while the request is queued or running."""
        case = self._cases[rid]
        rep = N.Report()
        prim = np.empty((case.n_cells, 4)) if with_state else None
        times = (C.c_double * 3)()
        st = N.lib.ccfd_server_result(self._s, int(rid), C.byref(rep),
                                      _dptr(prim) if with_state else None, times)
        if st == 16:  # CCFD_ERR_BUSY
            return None
        del self._cases[rid]
        out = report_dict(rep)
        out["status"] = st
        return out, prim, tuple(times)

    def memory(self) -> tuple[int, int]:
        used, budget = C.c_size_t(), C.c_size_t()
        _check(N.lib.ccfd_server_memory(self._s, C.byref(used), C.byref(budget)), "ccfd_server_memory")
        return used.value, budget.value

    def times(self) -> tuple[float, float, float]:
        """Host seconds spent admitting (upload), stepping and retiring."""
        out = (C.c_double * 3)()
        _check(N.lib.ccfd_server_times(self._s, out), "ccfd_server_times")
        return tuple(out)

    def close(self) -> None:
        if self._s:
            N.lib.ccfd_server_destroy(self._s)
            self._s = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def estimate_device_bytes(case: "CaseData") -> int:
    b = C.c_size_t()
    c = case.c
    _check(N.lib.ccfd_estimate_device_bytes(C.byref(c.params), C.byref(c.mesh), C.byref(b)),
           "ccfd_estimate_device_bytes")
    return b.value


def report_dict(rep: N.Report) -> dict:
    return {"t": rep.t, "dt": rep.dt, "iterations": rep.iterations,
            "residual": list(rep.residual), "cl": rep.cl, "cd": rep.cd,
            "converged": bool(rep.converged), "finished": bool(rep.finished),
            "newton_iterations": rep.newton_iterations, "gmres_iterations": rep.gmres_iterations,
            "first_residual": list(rep.first_residual), "status": rep.status,
            "device_ms": rep.device_ms}
