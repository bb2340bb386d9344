"""ctypes binding of the C ABI declared in include/ccfd_b200.h.

Loading fails loudly (ImportError) when the in-tree library has not been
built: there is no fallback implementation.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libccfd_b200.so")

c_int, c_long, c_double = C.c_int, C.c_long, C.c_double
P = C.POINTER

CCFD_OK, CCFD_ERR_ARG = 0, 1
NOALLOC_MAX_CELLS = 1 << 20  # CCFD_NOALLOC_MAX_CELLS
MAX_RECORD = 64  # CCFD_MAX_RECORD


class Params(C.Structure):
    _fields_ = [
        ("eqn", c_int), ("flux", c_int), ("spatial_order", c_int), ("limiter", c_int),
        ("venk_k", c_double), ("gamma", c_double), ("R", c_double), ("mu", c_double),
        ("Pr", c_double), ("time_order", c_int), ("n_rk_stages", c_int),
        ("cfl", c_double), ("dfl", c_double), ("time_step_1d", c_int), ("stationary", c_int),
        ("t_end", c_double), ("max_iter", c_long), ("io_time_interval", c_double),
        ("io_iter_interval", c_long), ("abort_residual", c_double), ("abort_variable", c_int),
        ("cl_abort_residual", c_double), ("cd_abort_residual", c_double),
        ("implicit", c_int), ("precond", c_int), ("n_kdim", c_int), ("n_newton_iter", c_int),
        ("eps_newton", c_double), ("eps_gmres", c_double), ("gamma_ew", c_double),
        ("calc_wing", c_int), ("wall_id", c_int), ("ref_length", c_double),
        ("precision", c_int), ("rel_abort_residual", c_double),
        ("source_func", c_int), ("exact_solution", c_int), ("ser_cfl_max", c_double),
    ]


class BC(C.Structure):
    _fields_ = [("type", c_int), ("id", c_int), ("exact_func", c_int), ("is_adiabatic", c_int),
                ("pvar", c_double * 4), ("connection", c_double * 2)]


class Exact(C.Structure):
    _fields_ = [("ref_state", (c_double * 4) * 2), ("rp1d_interface", c_double),
                ("alpha", c_double), ("x_min", c_double), ("x_max", c_double),
                ("y_min", c_double), ("y_max", c_double), ("dx_ref", c_double)]


class Mesh(C.Structure):
    _fields_ = [
        ("n_cells", c_long), ("n_faces", c_long), ("n_bc", c_long), ("n_half_sides", c_long),
        ("n_nodes", c_long),
        ("cell_type", P(c_int)), ("cell_domain", P(c_int)), ("cell_bary", P(c_double)),
        ("cell_geo", P(c_double)), ("hs_offset", P(c_long)), ("hs_face", P(c_long)),
        ("hs_sign", P(c_int)), ("hs_nb", P(c_long)), ("hs_gp", P(c_double)), ("hs_w", P(c_double)),
        ("face_cells", P(c_long)), ("face_hs", P(c_long)), ("face_n", P(c_double)),
        ("face_len", P(c_double)), ("face_bb", P(c_double)), ("ghost_gp", P(c_double)),
        ("bc_face", P(c_long)), ("bc_index", P(c_int)), ("bc_ghost_bary", P(c_double)),
        ("bc_x", P(c_double)), ("cell_gp5", P(c_double)), ("cell_nodes", P(c_long)),
        ("node_xy", P(c_double)),
        ("total_area_q", c_double), ("dx_ref", c_double), ("x_min", c_double),
        ("x_max", c_double), ("y_min", c_double), ("y_max", c_double),
    ]


class Case(C.Structure):
    _fields_ = [("params", Params), ("n_bc_table", c_int), ("bc_table", BC * 20),
                ("exact", Exact), ("mesh", Mesh), ("prim0", P(c_double)),
                ("file_name", C.c_char * 256), ("output_format", c_int),
                ("ic_type", c_int), ("exact_func", c_int), ("n_record", c_int),
                ("record_xy", (c_double * 2) * MAX_RECORD), ("record_cell", c_long * MAX_RECORD)]


class Report(C.Structure):
    _fields_ = [("t", c_double), ("dt", c_double), ("iterations", c_long),
                ("residual", c_double * 6), ("cl", c_double), ("cd", c_double),
                ("converged", c_int), ("finished", c_int), ("newton_iterations", c_long),
                ("gmres_iterations", c_long), ("first_residual", c_double * 4),
                ("status", c_int), ("device_ms", c_double)]


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"ccfd_b200 native library missing: {LIB_PATH}; run `python -m ccfd_b200.build`")
    lib = C.CDLL(LIB_PATH)
    sig = {
        "ccfd_case_load": (c_int, [C.c_char_p, P(P(Case))]),
        "ccfd_case_load_text": (c_int, [C.c_char_p, C.c_char_p, P(P(Case))]),
        "ccfd_mesh_build": (c_int, [P(c_double), c_long, P(c_long), c_long, P(c_long), c_long,
                                    P(c_long), c_long, P(BC), c_int, P(Mesh)]),
        "ccfd_mesh_free": (None, [P(Mesh)]),
        "ccfd_case_free": (None, [P(Case)]),
        "ccfd_venk_eps2": (None, [P(Mesh), c_double, P(c_double)]),
        "ccfd_write_gmsh2": (c_int, [C.c_char_p, P(c_double), c_long, P(c_long), c_long,
                                     P(c_long), c_long, P(c_long), c_long]),
        "ccfd_read_gmsh": (c_int, [C.c_char_p, P(P(c_double)), P(c_long), P(P(c_long)),
                                   P(c_long), P(P(c_long)), P(c_long), P(P(c_long)), P(c_long)]),
        "ccfd_strerror": (C.c_char_p, [c_int]),
        "ccfd_set_device": (c_int, [c_int]),
        "ccfd_create": (c_int, [P(Params), P(C.c_void_p)]),
        "ccfd_destroy": (None, [C.c_void_p]),
        "ccfd_upload_case": (c_int, [C.c_void_p, P(Mesh), P(BC), c_int, P(Exact), c_int]),
        "ccfd_set_state": (c_int, [C.c_void_p, P(c_double), c_int]),
        "ccfd_get_state": (c_int, [C.c_void_p, P(c_double), c_int]),
        "ccfd_set_time": (c_int, [C.c_void_p, c_double]),
        "ccfd_get_time": (c_int, [C.c_void_p, P(c_double)]),
        "ccfd_residual": (c_int, [C.c_void_p, c_double, P(c_double), P(c_double)]),
        "ccfd_time_step": (c_int, [C.c_void_p, P(c_double)]),
        "ccfd_run_explicit": (c_int, [C.c_void_p, c_long, P(Report)]),
        "ccfd_run_implicit": (c_int, [C.c_void_p, c_long, P(Report)]),
        "ccfd_global_residual": (c_int, [C.c_void_p, P(c_double)]),
        "ccfd_clcd": (c_int, [C.c_void_p, P(c_double), P(c_double)]),
        "ccfd_build_matrix": (c_int, [C.c_void_p, c_double, c_double, P(c_double), P(c_double),
                                      P(c_double)]),
        "ccfd_lusgs": (c_int, [C.c_void_p, P(c_double), P(c_double)]),
        "ccfd_colour_cells": (c_int, [C.c_long, P(C.c_long), P(C.c_long), C.c_long, P(C.c_int), P(C.c_int)]),
        "ccfd_set_profiling": (c_int, [C.c_void_p, c_int]),
        "ccfd_get_profile": (c_int, [C.c_void_p, P(c_double), P(c_long), c_int]),
        "ccfd_global_residual_noalloc": (c_int, [C.c_void_p, C.c_void_p, c_long, c_double,
                                                 C.c_void_p, C.c_void_p]),
        "ccfd_autotune": (c_int, [C.c_void_p, P(Mesh), P(BC), c_int, P(Exact), P(c_double), P(c_int),
                                  P(c_int), P(c_int), P(c_double)]),
        "ccfd_wall_cp": (c_int, [C.c_void_p, P(c_double), P(c_double), P(c_double), P(c_int), P(c_int)]),
        "ccfd_write_cp": (c_int, [C.c_void_p, C.c_char_p]),
        "ccfd_errors": (c_int, [C.c_void_p, c_int, P(c_double)]),
        "ccfd_exact_state": (c_int, [C.c_void_p, c_int, c_double, P(c_double)]),
        "ccfd_set_history": (c_int, [C.c_void_p, c_int, P(c_long), c_int]),
        "ccfd_get_history": (c_int, [C.c_void_p, P(c_double), c_long, P(c_long), P(c_int)]),
        "ccfd_write_history": (c_int, [C.c_void_p, P(c_double), c_long, c_int, c_int]),
        "ccfd_locate_points": (c_int, [P(Mesh), P(c_double), c_int, P(c_long)]),
        "ccfd_write_exact_output": (c_int, [C.c_void_p, P(c_double), c_double, c_long, C.c_char_p, C.c_size_t]),
        "ccfd_write_output": (c_int, [C.c_void_p, P(c_double), c_double, c_long, C.c_char_p, C.c_size_t]),
        "ccfd_batch_create": (c_int, [c_int, P(C.c_void_p)]),
        "ccfd_batch_destroy": (None, [C.c_void_p]),
        "ccfd_batch_add": (c_int, [C.c_void_p, C.c_void_p, c_long]),
        "ccfd_batch_remove": (c_int, [C.c_void_p, C.c_void_p]),
        "ccfd_batch_step": (c_int, [C.c_void_p, c_int, P(c_int)]),
        "ccfd_batch_report": (c_int, [C.c_void_p, C.c_void_p, P(Report)]),
        "ccfd_batch_size": (c_int, [C.c_void_p, P(c_int)]),
        "ccfd_estimate_device_bytes": (c_int, [P(Params), P(Mesh), P(C.c_size_t)]),
        "ccfd_device_bytes": (c_int, [C.c_void_p, P(C.c_size_t)]),
        "ccfd_server_create": (c_int, [c_int, C.c_size_t, c_int, P(C.c_void_p)]),
        "ccfd_server_destroy": (None, [C.c_void_p]),
        "ccfd_server_submit": (c_int, [C.c_void_p, C.c_void_p, c_long, P(c_long)]),
        "ccfd_server_poll": (c_int, [C.c_void_p, c_int, P(c_int), P(c_int), P(c_int)]),
        "ccfd_server_result": (c_int, [C.c_void_p, c_long, P(Report), P(c_double), P(c_double)]),
        "ccfd_server_memory": (c_int, [C.c_void_p, P(C.c_size_t), P(C.c_size_t)]),
        "ccfd_server_times": (c_int, [C.c_void_p, P(c_double)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()

PRIMITIVE, CONSERVATIVE = 0, 1
