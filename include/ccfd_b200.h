/*
 * ccfd_b200 -- B200-native residual-and-update path of the 2-D finite-volume
 * Euler / Navier-Stokes solver ccfd (hheinzer/ccfd), behind a C ABI.
 *
 * The reference has no plugin layer: its hot path is a set of global-state C
 * functions.  Each entry point below names the reference function or global it
 * replaces (paths relative to the reference project root).  Everything here is
 * plain C: pointers, sizes and status codes, no CUDA or torch types.  All
 * arrays passed in are owned by the caller and copied; nothing is retained.
 *
 * Threading: a context is used by one host thread at a time; distinct
 * contexts are independent (the reference is single-instance and global).
 * Errors: every call returns a status (0 = CCFD_OK).  The reference prints a
 * message and calls exit(1) instead; ccfd_strerror() gives the message and the
 * C driver (ccfd_run) maps a non-zero status to the same exit(1).
 */
#ifndef CCFD_B200_H
#define CCFD_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status */
enum ccfd_status {
	CCFD_OK = 0,
	CCFD_ERR_ARG = 1,          /* invalid argument / call order            */
	CCFD_ERR_CUDA = 2,         /* CUDA runtime failure                     */
	CCFD_ERR_NOMEM = 3,        /* host or device allocation failed         */
	CCFD_ERR_DT = 4,           /* non-finite time step, timeDiscretization.c:260-263,283-286,302-305 */
	CCFD_ERR_NEWTON = 5,       /* Newton not converged, timeDiscretization.c:544-549 */
	CCFD_ERR_SINGULAR = 6,     /* singular LU-SGS diagonal block, linearSolver.c:245-249 */
	CCFD_ERR_VACUUM = 7,       /* vacuum in exact Riemann solver, exactRiemann.c:77-90 */
	CCFD_ERR_TIMEOUT = 8,      /* bounded device wait gave up              */
	CCFD_ERR_INI = 9,          /* missing / invalid .ini key, readInTools.c:180-184 */
	CCFD_ERR_MESH = 10,        /* mesh read / connectivity error, mesh.c   */
	CCFD_ERR_STATE = 11,       /* non-finite state or residual             */
	CCFD_ERR_BUDGET = 12,      /* request exceeds the device-memory budget */
	CCFD_ERR_UNSUPPORTED = 13, /* option not built (e.g. CGNS output)      */
	CCFD_ERR_NOT_CONVERGED = 14, /* maxIter reached, timeDiscretization.c:737-750 */
	CCFD_ERR_GMRES = 15,         /* GMRES breakdown (zero Hessenberg pivot)  */
	CCFD_ERR_BUSY = 16           /* context is being stepped by a batch      */
};

/* enumerations: numbering identical to the reference's src/main.h */
enum ccfd_flux {               /* src/main.h:76-88 */
	CCFD_FLUX_GODUNOV = 1, CCFD_FLUX_ROE, CCFD_FLUX_HLL, CCFD_FLUX_HLLE,
	CCFD_FLUX_HLLC, CCFD_FLUX_LXF, CCFD_FLUX_STEGER_WARMING,
	CCFD_FLUX_CENTRAL, CCFD_FLUX_AUSMD, CCFD_FLUX_AUSMDV, CCFD_FLUX_VANLEER
};
enum ccfd_limiter {            /* src/main.h:93-96 */
	CCFD_LIM_BARTH_JESPERSEN = 1, CCFD_LIM_VENKATAKRISHNAN = 2
};
enum ccfd_bc_type {            /* src/main.h:44-53; BC code = type*100 + id */
	CCFD_BC_SLIPWALL = 1, CCFD_BC_WALL, CCFD_BC_INFLOW, CCFD_BC_OUTFLOW,
	CCFD_BC_CHARACTERISTIC, CCFD_BC_EXACTSOL, CCFD_BC_PERIODIC,
	CCFD_BC_PRESSURE_OUT
};
enum ccfd_eqn { CCFD_EULER = 0, CCFD_NAVIER_STOKES = 1 }; /* -Deuler / -Dnavierstokes */
enum ccfd_precision {
	CCFD_FP64 = 0,   /* every operation in FP64, as the reference          */
	CCFD_MIXED = 1   /* FP32 face fluxes / sweeps / Krylov basis, FP64
			    accumulation, state, FD difference, Newton update  */
};
enum ccfd_state_kind { CCFD_PRIMITIVE = 0, CCFD_CONSERVATIVE = 1 };

/* ------------------------------------------------------------ parameters */
/* Replaces the globals set by initEquation (src/equation.c:40-124), initFV
 * (src/finiteVolume.c:30-65), initTimeDisc (src/timeDiscretization.c:69-240),
 * initLinearSolver (src/linearSolver.c:68-107) and initAnalyze
 * (src/analyze.c:199-280). */
typedef struct ccfd_params {
	int eqn;               /* enum ccfd_eqn                                 */
	int flux;              /* enum ccfd_flux (fluxFunction)                 */
	int spatial_order;     /* 1 or 2 (spatialOrder)                         */
	int limiter;           /* enum ccfd_limiter (limiter)                   */
	double venk_k;         /* venk_k                                        */
	double gamma, R, mu, Pr;
	int time_order;        /* timeOrder 1..3                                */
	int n_rk_stages;       /* nRKstages 1..5                                */
	double cfl, dfl;
	int time_step_1d;      /* timeStep1D                                    */
	int stationary;        /* stationary                                    */
	double t_end;          /* tEnd                                          */
	long max_iter;         /* maxIter                                       */
	double io_time_interval; /* IOtimeInterval (clamps dt, timeDiscretization.c:317-321) */
	long io_iter_interval;   /* IOiterInterval                              */
	double abort_residual; /* abortResidual (absolute, like the reference)  */
	int abort_variable;    /* 0-based (abortVariable - 1)                   */
	double cl_abort_residual, cd_abort_residual;
	int implicit;          /* implicit                                      */
	int precond;           /* precond (LU-SGS)                              */
	int n_kdim;            /* nKdim                                         */
	int n_newton_iter;     /* nNewtonIter                                   */
	double eps_newton;     /* epsNewton (not squared)                       */
	double eps_gmres;      /* epsGMRES                                      */
	double gamma_ew;       /* gammaEW                                       */
	int calc_wing;         /* calcWing                                      */
	int wall_id;           /* wall_id (BC code of the wing surface)         */
	double ref_length;     /* referenceLength                               */
	int precision;         /* enum ccfd_precision                           */
	double rel_abort_residual; /* >0: stop when res/res_first <= this (extension) */
	int source_func;       /* calcSource / sourceFunction (0: none), src/source.c */
	int exact_solution;    /* exactSolution (error norms at the end of a run) */
	double ser_cfl_max;    /* >0: implicit runs ramp the CFL number by switched
				  evolution relaxation (Mulder and van Leer, 1985):
				  before step n >= 2, CFL = min(ser_cfl_max,
				  CFL_0 * r_1 / r_{n-1}), r the abort variable's
				  global residual after a step, and DFL =
				  DFL_0 * CFL / CFL_0 (extension, key serCFLmax;
				  0: the reference's fixed CFL and DFL) */
} ccfd_params;

/* one boundary condition, src/boundary.h:19-46, parsed by initBoundary
 * (src/boundary.c:29-137) */
typedef struct ccfd_bc {
	int type;              /* enum ccfd_bc_type                             */
	int id;                /* sub id (code % 100)                           */
	int exact_func;        /* BCexactFunc for EXACTSOL                      */
	int is_adiabatic;      /* adiabaticWall (parsed, unused like the reference) */
	double pvar[4];        /* rho, vx, vy, p (inflow / characteristic / pressure) */
	double connection[2];  /* periodic BC: offset to the paired boundary    */
} ccfd_bc;

/* exact-function / initial-condition data used on the device by EXACTSOL
 * ghost states (src/exactFunction.c:35-183) */
typedef struct ccfd_exact {
	double ref_state[2][4];  /* refState[0..1] (1-D Riemann; [0] also sets
				    q_inf of the wing coefficients)           */
	double rp1d_interface;   /* RP_1D_interface                             */
	double alpha;            /* angle of attack in degrees (global alpha of
				    src/initialCondition.c:161)               */
	double x_min, x_max, y_min, y_max, dx_ref;
} ccfd_exact;

/* ------------------------------------------------------------------ mesh */
/* Host view of a mesh in the reference's element / side order, as built by
 * createMesh (src/mesh.c:1405-1844).  Index conventions:
 *   cells       0..n_cells-1 in elem[] order (triangles then quadrilaterals)
 *   faces       0..n_faces-1 in side[] order; the owner is side[f]
 *   half-sides  per cell, CSR in the order of the cell's side list
 *               (elem->firstSide ... nextElemSide), the order of every
 *               per-cell sum of the reference
 *   ghosts      0..n_bc-1 in BCside[] order; a neighbour index < 0 encodes
 *               ghost b as -1-b
 */
typedef struct ccfd_mesh {
	long n_cells, n_faces, n_bc, n_half_sides, n_nodes;
	int *cell_type;        /* [N] 3 or 4                                    */
	int *cell_domain;      /* [N] physical group (IC domain)                */
	double *cell_bary;     /* [N][2]                                        */
	double *cell_geo;      /* [N][4] area, 1/area, sx, sy                   */
	long *hs_offset;       /* [N+1]                                         */
	long *hs_face;         /* [H] face of the half-side                     */
	int *hs_sign;          /* [H] +1: cell owns the face, -1: neighbour     */
	long *hs_nb;           /* [H] neighbour cell or -1-ghost                */
	double *hs_gp;         /* [H][2] bary -> face midpoint (side->GP)       */
	double *hs_w;          /* [H][2] least-squares weights (side->w)        */
	long *face_cells;      /* [F][2] owner cell, neighbour cell or -1-ghost */
	long *face_hs;         /* [F][2] owner half-side, neighbour half-side or -1 */
	double *face_n;        /* [F][2] unit normal, outward of the owner      */
	double *face_len;      /* [F]                                           */
	double *face_bb;       /* [F][3] owner side baryBaryVec x, y, baryBaryDist */
	double *ghost_gp;      /* [B][2] ghost side GP (face midpoint - ghost bary) */
	long *bc_face;         /* [B] face of the ghost                          */
	int *bc_index;         /* [B] index into the BC table                   */
	double *bc_ghost_bary; /* [B][2] mirrored ghost barycentre              */
	double *bc_x;          /* [B][2] face midpoint, side->GP + elem->bary   */
	double *cell_gp5;      /* [N][2] fifth quadrature point of a quad (midpoint
				  of its nodes 0 and 2, src/mesh.c:157-160);
				  the barycentre for triangles                */
	long *cell_nodes;      /* [N][4] element node ids (quads: 4, triangles:
				  3 and -1)                                   */
	double *node_xy;       /* [n_nodes][2] node coordinates                 */
	double total_area_q, dx_ref, x_min, x_max, y_min, y_max;
} ccfd_mesh;

/* Most record points of a case (the reference has no limit). */
#define CCFD_MAX_RECORD 64

/* A complete case: parameters, boundary table, mesh and initial state, as
 * the reference's init sequence (src/main.c:101-118) produces them. */
typedef struct ccfd_case {
	ccfd_params params;
	int n_bc_table;
	ccfd_bc bc_table[20];  /* NBC = 20, src/main.h:103                      */
	ccfd_exact exact;
	ccfd_mesh mesh;
	double *prim0;         /* [N][4] initial primitive state                */
	char file_name[256];   /* fileName                                      */
	int output_format;     /* outputFormat                                  */
	int ic_type, exact_func;
	int n_record;          /* nRecordPoints (src/analyze.c:283-286)         */
	double record_xy[CCFD_MAX_RECORD][2]; /* pointCoords                    */
	long record_cell[CCFD_MAX_RECORD];    /* containing cell (elem order)   */
} ccfd_case;

/* -------------------------------------------------------- host-side API */
/* Read a .ini parameter file with the reference's parser semantics
 * (src/readInTools.c:38-405: case-insensitive keys, values filtered to
 * [alnum _ . , -], keys consumed in read order) and build the full case
 * exactly as initOutput..setInitialCondition do, including the Cartesian
 * generator (src/mesh.c:385-486) or the gmsh 2/4 reader (src/mesh.c:498-992)
 * and createMesh (src/mesh.c:1405-1844).  Replaces main()'s init sequence. */
int ccfd_case_load(const char *ini_path, ccfd_case **out);
/* Same, from .ini text held in memory; relative mesh paths resolve against
 * base_dir (may be NULL). */
int ccfd_case_load_text(const char *ini_text, const char *base_dir, ccfd_case **out);
/* Build the mesh part of a case from raw elements (what a mesh reader
 * returns): nodes [n_nodes][2], triangles [n_tri][4] (3 nodes + domain),
 * quads [n_quad][5] (4 nodes + domain), BC edges [n_edge][3] (2 nodes + code).
 * Node indices are 0-based.  Replaces createMesh (src/mesh.c:1405-1844). */
int ccfd_mesh_build(const double *nodes, long n_nodes,
		    const long *tria, long n_tria, const long *quad, long n_quad,
		    const long *bc_edge, long n_bc_edge,
		    const ccfd_bc *bc_table, int n_bc_table, ccfd_mesh *out);
void ccfd_mesh_free(ccfd_mesh *m);
void ccfd_case_free(ccfd_case *c);
/* Venkatakrishnan epsilon^2 per cell, (K sqrt(A))^3, src/finiteVolume.c:47-52 */
void ccfd_venk_eps2(const ccfd_mesh *m, double venk_k, double *eps2_out);
/* The cell holding each point, as initRecordPoints finds it
 * (src/analyze.c:43-82): the first cell in element order for which no edge
 * has the point strictly on its outer side, with the reference's edge-normal
 * arithmetic.  CCFD_ERR_MESH if a point lies in no cell. */
int ccfd_locate_points(const ccfd_mesh *m, const double *xy, int n, long *cells_out);
/* Write a gmsh 2.2 ASCII mesh (the format src/mesh.c:498-742 reads). */
int ccfd_write_gmsh2(const char *path, const double *nodes, long n_nodes,
		     const long *tria, long n_tria, const long *quad, long n_quad,
		     const long *bc_edge, long n_bc_edge);
/* Read a gmsh 2.2 or 4 ASCII mesh into raw arrays as readGmsh does
 * (src/mesh.c:498-983; gmsh 4: boundary codes are the curves' physical
 * tags, cells domain 1); the caller frees them with free(). */
int ccfd_read_gmsh(const char *path, double **nodes, long *n_nodes,
		   long **tria, long *n_tria, long **quad, long *n_quad,
		   long **bc_edge, long *n_bc_edge);
/* Read an EMC2 (.mesh) mesh as readEMC2 does (src/mesh.c:1004-1139):
 * edges with reference 0 are not boundary edges; element references are
 * their domains.  Same outputs as ccfd_read_gmsh. */
int ccfd_read_emc2(const char *path, double **nodes, long *n_nodes,
		   long **tria, long *n_tria, long **quad, long *n_quad,
		   long **bc_edge, long *n_bc_edge);
const char *ccfd_strerror(int status);

/* ------------------------------------------------------ device context */
typedef struct ccfd_ctx ccfd_ctx;

/* Run report of an explicit or implicit run (the quantities timeDisc prints,
 * src/timeDiscretization.c:559-777). */
typedef struct ccfd_report {
	double t;              /* simulation time reached                       */
	double dt;             /* last time step                                */
	long iterations;       /* time steps taken                              */
	double residual[6];    /* resIter: L2 residual of RHO, MX, MY, E; CL, CD rates */
	double cl, cd;         /* wing coefficients (calcWing)                  */
	int converged;         /* stationary: abort criterion met               */
	int finished;          /* transient: tEnd reached                       */
	long newton_iterations, gmres_iterations;
	double first_residual[4]; /* resIter of the first step (relative stop)  */
	int status;            /* device error status                          */
	double device_ms;      /* device time of the call (CUDA events on the
				  context's stream, first launch to last)      */
} ccfd_report;

/* Select the CUDA device for the calling host thread (cudaSetDevice); the
 * next ccfd_create binds its context to it.  No counterpart in the reference
 * (single-process CPU code). */
int ccfd_set_device(int device);
/* Create a context on the current CUDA device.  Replaces the init* globals. */
int ccfd_create(const ccfd_params *params, ccfd_ctx **out);
void ccfd_destroy(ccfd_ctx *ctx);
/* Upload mesh connectivity / geometry once (mesh.c output -> device
 * arrays), boundary table and exact-function data.  Cells (and faces, by
 * owner) are stored in a locality order: reorder = 0 the reference's
 * numbering, 1 a Hilbert curve through the barycentres (the fastest
 * measured), 2 reverse Cuthill-McKee on the face-neighbour graph; results
 * are independent of the ordering. */
int ccfd_upload_case(ccfd_ctx *ctx, const ccfd_mesh *mesh, const ccfd_bc *bc,
		     int n_bc, const ccfd_exact *exact, int reorder);
/* State in reference cell order, [N][4], primitive or conservative.  Setting
 * primitives also sets cVar = primCons(pVar) like setInitialCondition
 * (src/initialCondition.c:346-350); setting conservatives sets
 * pVar = consPrim(cVar).  Returns once the array has been copied (the caller
 * may reuse it); the conversion finishes on the context's stream before any
 * later call on the context reads the state.  A failure of that conversion
 * kernel is therefore not seen by this call: the next call on the context
 * that synchronises its stream (a run, a residual, ccfd_get_state) returns
 * it as CCFD_ERR_CUDA. */
int ccfd_set_state(ccfd_ctx *ctx, const double *state, int kind);
int ccfd_get_state(ccfd_ctx *ctx, double *state, int kind);
/* Set / get the simulation time t (src/timeDiscretization.c:31). */
int ccfd_set_time(ccfd_ctx *ctx, double t);
int ccfd_get_time(ccfd_ctx *ctx, double *t);
/* Drop-in for fvTimeDerivative(time) (src/finiteVolume.c:78-121): evaluates
 * R(U) from the current primitive state; u_t_out ([N][4], reference order)
 * may be NULL to keep the result on the device.  grad_out ([N][8]: u_x[4],
 * u_y[4]) may be NULL. */
int ccfd_residual(ccfd_ctx *ctx, double time, double *u_t_out, double *grad_out);
/* Drop-in for calcTimeStep (src/timeDiscretization.c:249-329). */
int ccfd_time_step(ccfd_ctx *ctx, double *dt_out);
/* Explicit time stepping: up to nsteps iterations of the loop in timeDisc
 * (src/timeDiscretization.c:595-731) with explicitTimeStepEuler / RK
 * (:337-401), calcTimeStep and globalResidual (src/analyze.c:521-539) on the
 * device, captured as CUDA graphs.  nsteps <= 0 runs until tEnd, convergence
 * or maxIter. */
int ccfd_run_explicit(ccfd_ctx *ctx, long nsteps, ccfd_report *report);
/* Implicit backward-Euler stepping: implicitTimeStep
 * (src/timeDiscretization.c:412-552) with GMRES_M (src/linearSolver.c:
 * 385-510), matrixVector (:343-373) and, if params.precond, the LU-SGS
 * preconditioner (buildMatrix :186-252, calcDinv :136-179, LUSGS :261-333)
 * on block-sparse storage.  With params.ser_cfl_max > 0 the CFL number of
 * each step follows switched evolution relaxation (see ccfd_params). */
int ccfd_run_implicit(ccfd_ctx *ctx, long nsteps, ccfd_report *report);
/* buildMatrix + calcDinv (src/linearSolver.c:186-252, :136-179) at the
 * context's state, as at the first Newton iteration of an implicit step from
 * time t with step dt: R_XK = R(U, t + dt), the finite-difference columns
 * R(U + sqrt(DBL_EPSILON) e_k, t) of the primitive variables (mixed
 * precision: columns and their base R(U, t) with FP32 reconstruction and
 * fluxes, step sqrt(FLT_EPSILON); FP32 blocks).  Out (each may
 * be NULL), reference cell order, row-major 4x4 blocks (rows: residual
 * variables, columns: perturbed primitive variables): d and dinv [N][16],
 * the diagonal blocks of I - dt dR/dU and their inverses; off [H][16], per
 * half-side (reference side order) the block of its cell's row and the
 * column of the cell across it (zero at boundary sides).  Needs implicit
 * and precond.  CCFD_ERR_SINGULAR as calcDinv's exit. */
int ccfd_build_matrix(ccfd_ctx *ctx, double t, double dt, double *d, double *dinv, double *off);
/* LUSGS (src/linearSolver.c:261-333): x = M^-1 b with the blocks of the last
 * ccfd_build_matrix, b and x [N][4] in reference cell order (mixed
 * precision: the sweep runs on the FP32 blocks). */
int ccfd_lusgs(ccfd_ctx *ctx, const double *b, double *x);
/* The column grouping of the block-sparse buildMatrix: a distance-3
 * colouring of the face-neighbour graph (the reference evaluates one column
 * per residual, src/linearSolver.c:186-252; columns of cells more than three
 * face-neighbour steps apart are evaluated in one residual pass).  hs_offset
 * [n_cells + 1] and hs_nb (negative: boundary side) as in ccfd_mesh; budget:
 * candidate moves (cell, colour) the tabu search examines per colour-removal
 * attempt, 0 for greedy only, negative for the default the solver uses.
 * Out: color_out [n_cells], *n_colors.  Host only. */
int ccfd_colour_cells(long n_cells, const long *hs_offset, const long *hs_nb, long budget,
                      int *color_out, int *n_colors);
/* Profiling of the residual evaluations inside the timed step graphs: with
 * profiling on, every residual evaluation of a step (gradient, face flux and
 * update kernels of one Runge-Kutta stage) is bracketed by CUDA events on the
 * context's stream; ccfd_get_profile returns the accumulated device time and
 * count since the last reset.  No counterpart in the reference (its timer is
 * the wall clock around the time loop, src/timeDiscretization.c:583,734). */
int ccfd_set_profiling(ccfd_ctx *ctx, int on);
int ccfd_get_profile(ccfd_ctx *ctx, double *residual_ms, long *residual_count,
		     int reset);
/* Drop-in for globalResidual on the last residual (src/analyze.c:521-539). */
int ccfd_global_residual(ccfd_ctx *ctx, double res[4]);

/* Pressure coefficient along the wall params.wall_id (the CP part of
 * calcCoef, src/analyze.c:296-367), from the last residual evaluation: per
 * wall face in calcCoef's order (pressure side by increasing x, then suction
 * side) its point x, y and cp.  *n receives the face count, *n_pressure
 * (may be NULL) the pressure-side count; with x == NULL only the counts. */
int ccfd_wall_cp(ccfd_ctx *ctx, double *x, double *y, double *cp, int *n, int *n_pressure);
/* The reference's CP files <base>_CP_pressureSide.csv / _CP_suctionSide.csv
 * (rows x, y, phi, cp). */
int ccfd_write_cp(ccfd_ctx *ctx, const char *base);

/* Per-step history, the data of analyze (src/analyze.c:393-433): with
 * capacity > 0 every following step (explicit, implicit, alone or in a
 * batch) records one row of width 11 + 4 * n_record doubles: iteration, t
 * after the step, dt, the six residuals (four variables, CL, CD), CL, CD,
 * then rho, vx, vy, p of each record cell (reference cell index, e.g. from
 * ccfd_locate_points).  The device keeps a ring of `capacity` rows (at least
 * 64); runs move the rows to the host after each synchronisation.
 * capacity <= 0 switches it off.  ccfd_upload_case / ccfd_autotune reset
 * it.  A batch call may not step further than the ring holds. */
int ccfd_set_history(ccfd_ctx *ctx, int capacity, const long *record_cells, int n_record);
/* Moves up to max_rows recorded rows (oldest first) into rows and drops
 * them; *n_rows gets the count and *width (may be NULL) the row width.
 * rows == NULL: only the number waiting. */
int ccfd_get_history(ccfd_ctx *ctx, double *rows, long max_rows, long *n_rows, int *width);
/* The files analyze writes from those rows: <fileName>_analysis.csv (for
 * stationary runs or calcWing, with its gnuplot scripts
 * <fileName>_residuals.dem / _CLCD.dem, src/analyze.c:205-281, 411-433) and
 * <fileName>_recordPoint_<k>.csv (src/analyze.c:84-89, 393-403), with
 * their headers when `append` is 0. */
int ccfd_write_history(const ccfd_case *c, const double *rows, long n_rows, int width, int append);

/* Drop-in for calcErrors (src/analyze.c:445-514) at the current time: L1,
 * L2 and Linf norms of the primitive variables against exact function
 * exact_func (the case's exactFunc), over the element quadrature points
 * with the solution expanded by the limited gradients of the current
 * state.  out = {L1[4], L2[4], Linf[4]}.  Allocates a per-call partial-sum
 * buffer (stream-ordered). */
int ccfd_errors(ccfd_ctx *ctx, int exact_func, double out[12]);

/* Autotuner (no counterpart in the reference): re-uploads the case with
 * each candidate launch shape of the stage kernel (cells per tile 128..384,
 * Hilbert or reference cell order) and times residual evaluations of state
 * prim ([n_cells][4] primitive, reference order) at each CTA size (FP64
 * 256 / 320 / 384 threads, FP32 fluxes 128 / 192 / 256, so cells and faces
 * per thread vary with the tile), keeps the fastest; the context ends
 * uploaded with that shape and with prim as its state.  Results are
 * independent of the shape.  Outputs may be NULL. */
int ccfd_autotune(ccfd_ctx *ctx, const ccfd_mesh *m, const ccfd_bc *bc, int n_bc,
		  const ccfd_exact *ex, const double *prim, int *tile_cells, int *reorder,
		  int *threads, double *ms_per_residual);

/* Final-solution output in the reference's format (dataOutput, csvOutput,
 * curveOutput, src/output.c:53-112, 253-398): outputFormat = 3 (CSV) or 2
 * (curve), named <fileName>_<iter %09ld>.<ext> (stationary) or
 * <fileName>_<time %015.7f>.<ext>; prim is [n_cells][4] in reference order;
 * the file name is returned in path (may be NULL).  CCFD_ERR_UNSUPPORTED for
 * CGNS. */
int ccfd_write_output(const ccfd_case *c, const double *prim, double time, long iter,
		      char *path, size_t path_len);
/* The exact-solution file that dataOutput adds with exactSolution = T
 * (<fileName>_ex_...), from the exact state of ccfd_exact_state. */
int ccfd_write_exact_output(const ccfd_case *c, const double *prim_exact, double time, long iter,
			    char *path, size_t path_len);
/* Exact function exact_func (exactFunc, src/exactFunction.c:35-183) at the
 * cell barycentres at time `time`, evaluated on the device: [n_cells][4]
 * primitive state in reference order (what csvOutput / curveOutput write
 * for the exact solution). */
int ccfd_exact_state(ccfd_ctx *ctx, int exact_func, double time, double *prim_out);

/* ------------------------------------------------------------- batching
 * Many contexts stepped together on one GPU (no counterpart in the
 * reference, which runs one case per process).  A member is an uploaded
 * context; while it is in a batch, the batch owns it: ccfd_run_*,
 * ccfd_set_state, ccfd_residual and ccfd_set_time return CCFD_ERR_BUSY,
 * ccfd_get_state and ccfd_batch_report read its current state and control
 * block.  Explicit members advance in multi-instance stage launches over
 * their concatenated tiles (one launch per kernel variant and RK stage,
 * replayed from a CUDA graph); implicit members advance in lockstep Newton /
 * GMRES / LU-SGS iterations whose kernels cover every member at once.  Each
 * member keeps its own time step, CFL, stop criteria and flags. */
typedef struct ccfd_batch ccfd_batch;
int ccfd_batch_create(int device, ccfd_batch **out);
void ccfd_batch_destroy(ccfd_batch *b);   /* releases the members too */
/* join with a budget of nsteps time steps (<= 0: until the member stops) */
int ccfd_batch_add(ccfd_batch *b, ccfd_ctx *ctx, long nsteps);
int ccfd_batch_remove(ccfd_batch *b, ccfd_ctx *ctx);
/* advance every running member by up to `steps` time steps; *n_running
 * receives the number of members that can still step */
int ccfd_batch_step(ccfd_batch *b, int steps, int *n_running);
/* a member's report (device_ms: the batch's accumulated device time) */
int ccfd_batch_report(ccfd_batch *b, ccfd_ctx *ctx, ccfd_report *r);
int ccfd_batch_size(ccfd_batch *b, int *n);

/* ------------------------------------------------------------- serving
 * A request loop with continuous batching (no counterpart in the reference).
 * Requests queue in arrival order; ccfd_server_poll admits them first come,
 * first served while their estimated device memory fits the budget and fewer
 * than max_running run, uploads each into its own context, steps all running
 * requests together in one batch, and retires the ones that stopped (final
 * state copied to the host, device memory released). */
typedef struct ccfd_server ccfd_server;
/* device memory a case will hold once uploaded (an upper estimate) */
int ccfd_estimate_device_bytes(const ccfd_params *p, const ccfd_mesh *m, size_t *bytes);
/* device memory a context holds */
int ccfd_device_bytes(ccfd_ctx *ctx, size_t *bytes);
int ccfd_server_create(int device, size_t hbm_budget_bytes, int max_running, ccfd_server **out);
void ccfd_server_destroy(ccfd_server *s);
/* queue case c (kept alive by the caller until its result is fetched) with
 * a budget of nsteps steps (<= 0: until it stops); CCFD_ERR_BUDGET if it
 * can never fit */
int ccfd_server_submit(ccfd_server *s, const ccfd_case *c, long nsteps, long *id);
/* admit, advance the running requests by up to `steps` steps, retire */
int ccfd_server_poll(ccfd_server *s, int steps, int *n_queued, int *n_running, int *n_done);
/* a finished request: report, final primitive state [n_cells][4] (may be
 * NULL), times {submit, admit, done} in seconds of a monotonic host clock
 * (may be NULL); returns the request's status and forgets it, or
 * CCFD_ERR_BUSY while it is queued or running */
int ccfd_server_result(ccfd_server *s, long id, ccfd_report *rep, double *prim, double times[3]);
int ccfd_server_memory(ccfd_server *s, size_t *used, size_t *budget);
/* host seconds spent so far admitting (upload), stepping and retiring */
int ccfd_server_times(ccfd_server *s, double out[3]);

/* Largest cell count of ccfd_global_residual_noalloc (its static scratch
 * holds one 4-double partial sum per 256 cells: 128 KB). */
#define CCFD_NOALLOC_MAX_CELLS (1L << 20)
/* Allocation-free global residual, for callers that cannot allocate device
 * memory (a host application whose own pool allocator owns the device heap,
 * or a serving loop whose device-memory budget is already committed to
 * resident states).  No counterpart in the reference.  Inputs and output are
 * device memory owned by the caller: u_t [n_cells][4] (residual field), area
 * [n_cells] (cell areas), res [4] receives sqrt(sum(area * u_t^2) *
 * total_area_q) per variable.  stream is a cudaStream_t (NULL: legacy default
 * stream); the result is ready when the stream is.  Allocates nothing: the
 * partial sums live in a file-scope device array that every device loading
 * the library keeps until exit.  The first call on a device looks up that
 * array's device address (cudaGetSymbolAddress, with the device current), so
 * make the first call on each device before any stream capture.  That
 * address is kept for the life of the process: do not reset a device
 * (cudaDeviceReset) while this library is loaded.  All calls
 * share the array: calls that overlap on the GPU race.  Returns CCFD_ERR_ARG
 * for n_cells <= 0 or n_cells > CCFD_NOALLOC_MAX_CELLS. */
int ccfd_global_residual_noalloc(const double *u_t, const double *area, long n_cells,
				 double total_area_q, double *res, void *stream);
/* Lift / drag of the wall with BC code params.wall_id: the sums of calcCoef
 * (src/analyze.c:292-387) over the reconstructed wall-face pressures of the
 * last residual, with q_inf from exact.ref_state[0] and exact.alpha. */
int ccfd_clcd(ccfd_ctx *ctx, double *cl, double *cd);

#ifdef __cplusplus
}
#endif
#endif
