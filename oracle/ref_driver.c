/*
 * Test-oracle driver for the reference ccfd solver (hheinzer/ccfd).
 *
 * TEST INFRASTRUCTURE ONLY.  This program links the reference's own,
 * unmodified sources (src/*.c except main.c, compiled by oracle/Makefile into
 * oracle/_ref/) and calls its global-state functions directly, so that the
 * CUDA path can be checked against the reference's FP64 OpenMP code on
 * identical inputs.  It is never part of the product.
 *
 * Usage:  ccfd_ref <case.ini> <out.dump> <mode> [args...]
 *   mesh                 dump mesh geometry / connectivity and initial state
 *   residual <t> [state] one fvTimeDerivative(t) (src/finiteVolume.c:78); an
 *                        optional raw f64 file of N*4 primitive states (cell
 *                        order) replaces the initial condition first
 *   run <nsteps> [state] the time loop of timeDisc (src/timeDiscretization.c:
 *                        559-732) without file output, at most nsteps
 *                        iterations (<=0: until tEnd / convergence)
 *   coef                 like run, plus calcCoef (src/analyze.c:292) per step
 *                        (CCFD_REF_REL_ABORT=<r>: stationary runs also stop
 *                        once the abort variable's residual is at most r
 *                        times the first step's)
 *                        run / coef end with calcErrors (src/analyze.c:445)
 *                        when the case has an exact solution
 *
 * The initialisation order mirrors main() (src/main.c:53-118).  Output format
 * CGNS is replaced by CSV so that the CGNS stand-in is never reached; with
 * CCFD_REF_OUTPUT set in the environment, run / coef call the reference's
 * analyze every step (residual file, record points, CL / CD) and end with
 * dataOutput (solution file, and exact-solution file with exactSolution =
 * T).
 *
 *   jacobian <t> <dt> [state] [vector]
 *                        buildMatrix(t, dt) (src/linearSolver.c:186-252) at
 *                        the state, with R_XK = fvTimeDerivative(t + dt) as
 *                        at the first Newton iteration of implicitTimeStep;
 *                        dumps the diagonal blocks D, their inverses Dinv,
 *                        the face-neighbour blocks of the dense dRdU per
 *                        half-side, the state after buildMatrix (it perturbs
 *                        and restores pVar in place) and, given a raw f64
 *                        vector file (N*4, cell order), LUSGS of it
 *                        (src/linearSolver.c:261-333); needs precond = T
 *
 * Dump format: magic "CCFDDMP1", then records of
 *   char name[32]; int32 type (0 = f64, 1 = i64); int32 pad; int64 count; data
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include <stdbool.h>
#include <omp.h>

#include "main.h"
#include "readInTools.h"
#include "timeDiscretization.h"
#include "output.h"
#include "equation.h"
#include "boundary.h"
#include "mesh.h"
#include "initialCondition.h"
#include "finiteVolume.h"
#include "reconstruction.h"
#include "linearSolver.h"
#include "analyze.h"
#include "equationOfState.h"

/* reference functions with external linkage but no header declaration */
void calcTimeStep(double pTime, double *dt, bool *viscousTimeStepDominates);
void explicitTimeStepEuler(double time, double dt, double resIter[NVAR + 2]);
void explicitTimeStepRK(double time, double dt, double resIter[NVAR + 2]);
void implicitTimeStep(double time, double dt, double resIter[NVAR + 2]);
void calcCoef(void);
void buildMatrix(double time, double dt);
void LUSGS(double **B, double **delX);
extern double ***D;
extern double ***Dinv;
extern double **dRdU;

static FILE *dumpFile;

static void dump_rec(const char *name, int type, const void *data, long count)
{
	char nm[32] = {0};
	strncpy(nm, name, 31);
	int hdr[2] = {type, 0};
	long cnt = count;
	fwrite(nm, 1, 32, dumpFile);
	fwrite(hdr, sizeof(int), 2, dumpFile);
	fwrite(&cnt, sizeof(long), 1, dumpFile);
	if (count > 0)
		fwrite(data, 8, count, dumpFile);
}

static void dump_f64(const char *name, const double *d, long n) { dump_rec(name, 0, d, n); }
static void dump_i64(const char *name, const long *d, long n) { dump_rec(name, 1, d, n); }

static void dump_scalar(const char *name, double v) { dump_f64(name, &v, 1); }

static void dump_state(void)
{
	double *pv = malloc(sizeof(double) * 4 * nElems);
	double *cv = malloc(sizeof(double) * 4 * nElems);
	double *ut = malloc(sizeof(double) * 4 * nElems);
	double *ux = malloc(sizeof(double) * 4 * nElems);
	double *uy = malloc(sizeof(double) * 4 * nElems);
	for (long i = 0; i < nElems; ++i)
		for (int v = 0; v < 4; ++v) {
			pv[4 * i + v] = elem[i]->pVar[v];
			cv[4 * i + v] = elem[i]->cVar[v];
			ut[4 * i + v] = elem[i]->u_t[v];
			ux[4 * i + v] = elem[i]->u_x[v];
			uy[4 * i + v] = elem[i]->u_y[v];
		}
	dump_f64("pvar", pv, 4 * nElems);
	dump_f64("cvar", cv, 4 * nElems);
	dump_f64("u_t", ut, 4 * nElems);
	dump_f64("u_x", ux, 4 * nElems);
	dump_f64("u_y", uy, 4 * nElems);
	free(pv); free(cv); free(ut); free(ux); free(uy);

	/* per-face states and fluxes, in side[] order (owner, then connection) */
	double *fs = malloc(sizeof(double) * 8 * nSides);
	double *ff = malloc(sizeof(double) * 4 * nSides);
	for (long s = 0; s < nSides; ++s) {
		for (int v = 0; v < 4; ++v) {
			fs[8 * s + v] = side[s]->pVar[v];
			fs[8 * s + 4 + v] = side[s]->connection->pVar[v];
			ff[4 * s + v] = side[s]->flux[v];
		}
	}
	dump_f64("face_pvar", fs, 8 * nSides);
	dump_f64("face_flux", ff, 4 * nSides);
	free(fs); free(ff);

	/* ghost cell primitive states at barycentres, BCside order */
	double *gp = malloc(sizeof(double) * 4 * (nBCsides + 1));
	for (long b = 0; b < nBCsides; ++b)
		for (int v = 0; v < 4; ++v)
			gp[4 * b + v] = BCside[b]->elem->pVar[v];
	dump_f64("ghost_pvar", gp, 4 * nBCsides);
	free(gp);
}

static void dump_mesh(void)
{
	long n = nElems;
	long *etype = malloc(sizeof(long) * n);
	long *edomain = malloc(sizeof(long) * n);
	double *bary = malloc(sizeof(double) * 2 * n);
	double *geo = malloc(sizeof(double) * 5 * n);
	long nhs = 0;
	for (long i = 0; i < n; ++i)
		nhs += elem[i]->elemType;
	long *hs_off = malloc(sizeof(long) * (n + 1));
	long *hs_id = malloc(sizeof(long) * nhs);
	long *hs_conn_elem = malloc(sizeof(long) * nhs);
	long *hs_conn_id = malloc(sizeof(long) * nhs);
	long *hs_bc = malloc(sizeof(long) * nhs);
	double *hs_geo = malloc(sizeof(double) * 12 * nhs);
	long k = 0;
	for (long i = 0; i < n; ++i) {
		elem_t *e = elem[i];
		etype[i] = e->elemType;
		edomain[i] = e->domain;
		bary[2 * i] = e->bary[X];
		bary[2 * i + 1] = e->bary[Y];
		geo[5 * i + 0] = e->area;
		geo[5 * i + 1] = e->areaq;
		geo[5 * i + 2] = e->sx;
		geo[5 * i + 3] = e->sy;
		geo[5 * i + 4] = e->venkEps_sq;
		hs_off[i] = k;
		for (side_t *s = e->firstSide; s; s = s->nextElemSide, ++k) {
			hs_id[k] = s->id;
			hs_conn_elem[k] = s->connection->elem->id;
			hs_conn_id[k] = s->connection->id;
			hs_bc[k] = s->connection->BC ?
				s->connection->BC->BCtype * 100 + s->connection->BC->BCid : 0;
			double *g = &hs_geo[12 * k];
			g[0] = s->GP[X]; g[1] = s->GP[Y];
			g[2] = s->w[X]; g[3] = s->w[Y];
			g[4] = s->n[X]; g[5] = s->n[Y];
			g[6] = s->len;
			g[7] = s->baryBaryVec[X]; g[8] = s->baryBaryVec[Y];
			g[9] = s->baryBaryDist;
			g[10] = s->connection->elem->bary[X];
			g[11] = s->connection->elem->bary[Y];
		}
	}
	hs_off[n] = k;
	dump_i64("elem_type", etype, n);
	dump_i64("elem_domain", edomain, n);
	dump_f64("elem_bary", bary, 2 * n);
	dump_f64("elem_geo", geo, 5 * n);
	dump_i64("hs_off", hs_off, n + 1);
	dump_i64("hs_id", hs_id, nhs);
	dump_i64("hs_conn_elem", hs_conn_elem, nhs);
	dump_i64("hs_conn_id", hs_conn_id, nhs);
	dump_i64("hs_bc", hs_bc, nhs);
	dump_f64("hs_geo", hs_geo, 12 * nhs);

	long *f_owner = malloc(sizeof(long) * 4 * nSides);
	double *f_geo = malloc(sizeof(double) * 3 * nSides);
	for (long s = 0; s < nSides; ++s) {
		f_owner[4 * s + 0] = side[s]->id;
		f_owner[4 * s + 1] = side[s]->elem->id;
		f_owner[4 * s + 2] = side[s]->connection->id;
		f_owner[4 * s + 3] = side[s]->connection->elem->id;
		f_geo[3 * s + 0] = side[s]->n[X];
		f_geo[3 * s + 1] = side[s]->n[Y];
		f_geo[3 * s + 2] = side[s]->len;
	}
	dump_i64("face_sides", f_owner, 4 * nSides);
	dump_f64("face_geo", f_geo, 3 * nSides);

	long *bc_ids = malloc(sizeof(long) * (nBCsides + 1));
	for (long b = 0; b < nBCsides; ++b)
		bc_ids[b] = BCside[b]->id;
	dump_i64("bcside_id", bc_ids, nBCsides);

	double sc[8] = {totalArea_q, dxRef, xMin, xMax, yMin, yMax, gam, mu};
	dump_f64("mesh_scalars", sc, 8);
	long cnt[4] = {nElems, nSides, nBCsides, nNodes};
	dump_i64("counts", cnt, 4);

	free(etype); free(edomain); free(bary); free(geo); free(hs_off);
	free(hs_id); free(hs_conn_elem); free(hs_conn_id); free(hs_bc);
	free(hs_geo); free(f_owner); free(f_geo); free(bc_ids);
}

static void load_state(const char *path)
{
	FILE *f = fopen(path, "rb");
	if (!f) {
		fprintf(stderr, "ccfd_ref: cannot open state file %s\n", path);
		exit(2);
	}
	double *pv = malloc(sizeof(double) * 4 * nElems);
	if (fread(pv, sizeof(double), 4 * nElems, f) != (size_t)(4 * nElems)) {
		fprintf(stderr, "ccfd_ref: short state file %s\n", path);
		exit(2);
	}
	fclose(f);
	for (long i = 0; i < nElems; ++i) {
		for (int v = 0; v < 4; ++v)
			elem[i]->pVar[v] = pv[4 * i + v];
		primCons(elem[i]->pVar, elem[i]->cVar);
	}
	free(pv);
}

int main(int argc, char *argv[])
{
	if (argc < 4) {
		fprintf(stderr, "usage: ccfd_ref <case.ini> <out.dump> <mode> [args]\n");
		return 2;
	}
	const char *mode = argv[3];

	fillCmds(argv[1]);
	isStationary = getBool("stationary", "T");
	isRestart = false;
	iniIterationNumber = 0;
	startTime = 0.0;

	initOutput();
	if (iVisuProg != CURVE)
		iVisuProg = CSV;
	initEquation();
	initBoundary();
	initMesh();
	initInitialCondition();
	initFV();
	initTimeDisc();
	initLinearSolver();
	outputTimes = NULL;
	setInitialCondition();
	initAnalyze();
	ignoredCmds();

	dumpFile = fopen(argv[2], "wb");
	if (!dumpFile) {
		fprintf(stderr, "ccfd_ref: cannot open %s\n", argv[2]);
		return 2;
	}
	fwrite("CCFDDMP1", 1, 8, dumpFile);

	if (!strcmp(mode, "mesh")) {
		dump_mesh();
		dump_state();
	} else if (!strcmp(mode, "residual")) {
		double time = argc > 4 ? strtod(argv[4], NULL) : 0.0;
		if (argc > 5)
			load_state(argv[5]);
		/* the reference sets elem->dt in calcTimeStep before any residual */
		double dt;
		bool visc;
		calcTimeStep(printTime, &dt, &visc);
		double t0 = omp_get_wtime();
		fvTimeDerivative(time);
		double t1 = omp_get_wtime();
		double res[NVAR + 2];
		globalResidual(res);
		dump_state();
		dump_f64("global_residual", res, 4);
		dump_scalar("wall_s", t1 - t0);
		dump_scalar("dt", dt);
	} else if (!strcmp(mode, "run") || !strcmp(mode, "coef")) {
		bool doCoef = !strcmp(mode, "coef");
		bool write_out = getenv("CCFD_REF_OUTPUT") != NULL;
		const char *rel = getenv("CCFD_REF_REL_ABORT");
		double relAbort = rel ? strtod(rel, NULL) : 0.0, relFirst = 0.0;
		/* switched evolution relaxation of the CFL number (Mulder and van
		 * Leer, 1985) around the reference's own step: before step n >= 2,
		 * cfl = min(cap, CFL_0 * r_1 / r_{n-1}), r the abort variable's
		 * residual after a step (the reference's global cfl,
		 * src/timeDiscretization.c:72, read by calcTimeStep), and the
		 * viscous number follows, dfl = DFL_0 * cfl / CFL_0 */
		const char *ser = getenv("CCFD_REF_SER_CFL_MAX");
		double serMax = ser ? strtod(ser, NULL) : 0.0, cfl0 = cfl, dfl0 = dfl, serFirst = 0.0,
		       serPrev = 0.0;
		long nsteps = argc > 4 ? strtol(argv[4], NULL, 10) : 0;
		if (argc > 5)
			load_state(argv[5]);
		bool visc;
		double dt;
		calcTimeStep(printTime, &dt, &visc);
		double resIter[NVAR + 2] = {0.0};
		double *hist = malloc(sizeof(double) * 8 * (maxIter + 2));
		double *wall = malloc(sizeof(double) * (maxIter + 2));
		long iter, nhist = 0;
		bool converged = false;
		double tStart = omp_get_wtime();
		for (iter = 1; iter <= maxIter; ++iter) {
			if (nsteps > 0 && iter > nsteps)
				break;
			if (serMax > 0.0 && iter >= 2 && serPrev > 0.0) {
				cfl = fmin(serMax, cfl0 * serFirst / serPrev);
				dfl = dfl0 * cfl / cfl0;
			}
			calcTimeStep(printTime, &dt, &visc);
			memset(resIter, 0, sizeof(resIter));
			if (!isImplicit) {
				if ((timeOrder == 1) && (nRKstages == 1))
					explicitTimeStepEuler(t, dt, resIter);
				else
					explicitTimeStepRK(t, dt, resIter);
			} else {
				implicitTimeStep(t, dt, resIter);
			}
			t += dt;
			if (write_out) {
				/* the reference's own analyze: record points,
				 * calcCoef, residual file */
				analyze(t, iter, resIter);
			} else if (doCoef && doCalcWing) {
				/* analyze() (src/analyze.c:411-433) without the
				 * residual-file write */
				resIter[4] = wing.cl;
				resIter[5] = wing.cd;
				calcCoef();
				resIter[4] = fabs(resIter[4] - wing.cl) / firstElem->dt;
				resIter[5] = fabs(resIter[5] - wing.cd) / firstElem->dt;
			}
			if (iter == 1)
				serFirst = resIter[abortVariable];
			serPrev = resIter[abortVariable];
			wall[nhist] = omp_get_wtime() - tStart;
			double *h = &hist[8 * nhist++];
			h[0] = t; h[1] = dt;
			for (int v = 0; v < 6; ++v)
				h[2 + v] = resIter[v];
			if (stopTime - t <= 1e-15)
				break;
			if (isStationary && fabs(resIter[abortVariable]) <= abortResidual) {
				if (doAbortOnClResidual) {
					if (fabs(resIter[4]) <= clAbortResidual)
						converged = true;
				} else if (doAbortOnCdResidual) {
					if (fabs(resIter[5]) <= cdAbortResidual)
						converged = true;
				} else {
					converged = true;
				}
				if (converged)
					break;
			}
			/* relative stop around the reference's loop (the residual
			 * of the abort variable relative to the first step's) */
			if (isStationary && relAbort > 0.0) {
				if (nhist == 1)
					relFirst = resIter[abortVariable];
				if (resIter[abortVariable] <= relAbort * relFirst) {
					converged = true;
					break;
				}
			}
			if ((printTime - t <= 1e-15) || (iter == printIter)) {
				if (printTime - t <= 1e-15)
					printTime += IOtimeInterval;
				if (iter == printIter)
					printIter += IOiterInterval;
			}
		}
		double tEnd = omp_get_wtime();
		if (write_out) {
			/* the final solution file (and the exact-solution file)
			 * of dataOutput (src/output.c:334-398) */
			dataOutput(t, nhist);
			finalizeDataOutput();
		}
		dump_state();
		if (hasExactSolution) {
			/* the error analysis that ends timeDisc (src/analyze.c:
			 * 445-514) prints the norms; the gradients it reconstructs
			 * are dumped for a full-precision check */
			calcErrors(t);
			double *ux = malloc(sizeof(double) * 4 * nElems);
			double *uy = malloc(sizeof(double) * 4 * nElems);
			for (long i = 0; i < nElems; ++i)
				for (int v = 0; v < 4; ++v) {
					ux[4 * i + v] = elem[i]->u_x[v];
					uy[4 * i + v] = elem[i]->u_y[v];
				}
			dump_f64("err_u_x", ux, 4 * nElems);
			dump_f64("err_u_y", uy, 4 * nElems);
			free(ux);
			free(uy);
		}
		dump_f64("history", hist, 8 * nhist);
		dump_f64("step_wall", wall, nhist);
		double info[8] = {t, (double)nhist, tEnd - tStart,
				  (double)omp_get_max_threads(), converged ? 1.0 : 0.0,
				  isImplicit ? (double)nNewtonIterGlobal : 0.0,
				  isImplicit ? (double)nGMRESiterGlobal : 0.0,
				  doCalcWing ? wing.cl : 0.0};
		dump_f64("run_info", info, 8);
		if (doCalcWing) {
			double clcd[2] = {wing.cl, wing.cd};
			dump_f64("clcd", clcd, 2);
		}
		free(hist);
		free(wall);
	} else if (!strcmp(mode, "jacobian")) {
		double tb = argc > 4 ? strtod(argv[4], NULL) : 0.0;
		double dtb = argc > 5 ? strtod(argv[5], NULL) : 1e-3;
		if (argc > 6 && strcmp(argv[6], "-"))
			load_state(argv[6]);
		if (!usePrecond) {
			fprintf(stderr, "ccfd_ref: jacobian needs precond = T\n");
			return 2;
		}
		double dt;
		bool visc;
		calcTimeStep(printTime, &dt, &visc);
		t = tb;
		fvTimeDerivative(tb + dtb);
		for (long i = 0; i < nElems; ++i)
			for (int v = 0; v < NVAR; ++v)
				R_XK[v][i] = elem[i]->u_t[v];
		buildMatrix(tb, dtb);
		double *dd = malloc(sizeof(double) * 16 * nElems);
		double *di = malloc(sizeof(double) * 16 * nElems);
		long nhs = 0;
		for (long i = 0; i < nElems; ++i)
			nhs += elem[i]->elemType;
		double *off = calloc(16 * (nhs + 1), sizeof(double));
		double *pv = malloc(sizeof(double) * 4 * nElems);
		long k = 0;
		for (long i = 0; i < nElems; ++i) {
			for (int a = 0; a < 4; ++a) {
				pv[4 * i + a] = elem[i]->pVar[a];
				for (int b = 0; b < 4; ++b) {
					dd[16 * i + 4 * a + b] = D[i][a][b];
					di[16 * i + 4 * a + b] = Dinv[i][a][b];
				}
			}
			for (side_t *sd = elem[i]->firstSide; sd; sd = sd->nextElemSide, ++k) {
				long j = sd->connection->elem->id;
				if (j < 0 || j >= nElems)
					continue;
				for (int a = 0; a < 4; ++a)
					for (int b = 0; b < 4; ++b)
						off[16 * k + 4 * a + b] = dRdU[4 * i + a][4 * j + b];
			}
		}
		dump_f64("jac_d", dd, 16 * nElems);
		dump_f64("jac_dinv", di, 16 * nElems);
		dump_f64("jac_off", off, 16 * nhs);
		dump_f64("pvar_after", pv, 4 * nElems);
		if (argc > 7) {
			FILE *f = fopen(argv[7], "rb");
			if (!f) {
				fprintf(stderr, "ccfd_ref: cannot open vector file %s\n", argv[7]);
				return 2;
			}
			double **bv = malloc(sizeof(double *) * NVAR), **xv = malloc(sizeof(double *) * NVAR);
			for (int v = 0; v < NVAR; ++v) {
				bv[v] = malloc(sizeof(double) * nElems);
				xv[v] = malloc(sizeof(double) * nElems);
			}
			double *raw = malloc(sizeof(double) * 4 * nElems);
			if (fread(raw, sizeof(double), 4 * nElems, f) != (size_t)(4 * nElems)) {
				fprintf(stderr, "ccfd_ref: short vector file\n");
				return 2;
			}
			fclose(f);
			for (long i = 0; i < nElems; ++i)
				for (int v = 0; v < NVAR; ++v)
					bv[v][i] = raw[4 * i + v];
			LUSGS(bv, xv);
			for (long i = 0; i < nElems; ++i)
				for (int v = 0; v < NVAR; ++v)
					raw[4 * i + v] = xv[v][i];
			dump_f64("lusgs", raw, 4 * nElems);
		}
		double *rx = malloc(sizeof(double) * 4 * nElems);
		for (long i = 0; i < nElems; ++i)
			for (int v = 0; v < NVAR; ++v)
				rx[4 * i + v] = R_XK[v][i];
		dump_f64("r_xk_used", rx, 4 * nElems);
	} else {
		fprintf(stderr, "ccfd_ref: unknown mode %s\n", mode);
		return 2;
	}
	fclose(dumpFile);
	return 0;
}
