/*
 * ccfd_run: command-line driver in the manner of the reference's main
 * (src/main.c:53-130): reads a case .ini, sets the case up, runs the time
 * loop on the GPU (explicit Runge-Kutta or implicit Newton / GMRES / LU-SGS
 * as the .ini selects) and writes the final solution in the reference's
 * output format.
 *
 *   ccfd_run case.ini [--steps N] [--device D] [--no-output]
 *
 * --steps N runs at most N time steps.  Exit status 0 on success, 1 on an
 * error (the message is printed, as the reference prints before exit(1)).
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "ccfd_b200.h"

static int fail(const char *what, int st)
{
	printf("| ERROR: %s: %s\n", what, ccfd_strerror(st));
	return 1;
}

int main(int argc, char **argv)
{
	const char *ini = NULL;
	long steps = 0;
	int device = 0, output = 1;
	for (int i = 1; i < argc; ++i) {
		if (!strcmp(argv[i], "--steps") && i + 1 < argc)
			steps = atol(argv[++i]);
		else if (!strcmp(argv[i], "--device") && i + 1 < argc)
			device = atoi(argv[++i]);
		else if (!strcmp(argv[i], "--no-output"))
			output = 0;
		else if (!ini)
			ini = argv[i];
		else {
			fprintf(stderr, "usage: %s case.ini [--steps N] [--device D] [--no-output]\n", argv[0]);
			return 2;
		}
	}
	if (!ini) {
		fprintf(stderr, "usage: %s case.ini [--steps N] [--device D] [--no-output]\n", argv[0]);
		return 2;
	}
	int st;
	ccfd_case *c = NULL;
	ccfd_ctx *ctx = NULL;
	if ((st = ccfd_set_device(device)))
		return fail("device", st);
	if ((st = ccfd_case_load(ini, &c)))
		return fail(ini, st);
	printf("case %s: %ld cells, %ld faces, %ld boundary faces\n", ini, c->mesh.n_cells,
	       c->mesh.n_faces, c->mesh.n_bc);
	if ((st = ccfd_create(&c->params, &ctx)))
		return fail("create", st);
	if ((st = ccfd_upload_case(ctx, &c->mesh, c->bc_table, c->n_bc_table, &c->exact, 1)))
		return fail("upload", st);
	if ((st = ccfd_set_state(ctx, c->prim0, CCFD_PRIMITIVE)))
		return fail("initial state", st);
	/* analyze's per-step files (residual file, record points) */
	const int history = output && (c->n_record > 0 || c->params.stationary || c->params.calc_wing);
	if (history && (st = ccfd_set_history(ctx, 4096, c->record_cell, c->n_record)))
		return fail("history", st);
	ccfd_report rep;
	st = c->params.implicit ? ccfd_run_implicit(ctx, steps, &rep) : ccfd_run_explicit(ctx, steps, &rep);
	if (history) {
		/* written also when the loop stopped on an error, as the
		 * reference's files hold every step it finished */
		long n = 0;
		int w = 0;
		int hs = ccfd_get_history(ctx, NULL, 0, &n, &w);
		double *rows = hs == CCFD_OK ? malloc(sizeof(double) * (size_t)(n > 0 ? n : 1) * w) : NULL;
		if (!rows)
			return fail("history", hs ? hs : CCFD_ERR_NOMEM);
		if ((hs = ccfd_get_history(ctx, rows, n, &n, &w)) ||
		    (hs = ccfd_write_history(c, rows, n, w, 0)))
			return fail("history", hs);
		free(rows);
	}
	if (st)
		return fail("time loop", st);
	printf("iterations %ld  t %.9g  dt %.6g  residual %.6e %.6e %.6e %.6e  device %.3f ms\n",
	       rep.iterations, rep.t, rep.dt, rep.residual[0], rep.residual[1], rep.residual[2],
	       rep.residual[3], rep.device_ms);
	if (c->params.calc_wing) {
		printf("cl %.12g  cd %.12g\n", rep.cl, rep.cd);
		/* the CP files calcCoef leaves after the last step */
		if (output && (st = ccfd_write_cp(ctx, c->file_name)))
			return fail("CP files", st);
	}
	if (c->params.implicit)
		printf("newton %ld  gmres %ld\n", rep.newton_iterations, rep.gmres_iterations);
	if (c->params.exact_solution && c->exact_func > 0) {
		/* the error analysis printed at the end of timeDisc
		 * (src/analyze.c:506-513) */
		double e[12];
		if ((st = ccfd_errors(ctx, c->exact_func, e)))
			return fail("errors", st);
		printf("\nError Analysis at t = %g\n", rep.t);
		printf("|                RHO           VX           VY            P\n");
		printf("| L1  :  %7.5e  %7.5e  %7.5e  %7.5e\n", e[0], e[1], e[2], e[3]);
		printf("| L2  :  %7.5e  %7.5e  %7.5e  %7.5e\n", e[4], e[5], e[6], e[7]);
		printf("| Linf:  %7.5e  %7.5e  %7.5e  %7.5e\n", e[8], e[9], e[10], e[11]);
	}
	if (output) {
		double *prim = malloc(sizeof(double) * 4 * (size_t)c->mesh.n_cells);
		if (!prim)
			return fail("output", CCFD_ERR_NOMEM);
		if ((st = ccfd_get_state(ctx, prim, CCFD_PRIMITIVE)))
			return fail("state", st);
		char path[600];
		st = ccfd_write_output(c, prim, rep.t, rep.iterations, path, sizeof(path));
		if (st == CCFD_OK)
			printf("wrote %s\n", path);
		else if (st != CCFD_ERR_UNSUPPORTED)
			return fail("output", st);
		if (st == CCFD_OK && c->params.exact_solution && c->exact_func > 0) {
			/* the exact-solution file of dataOutput (src/output.c:375-397) */
			if ((st = ccfd_exact_state(ctx, c->exact_func, rep.t, prim)))
				return fail("exact state", st);
			if ((st = ccfd_write_exact_output(c, prim, rep.t, rep.iterations, path, sizeof(path))))
				return fail("output", st);
			printf("wrote %s\n", path);
		}
		free(prim);
	}
	ccfd_destroy(ctx);
	ccfd_case_free(c);
	return 0;
}
