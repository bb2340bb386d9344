/*
 * Solution output in the reference's formats (src/output.c).
 *
 * The tabular formats are written: CSV (outputFormat = 3, csvOutput,
 * src/output.c:53-112: cell barycentre x, density, x-velocity and pressure
 * per row) and curve (outputFormat = 2, curveOutput, src/output.c:253-327:
 * the x-density, x-velocity and x-pressure series one after another), rows
 * sorted by x with a stable sort (the reference's bubble sort is stable
 * too), "%15.9f" columns.  File names follow dataOutput (src/output.c:
 * 334-398): <fileName>_<iter %09ld> for stationary runs, <fileName>_<time
 * %015.7f> otherwise, and <fileName>_ex_... for the exact solution.  CGNS
 * (outputFormat = 1) needs the CGNS library and is not built
 * (CCFD_ERR_UNSUPPORTED).
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "ccfd_b200.h"

static void merge_sort_by_x(long *idx, long *tmp, const double *x, long n)
{
	/* bottom-up stable merge sort of indices by x */
	for (long w = 1; w < n; w *= 2) {
		for (long lo = 0; lo < n; lo += 2 * w) {
			long mid = lo + w < n ? lo + w : n;
			long hi = lo + 2 * w < n ? lo + 2 * w : n;
			long a = lo, b = mid, k = lo;
			while (a < mid && b < hi)
				tmp[k++] = (x[idx[b]] < x[idx[a]]) ? idx[b++] : idx[a++];
			while (a < mid)
				tmp[k++] = idx[a++];
			while (b < hi)
				tmp[k++] = idx[b++];
		}
		memcpy(idx, tmp, sizeof(long) * n);
	}
}

static int write_tabular(const ccfd_case *c, const double *prim, double time, long iter,
			 int exact, char *path, size_t path_len)
{
	if (!c || !prim)
		return CCFD_ERR_ARG;
	const int fmt = c->output_format;
	if (fmt != 2 && fmt != 3)
		return CCFD_ERR_UNSUPPORTED;
	const char *ext = fmt == 2 ? "curve" : "csv";
	const char *tag = exact ? "_ex" : "";
	char name[600];
	if (c->params.stationary)
		snprintf(name, sizeof(name), "%s%s_%09ld.%s", c->file_name, tag, iter, ext);
	else
		snprintf(name, sizeof(name), "%s%s_%015.7f.%s", c->file_name, tag, time, ext);
	if (path && path_len) {
		strncpy(path, name, path_len - 1);
		path[path_len - 1] = '\0';
	}
	const long n = c->mesh.n_cells;
	long *idx = malloc(sizeof(long) * (size_t)(n > 0 ? n : 1));
	long *tmp = malloc(sizeof(long) * (size_t)(n > 0 ? n : 1));
	double *x = malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
	if (!idx || !tmp || !x) {
		free(idx);
		free(tmp);
		free(x);
		return CCFD_ERR_NOMEM;
	}
	for (long i = 0; i < n; ++i) {
		idx[i] = i;
		x[i] = c->mesh.cell_bary[2 * i];
	}
	merge_sort_by_x(idx, tmp, x, n);
	FILE *f = fopen(name, "w");
	if (!f) {
		free(idx);
		free(tmp);
		free(x);
		return CCFD_ERR_ARG;
	}
	if (fmt == 3) {
		fprintf(f, "CoordinateX, Density, Velocity, Pressure\n");
		for (long k = 0; k < n; ++k) {
			long i = idx[k];
			fprintf(f, "%15.9f,%15.9f,%15.9f,%15.9f\n", x[i], prim[4 * i], prim[4 * i + 1],
				prim[4 * i + 3]);
		}
	} else {
		static const char *title[3] = {"#Density\n", "\n#Velocity\n", "\n#Pressure\n"};
		static const int var[3] = {0, 1, 3};
		for (int s = 0; s < 3; ++s) {
			fputs(title[s], f);
			for (long k = 0; k < n; ++k) {
				long i = idx[k];
				fprintf(f, "%15.9f,%15.9f\n", x[i], prim[4 * i + var[s]]);
			}
		}
	}
	fclose(f);
	free(idx);
	free(tmp);
	free(x);
	return CCFD_OK;
}

int ccfd_write_output(const ccfd_case *c, const double *prim, double time, long iter,
		      char *path, size_t path_len)
{
	return write_tabular(c, prim, time, iter, 0, path, path_len);
}

int ccfd_write_exact_output(const ccfd_case *c, const double *prim_exact, double time, long iter,
			    char *path, size_t path_len)
{
	return write_tabular(c, prim_exact, time, iter, 1, path, path_len);
}

/* analyze's files from history rows (ccfd_set_history): the residual file
 * <fileName>_analysis.csv with its gnuplot scripts for stationary runs or
 * calcWing (initAnalyze, src/analyze.c:205-281; analyze, :411-433) and one
 * file per record point (initRecordPoints / evalRecordPoints, :84-89,
 * 393-403).  The reference prints the time as t + dt of the step (its
 * elements' dt after the step). */
int ccfd_write_history(const ccfd_case *c, const double *rows, long n_rows, int width, int append)
{
	if (!c || (n_rows > 0 && !rows) || width < 11 + 4 * c->n_record)
		return CCFD_ERR_ARG;
	static const char *var_name[4] = {"RHO", "MX", "MY", "E"};
	const ccfd_params *p = &c->params;
	const int av = p->abort_variable >= 0 && p->abort_variable < 4 ? p->abort_variable : 0;
	char name[600];
	if (p->calc_wing || p->stationary) {
		snprintf(name, sizeof(name), "%s_analysis.csv", c->file_name);
		if (!append) {
			char res_name[600];
			snprintf(res_name, sizeof(res_name), "%s", name);
			FILE *d;
			snprintf(name, sizeof(name), "%s_residuals.dem", c->file_name);
			if (!(d = fopen(name, "w")))
				return CCFD_ERR_ARG;
			fprintf(d, "set title 'Residual Plot'\n");
			fprintf(d, "set logscale y\n");
			if (p->calc_wing) {
				fprintf(d, "plot '%s' using 1:3 title '%s' with lines\n", res_name, var_name[av]);
			} else {
				fprintf(d, "plot '%s' using 1:3 title 'RHO' with lines, \\\n", res_name);
				fprintf(d, "     '%s' using 1:4 title 'MX' with lines, \\\n", res_name);
				fprintf(d, "     '%s' using 1:5 title 'MY' with lines, \\\n", res_name);
				fprintf(d, "     '%s' using 1:6 title 'E' with lines\n", res_name);
			}
			fprintf(d, "pause -1");
			fclose(d);
			if (p->calc_wing) {
				snprintf(name, sizeof(name), "%s_CLCD.dem", c->file_name);
				if (!(d = fopen(name, "w")))
					return CCFD_ERR_ARG;
				fprintf(d, "set title 'CL/CD Plot'\n");
				fprintf(d, "plot '%s' using 1:4 title 'CL' with lines, \\\n", res_name);
				fprintf(d, "     '%s' using 1:5 title 'CD' with lines\n", res_name);
				fprintf(d, "pause -1");
				fclose(d);
			}
			snprintf(name, sizeof(name), "%s", res_name);
		}
		FILE *f = fopen(name, append ? "a" : "w");
		if (!f)
			return CCFD_ERR_ARG;
		if (!append) {
			if (p->calc_wing)
				fprintf(f, "Iter, Time, Residual(%s), CL, CD\n", var_name[av]);
			else
				fprintf(f, "Iter, Time, Residual(RHO), Residual(VX), Residual(VY), Residual(E)\n");
		}
		for (long r = 0; r < n_rows; ++r) {
			const double *w = &rows[(size_t)r * width];
			long iter = (long)w[0];
			double time = w[1] + w[2];
			if (p->calc_wing)
				fprintf(f, "%7ld, %13.8f, %15.8e, %15.10f, %15.10f\n", iter, time, w[3 + av], w[9],
					w[10]);
			else
				fprintf(f, "%7ld, %13.8f, %15.8e, %15.8e, %15.8e, %15.8e\n", iter, time, w[3], w[4],
					w[5], w[6]);
		}
		fclose(f);
	}
	for (int k = 0; k < c->n_record; ++k) {
		snprintf(name, sizeof(name), "%s_recordPoint_%d.csv", c->file_name, k);
		FILE *f = fopen(name, append ? "a" : "w");
		if (!f)
			return CCFD_ERR_ARG;
		if (!append)
			fprintf(f, "Time, Density, VelocityX, VelocityY, Pressure\n");
		for (long r = 0; r < n_rows; ++r) {
			const double *w = &rows[(size_t)r * width];
			const double *q = &w[11 + 4 * k];
			fprintf(f, "%20.12f,%20.12f,%20.12f,%20.12f,%20.12f\n", w[1] + w[2], q[0], q[1], q[2],
				q[3]);
		}
		fclose(f);
	}
	return CCFD_OK;
}
