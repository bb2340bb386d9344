/*
 * Internal declarations of the C host layer (parameter parsing, mesh
 * construction, case set-up).  Public entry points live in
 * include/ccfd_b200.h.
 */
#ifndef CCFD_HOST_H
#define CCFD_HOST_H

#include <stddef.h>
#include "ccfd_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---- .ini parameter list (semantics of src/readInTools.c) ---- */
typedef struct ccfd_ini ccfd_ini;

ccfd_ini *ccfd_ini_parse(const char *text);
void ccfd_ini_free(ccfd_ini *ini);
/* Each getter consumes the first matching key, like findCmd
 * (src/readInTools.c:147-197).  def == NULL makes the key mandatory:
 * a missing key returns CCFD_ERR_INI. */
int ccfd_ini_str(ccfd_ini *ini, const char *key, const char *def, char *out, size_t n);
int ccfd_ini_int(ccfd_ini *ini, const char *key, const char *def, long *out);
int ccfd_ini_dbl(ccfd_ini *ini, const char *key, const char *def, double *out);
int ccfd_ini_bool(ccfd_ini *ini, const char *key, const char *def, int *out);
int ccfd_ini_dbl_array(ccfd_ini *ini, const char *key, int n, const char *def, double *out);
int ccfd_ini_int_array(ccfd_ini *ini, const char *key, int n, const char *def, int *out);
/* occurrences of key; proposal when absent (-1: mandatory), countKeys */
int ccfd_ini_count(ccfd_ini *ini, const char *key, int proposal, int *out);
/* keys never read (ignoredCmds, src/readInTools.c:427-436) */
int ccfd_ini_remaining(const ccfd_ini *ini);

/* ---- physics helpers shared by the host set-up ---- */
void ccfd_host_prim_cons(double gam1q, const double p[4], double c[4]);
void ccfd_host_cons_prim(double gam1, const double c[4], double p[4]);
int ccfd_host_exact_func(int which, const double x[2], double time,
			 double gam, const ccfd_exact *ex, double out[4]);

/* ---- Cartesian generator (src/mesh.c:385-486) ---- */
typedef struct ccfd_cart {
	long i_max, j_max;
	double x_min, y_min, x_max, y_max;
	int n_bc[4];              /* segments per side: bottom, right, top, left */
	int bc_type[4][20];
	int bc_range[4][20][2];
} ccfd_cart;

int ccfd_cart_generate(const ccfd_cart *cart, double **nodes, long *n_nodes,
		       long **quad, long *n_quad, long **bc_edge, long *n_bc_edge);

#ifdef __cplusplus
}
#endif
#endif
