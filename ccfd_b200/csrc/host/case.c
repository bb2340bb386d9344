/*
 * Case set-up on the host: the parameter reads and one-time constructions of
 * the reference's initialisation sequence (src/main.c:53-118), in the same
 * order, because repeated keys (BCtype, rho, mach, ...) are consumed in read
 * order:
 *   initOutput          src/output.c:36-47
 *   initEquation        src/equation.c:40-124
 *   initBoundary        src/boundary.c:29-137
 *   initMesh/readMesh   src/mesh.c:1849-1924
 *   initInitialCondition src/initialCondition.c:37-89
 *   initFV              src/finiteVolume.c:30-65
 *   initTimeDisc        src/timeDiscretization.c:69-240
 *   initLinearSolver    src/linearSolver.c:68-107
 *   setInitialCondition src/initialCondition.c:163-223
 *   initAnalyze         src/analyze.c:199-280
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "ccfd_host.h"

const char *ccfd_strerror(int s)
{
	switch (s) {
	case CCFD_OK: return "ok";
	case CCFD_ERR_ARG: return "invalid argument";
	case CCFD_ERR_CUDA: return "CUDA runtime error";
	case CCFD_ERR_NOMEM: return "out of memory";
	case CCFD_ERR_DT: return "Convective Time Step NaN";
	case CCFD_ERR_NEWTON: return "Newton NOT converged";
	case CCFD_ERR_SINGULAR: return "LUSGS D-Matrix is singular";
	case CCFD_ERR_VACUUM: return "Vacuum is generated by given data";
	case CCFD_ERR_TIMEOUT: return "device wait timed out";
	case CCFD_ERR_INI: return "Inifile missing necessary keyword or invalid value";
	case CCFD_ERR_MESH: return "mesh error (Problem in Connect / undefined BC)";
	case CCFD_ERR_STATE: return "non-finite state or residual";
	case CCFD_ERR_BUDGET: return "request exceeds the device-memory budget";
	case CCFD_ERR_UNSUPPORTED: return "option not supported";
	case CCFD_ERR_NOT_CONVERGED: return "Maximum Iteration Number Reached";
	case CCFD_ERR_GMRES: return "GMRES breakdown";
	case CCFD_ERR_BUSY: return "context is being stepped by a batch";
	default: return "unknown status";
	}
}

void ccfd_host_prim_cons(double gam1q, const double p[4], double c[4])
{
	/* primCons, src/equationOfState.c:19-26 */
	c[0] = p[0];
	c[1] = p[1] * p[0];
	c[2] = p[2] * p[0];
	c[3] = gam1q * p[3] + 0.5 * (c[1] * p[1] + c[2] * p[2]);
}

void ccfd_host_cons_prim(double gam1, const double c[4], double p[4])
{
	/* consPrim, src/equationOfState.c:37-52 */
	p[0] = c[0];
	p[1] = c[1] / c[0];
	p[2] = c[2] / c[0];
	p[3] = gam1 * (c[3] - 0.5 * (c[1] * p[1] + c[2] * p[2]));
	if (p[0] < 1e-19)
		p[0] = 1e-10;
	if (p[3] < 1e-19)
		p[3] = 1e-10;
}

/* exactFunc for initial conditions, src/exactFunction.c:35-183 (case 5 is
 * only evaluated at time 0 on the host) */
int ccfd_host_exact_func(int which, const double x[2], double time,
			 double gam, const ccfd_exact *ex, double pv[4])
{
	double pi = acos(-1.0), gam1 = gam - 1.0;
	switch (which) {
	case 1: {
		pv[0] = 1.0; pv[1] = 0.0; pv[2] = 0.0; pv[3] = 1.0;
		double xLen = ex->x_max - ex->x_min, yLen = ex->y_max - ex->y_min;
		if (x[0] >= 0.3 * xLen + 1.0 / 30.0 * xLen * cos(2.0 * pi * 3.0 / yLen * x[1]))
			pv[0] = 0.25;
		if ((x[0] <= 0.1 * xLen) && (x[0] >= 1.0 / 30.0 * xLen)) {
			pv[0] = 4.22;
			pv[3] = 4.9;
		}
		return CCFD_OK;
	}
	case 2: {
		pv[0] = 1.0; pv[1] = 0.0; pv[2] = 0.0;
		double hWidth = fmin((ex->x_max - ex->x_min), (ex->y_max - ex->y_min)) / 100.0 * 6.0;
		double amplitude = 1.0;
		double xPeak = ex->x_min + 0.5 * (ex->x_max - ex->x_min);
		double yPeak = ex->y_min + 0.5 * (ex->y_max - ex->y_min);
		double expLog = exp(-log(2.0));
		double hWidth2 = hWidth * hWidth;
		double dr2 = (x[0] - xPeak) * (x[0] - xPeak) + (x[1] - yPeak) * (x[1] - yPeak);
		pv[3] = 1.0 + amplitude * pow(expLog, dr2 / hWidth2);
		return CCFD_OK;
	}
	case 3: {
		double omega = pi * 1.0, a = 2.0 * pi, resu[4];
		resu[0] = resu[1] = resu[2] = 2.0 + 0.1 * sin(omega * (x[0] + x[1]) - a * time);
		resu[3] = resu[0] * resu[0];
		ccfd_host_cons_prim(gam1, resu, pv);
		return CCFD_OK;
	}
	case 4: {
		double sqrt3q = 1 / sqrt(3.0);
		double factor = pi / (0.2 * ex->dx_ref);
		double cSum[4] = {9.4, 57.157676649772950686, -33.0, 566.0};
		double cDiff[4] = {6.6, 57.157676649772950686, -33.0, 561.0};
		double cv[4];
		for (int i = 0; i < 4; ++i)
			cv[i] = 0.5 * (cSum[i] - cDiff[i] * tanh((x[0] - (1.0 / 6.0 + (20.0 * time + x[1]) * sqrt3q)) * factor));
		pv[0] = cv[0];
		pv[1] = cv[1] / cv[0];
		pv[2] = cv[2] / cv[0];
		pv[3] = gam1 * (cv[3] - 0.5 * (cv[1] * cv[1] + cv[2] * cv[2]) / cv[0]);
		return CCFD_OK;
	}
	case 5:
		if (time != 0.0)
			return CCFD_ERR_UNSUPPORTED;
		if (x[0] <= ex->rp1d_interface) {
			pv[0] = ex->ref_state[0][0];
			pv[1] = ex->ref_state[0][1];
			pv[3] = ex->ref_state[0][3];
		} else {
			pv[0] = ex->ref_state[1][0];
			pv[1] = ex->ref_state[1][1];
			pv[3] = ex->ref_state[1][3];
		}
		pv[2] = 0.0;
		return CCFD_OK;
	case 6: {
		double omega = pi * 1.0, amplitude = 0.00001;
		double cons0[4] = {1.0, 0.1, 0.0, 1.0}, p0[4];
		ccfd_host_cons_prim(gam1, cons0, p0);
		double c0 = sqrt(gam * p0[3] / p0[0]);
		double H0 = (cons0[3] + p0[3]) / p0[0];
		double R[4][4] = {
			{1.0, 1.0, 0.0, 1.0},
			{p0[1] - c0, p0[1], 0.0, p0[1] + c0},
			{p0[2], p0[2], 1.0, p0[2]},
			{H0 - p0[1] * c0, (p0[1] * p0[1] + p0[2] * p0[2]) / 2.0, p0[2], H0 + p0[1] * c0}};
		double resu[4], vec[4] = {0.0, 0.0, 0.0, amplitude * sin(omega * (x[0] - (c0 + p0[1]) * time))};
		for (int i = 0; i < 4; ++i) {
			resu[i] = cons0[i];
			for (int j = 0; j < 4; ++j)
				resu[i] += R[i][j] * vec[j];
		}
		ccfd_host_cons_prim(gam1, resu, pv);
		return CCFD_OK;
	}
	default:
		return CCFD_ERR_INI;
	}
}

void ccfd_case_free(ccfd_case *c)
{
	if (!c)
		return;
	ccfd_mesh_free(&c->mesh);
	free(c->prim0);
	free(c);
}

#define TRY(x) do { if ((st = (x)) != CCFD_OK) goto fail; } while (0)

static int dir_join(const char *base, const char *name, char *out, size_t n)
{
	if (name[0] == '/' || !base || !base[0])
		snprintf(out, n, "%s", name);
	else
		snprintf(out, n, "%s/%s", base, name);
	return CCFD_OK;
}

int ccfd_case_load_text(const char *text, const char *base_dir, ccfd_case **out)
{
	*out = NULL;
	ccfd_ini *ini = ccfd_ini_parse(text);
	if (!ini)
		return CCFD_ERR_NOMEM;
	ccfd_case *c = calloc(1, sizeof(ccfd_case));
	double *nodes = NULL;
	long *tria = NULL, *quad = NULL, *bcedge = NULL;
	long nn = 0, nt = 0, nq = 0, nb = 0;
	int st = CCFD_OK;
	if (!c) {
		ccfd_ini_free(ini);
		return CCFD_ERR_NOMEM;
	}
	ccfd_params *P = &c->params;
	long lv;
	int bv;
	int n_domains = 1;
	double (*dom_state)[4] = NULL;
	double pi = acos(-1.0);

	TRY(ccfd_ini_bool(ini, "stationary", "T", &P->stationary));

	/* initOutput */
	TRY(ccfd_ini_str(ini, "fileName", NULL, c->file_name, sizeof(c->file_name)));
	TRY(ccfd_ini_dbl(ini, "IOtimeInterval", NULL, &P->io_time_interval));
	double io_iter;
	TRY(ccfd_ini_dbl(ini, "IOiterInterval", NULL, &io_iter));
	P->io_iter_interval = (int)io_iter;
	TRY(ccfd_ini_int(ini, "outputFormat", "1", &lv));
	c->output_format = (int)lv;

	/* initEquation */
	P->eqn = CCFD_EULER;
	TRY(ccfd_ini_dbl(ini, "gamma", "1.4", &P->gamma));
	TRY(ccfd_ini_dbl(ini, "R", "287", &P->R));
	P->mu = 0.0;
	P->Pr = 0.72;
	/* the equation system is a compile-time choice in the reference; here a
	 * key (default Euler) selects it */
	TRY(ccfd_ini_bool(ini, "navierStokes", "F", &bv));
	if (bv) {
		P->eqn = CCFD_NAVIER_STOKES;
		TRY(ccfd_ini_dbl(ini, "mu", "0.0", &P->mu));
		TRY(ccfd_ini_dbl(ini, "Pr", "0.72", &P->Pr));
	}
	TRY(ccfd_ini_int(ini, "fluxFunction", NULL, &lv));
	if (lv < 1 || lv > 11) {
		st = CCFD_ERR_INI;
		goto fail;
	}
	P->flux = (int)lv;
	TRY(ccfd_ini_bool(ini, "calcSource", "F", &bv));
	P->source_func = 0;
	if (bv) {
		TRY(ccfd_ini_int(ini, "sourceFunction", NULL, &lv));
		if (lv != 1) {
			st = CCFD_ERR_INI; /* src/source.c knows source 1 only */
			goto fail;
		}
		P->source_func = (int)lv;
	}

	/* initBoundary */
	TRY(ccfd_ini_int(ini, "nBC", NULL, &lv));
	if (lv < 0 || lv > 20) {
		st = CCFD_ERR_INI;
		goto fail;
	}
	c->n_bc_table = (int)lv;
	for (int i = 0; i < c->n_bc_table; ++i) {
		ccfd_bc *b = &c->bc_table[i];
		TRY(ccfd_ini_int(ini, "BCtype", NULL, &lv));
		b->type = (int)(lv / 100);
		b->id = (int)(lv % 100);
		double Ma, alpha, cs, v;
		switch (b->type) {
		case CCFD_BC_SLIPWALL:
		case CCFD_BC_OUTFLOW:
			break;
		case CCFD_BC_WALL:
			if (P->eqn != CCFD_NAVIER_STOKES) {
				st = CCFD_ERR_INI; /* "Illegal boundary condition" */
				goto fail;
			}
			TRY(ccfd_ini_bool(ini, "adiabaticWall", NULL, &b->is_adiabatic));
			if (!b->is_adiabatic) {
				/* countKeys(.., -1) > 1 (src/boundary.c:68-77): a
				 * missing key is fatal; the value is never used */
				int n1, n2;
				TRY(ccfd_ini_count(ini, "wallTemperature", -1, &n1));
				if (n1 > 1) {
					TRY(ccfd_ini_dbl(ini, "wallTemperature", NULL, &b->pvar[0]));
				} else {
					TRY(ccfd_ini_count(ini, "wallHeatFlux", -1, &n2));
					if (n2 > 1) {
						TRY(ccfd_ini_dbl(ini, "wallHeatFlux", NULL, &b->pvar[0]));
					} else {
						st = CCFD_ERR_INI;
						goto fail;
					}
				}
			}
			break;
		case CCFD_BC_INFLOW:
		case CCFD_BC_CHARACTERISTIC:
			TRY(ccfd_ini_dbl(ini, "rho", NULL, &b->pvar[0]));
			TRY(ccfd_ini_dbl(ini, "mach", NULL, &Ma));
			TRY(ccfd_ini_dbl(ini, "alpha", NULL, &alpha));
			TRY(ccfd_ini_dbl(ini, "pressure", NULL, &b->pvar[3]));
			cs = sqrt(P->gamma * b->pvar[3] / b->pvar[0]);
			v = Ma * cs;
			b->pvar[1] = v * cos(alpha * pi / 180.0);
			b->pvar[2] = v * sin(alpha * pi / 180.0);
			break;
		case CCFD_BC_EXACTSOL:
			TRY(ccfd_ini_int(ini, "BCexactFunc", NULL, &lv));
			b->exact_func = (int)lv;
			break;
		case CCFD_BC_PERIODIC:
			TRY(ccfd_ini_dbl_array(ini, "connection", 2, NULL, b->connection));
			break;
		case CCFD_BC_PRESSURE_OUT:
			TRY(ccfd_ini_dbl(ini, "pressure", NULL, &b->pvar[3]));
			break;
		default:
			st = CCFD_ERR_INI;
			goto fail;
		}
	}

	/* initMesh / readMesh */
	TRY(ccfd_ini_int(ini, "meshType", "1", &lv));
	if (lv == 0) {
		char fmt[256], file[256], path[600];
		TRY(ccfd_ini_str(ini, "meshFormat", NULL, fmt, sizeof(fmt)));
		TRY(ccfd_ini_str(ini, "meshFile", NULL, file, sizeof(file)));
		char full[520];
		snprintf(full, sizeof(full), "%s%s", file, fmt);
		dir_join(base_dir, full, path, sizeof(path));
		if (!strcmp(fmt, ".mesh")) {
			TRY(ccfd_read_emc2(path, &nodes, &nn, &tria, &nt, &quad, &nq, &bcedge, &nb));
		} else if (strcmp(fmt, ".msh") && strcmp(fmt, ".msh2") && strcmp(fmt, ".msh4")) {
			st = CCFD_ERR_UNSUPPORTED; /* the CGNS reader needs the CGNS library */
			goto fail;
		} else {
			TRY(ccfd_read_gmsh(path, &nodes, &nn, &tria, &nt, &quad, &nq, &bcedge, &nb));
		}
	} else if (lv == 1) {
		ccfd_cart cart;
		memset(&cart, 0, sizeof(cart));
		TRY(ccfd_ini_int(ini, "nElemsX", NULL, &cart.i_max));
		TRY(ccfd_ini_int(ini, "nElemsY", NULL, &cart.j_max));
		double x0[2], x1[2];
		TRY(ccfd_ini_dbl_array(ini, "X0", 2, NULL, x0));
		TRY(ccfd_ini_dbl_array(ini, "Xmax", 2, NULL, x1));
		cart.x_min = x0[0]; cart.y_min = x0[1];
		cart.x_max = x1[0]; cart.y_max = x1[1];
		TRY(ccfd_ini_int_array(ini, "nBCsegments", 4, NULL, cart.n_bc));
		for (int s = 0; s < 4; ++s) {
			if (cart.n_bc[s] < 0 || cart.n_bc[s] > 20) {
				st = CCFD_ERR_INI;
				goto fail;
			}
			if (cart.n_bc[s] == 1) {
				TRY(ccfd_ini_int(ini, "meshBCtype", NULL, &lv));
				cart.bc_type[s][0] = (int)lv;
				cart.bc_range[s][0][0] = 1;
				cart.bc_range[s][0][1] = (int)((s % 2) == 0 ? cart.i_max : cart.j_max);
			} else {
				for (int i = 0; i < cart.n_bc[s]; ++i) {
					TRY(ccfd_ini_int(ini, "meshBCtype", NULL, &lv));
					cart.bc_type[s][i] = (int)lv;
					TRY(ccfd_ini_int(ini, "BCstart", NULL, &lv));
					cart.bc_range[s][i][0] = (int)lv;
					TRY(ccfd_ini_int(ini, "BCend", NULL, &lv));
					cart.bc_range[s][i][1] = (int)lv;
				}
			}
		}
		TRY(ccfd_cart_generate(&cart, &nodes, &nn, &quad, &nq, &bcedge, &nb));
	} else {
		st = CCFD_ERR_INI;
		goto fail;
	}
	TRY(ccfd_mesh_build(nodes, nn, tria, nt, quad, nq, bcedge, nb,
			    c->bc_table, c->n_bc_table, &c->mesh));
	ccfd_exact *ex = &c->exact;
	ex->x_min = c->mesh.x_min; ex->x_max = c->mesh.x_max;
	ex->y_min = c->mesh.y_min; ex->y_max = c->mesh.y_max;
	ex->dx_ref = c->mesh.dx_ref;

	/* initInitialCondition */
	TRY(ccfd_ini_int(ini, "icType", NULL, &lv));
	c->ic_type = (int)lv;
	if (c->ic_type == 1) {
		TRY(ccfd_ini_int(ini, "nDomains", "1", &lv));
		n_domains = (int)lv;
		if (n_domains < 1) {
			st = CCFD_ERR_INI;
			goto fail;
		}
		dom_state = calloc(n_domains, sizeof(*dom_state));
		if (!dom_state) {
			st = CCFD_ERR_NOMEM;
			goto fail;
		}
		for (int i = 0; i < n_domains; ++i) {
			double Ma, cs, v;
			TRY(ccfd_ini_int(ini, "domainID", NULL, &lv));
			TRY(ccfd_ini_dbl(ini, "rho", NULL, &dom_state[i][0]));
			TRY(ccfd_ini_dbl(ini, "mach", NULL, &Ma));
			TRY(ccfd_ini_dbl(ini, "alpha", NULL, &ex->alpha));
			TRY(ccfd_ini_dbl(ini, "pressure", NULL, &dom_state[i][3]));
			cs = sqrt(P->gamma * dom_state[i][3] / dom_state[i][0]);
			v = Ma * cs;
			dom_state[i][1] = v * cos(ex->alpha * pi / 180.0);
			dom_state[i][2] = v * sin(ex->alpha * pi / 180.0);
		}
		memcpy(ex->ref_state[0], dom_state[0], sizeof(double) * 4);
		if (n_domains > 1)
			memcpy(ex->ref_state[1], dom_state[1], sizeof(double) * 4);
	} else if (c->ic_type == 2) {
		TRY(ccfd_ini_int(ini, "exactFunc", NULL, &lv));
		c->exact_func = (int)lv;
		if (c->exact_func == 5) {
			TRY(ccfd_ini_dbl(ini, "RP_1D_interface", "0.5", &ex->rp1d_interface));
			TRY(ccfd_ini_dbl_array(ini, "StateLeft", 4, NULL, ex->ref_state[0]));
			TRY(ccfd_ini_dbl_array(ini, "StateRight", 4, NULL, ex->ref_state[1]));
		}
	} else {
		st = CCFD_ERR_INI; /* "Initial Condition not known" */
		goto fail;
	}

	/* initFV */
	TRY(ccfd_ini_int(ini, "spatialOrder", "1", &lv));
	if (lv < 1 || lv > 2) {
		st = CCFD_ERR_INI;
		goto fail;
	}
	P->spatial_order = (int)lv;
	P->limiter = CCFD_LIM_BARTH_JESPERSEN;
	P->venk_k = 0.0;
	if (P->spatial_order == 2) {
		TRY(ccfd_ini_int(ini, "limiter", "1", &lv));
		if (lv != 1 && lv != 2) {
			st = CCFD_ERR_INI;
			goto fail;
		}
		P->limiter = (int)lv;
		if (P->limiter == CCFD_LIM_VENKATAKRISHNAN)
			TRY(ccfd_ini_dbl(ini, "venk_k", "1", &P->venk_k));
	}

	/* initTimeDisc */
	TRY(ccfd_ini_dbl(ini, "CFL", "0.9", &P->cfl));
	TRY(ccfd_ini_dbl(ini, "DFL", "0.9", &P->dfl));
	TRY(ccfd_ini_bool(ini, "timeStep1D", "F", &P->time_step_1d));
	TRY(ccfd_ini_int(ini, "timeOrder", "1", &lv));
	if (lv > 3 || lv < 1) {
		st = CCFD_ERR_INI;
		goto fail;
	}
	P->time_order = (int)lv;
	TRY(ccfd_ini_bool(ini, "implicit", "F", &P->implicit));
	TRY(ccfd_ini_int(ini, "nRKstages", "1", &lv));
	P->n_rk_stages = (int)lv;
	if (!(P->n_rk_stages == 1 && P->time_order == 1) &&
	    (P->n_rk_stages < 3 || P->n_rk_stages > 5)) {
		st = CCFD_ERR_INI; /* "Wrong Number of RK Coefficients" */
		goto fail;
	}
	if (P->stationary) {
		TRY(ccfd_ini_dbl(ini, "abortResidual", "1e-6", &P->abort_residual));
		TRY(ccfd_ini_int(ini, "abortVariable", "1", &lv));
		P->abort_variable = (int)lv - 1;
		if (P->abort_variable < 0 || P->abort_variable > 3) {
			st = CCFD_ERR_INI;
			goto fail;
		}
		TRY(ccfd_ini_dbl(ini, "cl_abortResidual", "0.0", &P->cl_abort_residual));
		TRY(ccfd_ini_dbl(ini, "cd_abortResidual", "0.0", &P->cd_abort_residual));
		if (!((P->cl_abort_residual == 0.0) && (P->cd_abort_residual == 0)) &&
		    !(P->cl_abort_residual > 0.0) && !(P->cd_abort_residual > 0.0)) {
			st = CCFD_ERR_INI; /* "Wrong Definition of Abort Residual" */
			goto fail;
		}
	}
	TRY(ccfd_ini_int(ini, "maxIter", "100000", &P->max_iter));
	TRY(ccfd_ini_dbl(ini, "tEnd", NULL, &P->t_end));

	/* initLinearSolver */
	P->n_kdim = 5;
	P->n_newton_iter = 20;
	P->eps_newton = 0.001;
	P->eps_gmres = 0.001;
	P->gamma_ew = 0.9;
	if (P->implicit) {
		TRY(ccfd_ini_int(ini, "nKdim", "5", &lv));
		P->n_kdim = (int)lv;
		TRY(ccfd_ini_dbl(ini, "epsNewton", "0.001", &P->eps_newton));
		TRY(ccfd_ini_dbl(ini, "epsGMRES", "0.001", &P->eps_gmres));
		TRY(ccfd_ini_int(ini, "nNewtonIter", "20", &lv));
		P->n_newton_iter = (int)lv;
		TRY(ccfd_ini_dbl(ini, "gammaEW", "0.9", &P->gamma_ew));
		TRY(ccfd_ini_bool(ini, "precond", "F", &P->precond));
		if (P->n_kdim < 1) {
			st = CCFD_ERR_INI;
			goto fail;
		}
	}

	/* setInitialCondition */
	long N = c->mesh.n_cells;
	c->prim0 = malloc(sizeof(double) * 4 * N);
	if (!c->prim0) {
		st = CCFD_ERR_NOMEM;
		goto fail;
	}
	for (long e = 0; e < N; ++e) {
		double *pv = &c->prim0[4 * e];
		if (c->ic_type == 1) {
			int d = n_domains == 1 ? 0 : c->mesh.cell_domain[e] - 1;
			if (d < 0 || d >= n_domains) {
				st = CCFD_ERR_INI;
				goto fail;
			}
			memcpy(pv, dom_state[d], sizeof(double) * 4);
		} else {
			TRY(ccfd_host_exact_func(c->exact_func, &c->mesh.cell_bary[2 * e],
						 0.0, P->gamma, ex, pv));
		}
	}
	free(dom_state);
	dom_state = NULL;

	/* initAnalyze */
	int has_exact;
	TRY(ccfd_ini_bool(ini, "exactSolution", "F", &has_exact));
	P->exact_solution = has_exact;
	TRY(ccfd_ini_bool(ini, "calcWing", "F", &P->calc_wing));
	P->ref_length = 1.0;
	if (P->calc_wing) {
		TRY(ccfd_ini_dbl(ini, "referenceLength", "1.0", &P->ref_length));
		TRY(ccfd_ini_int(ini, "wall_id", NULL, &lv));
		P->wall_id = (int)lv;
	}
	/* record points (initRecordPoints, src/analyze.c:34-90) */
	TRY(ccfd_ini_int(ini, "nRecordPoints", "0", &lv));
	if (lv < 0 || lv > CCFD_MAX_RECORD) {
		st = CCFD_ERR_INI;
		goto fail;
	}
	c->n_record = (int)lv;
	for (int k = 0; k < c->n_record; ++k)
		TRY(ccfd_ini_dbl_array(ini, "pointCoords", 2, NULL, c->record_xy[k]));
	TRY(ccfd_locate_points(&c->mesh, &c->record_xy[0][0], c->n_record, c->record_cell));
	/* extensions of this implementation (defaults keep the reference's
	 * behaviour): precision mode and a relative steady stop criterion */
	TRY(ccfd_ini_int(ini, "precision", "0", &lv));
	P->precision = (int)lv;
	TRY(ccfd_ini_dbl(ini, "relAbortResidual", "0", &P->rel_abort_residual));
	TRY(ccfd_ini_dbl(ini, "serCFLmax", "0", &P->ser_cfl_max));

	free(nodes); free(tria); free(quad); free(bcedge);
	ccfd_ini_free(ini);
	*out = c;
	return CCFD_OK;
fail:
	free(dom_state);
	free(nodes); free(tria); free(quad); free(bcedge);
	ccfd_ini_free(ini);
	ccfd_case_free(c);
	return st;
}

int ccfd_case_load(const char *path, ccfd_case **out)
{
	FILE *f = fopen(path, "rb");
	if (!f)
		return CCFD_ERR_INI;
	fseek(f, 0, SEEK_END);
	long n = ftell(f);
	fseek(f, 0, SEEK_SET);
	char *buf = malloc(n + 1);
	if (!buf) {
		fclose(f);
		return CCFD_ERR_NOMEM;
	}
	size_t got = fread(buf, 1, n, f);
	fclose(f);
	buf[got] = '\0';
	char dir[512];
	snprintf(dir, sizeof(dir), "%s", path);
	char *slash = strrchr(dir, '/');
	if (slash)
		*slash = '\0';
	else
		strcpy(dir, ".");
	int st = ccfd_case_load_text(buf, dir, out);
	free(buf);
	return st;
}
