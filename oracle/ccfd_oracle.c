/*
 * CPU restatement of the reference ccfd residual-and-update path
 * (hheinzer/ccfd), plain C99, single-threaded.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA path.  Only tests/,
 * __graft_entry__.smoke() and the CPU-baseline leg of bench.py load it.  It
 * reads a case (parameters, boundary table, mesh in the reference's element /
 * face / side order) from the ccfd_case structure of include/ccfd_b200.h and
 * restates, function by function, the reference's arithmetic.  Its own
 * correctness is pinned two ways (see tests/): against the golden CSVs of the
 * reference's regression suite (check/targetOutput/*.csv) and against the
 * compiled reference itself (oracle/_ref/, built from the reference sources).
 *
 * Equation numbers follow the reference files cited beside each function.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "ccfd_b200.h"

#define NV 4

typedef struct {
	double gam, gam1, gam1q, mu, Pr, pi, sqrt3q;
	int eqn, order, limiter, flux;
	const ccfd_case *cs;
	const double *eps2;
	int vacuum;
} orc;

/* ---------------- equation of state, src/equationOfState.c:19-110 -------- */
static void o_prim_cons(const orc *o, const double p[4], double c[4])
{
	c[0] = p[0];
	c[1] = p[1] * p[0];
	c[2] = p[2] * p[0];
	c[3] = o->gam1q * p[3] + 0.5 * (c[1] * p[1] + c[2] * p[2]);
}

static void o_cons_prim(const orc *o, const double c[4], double p[4])
{
	p[0] = c[0];
	p[1] = c[1] / c[0];
	p[2] = c[2] / c[0];
	p[3] = o->gam1 * (c[3] - 0.5 * (c[1] * p[1] + c[2] * p[2]));
	if (p[0] < 1e-19)
		p[0] = 1e-10;
	if (p[3] < 1e-19)
		p[3] = 1e-10;
}

static void o_cons_char(const orc *o, const double c[4], double ch[3], const double r[4])
{
	double a = sqrt(o->gam * r[3] / r[0]);
	double u = r[1];
	double H = o->gam1q * a * a + 0.5 * u * u;
	double phi = u * u - 2.0 * H;
	double a1 = 1.0 / (2.0 * a * phi), a2 = 1.0 / phi, a3 = u * a;
	double v[3] = {c[0], c[1], c[3]};
	double K[3][3] = {
		{a1 * u * (phi - a3), -a1 * (phi - 2.0 * a3), -a2},
		{a2 * (u * u + phi), -2.0 * u * a2, 2.0 * a2},
		{-a1 * u * (a3 + phi), a1 * (phi + 2.0 * a3), -a2}};
	for (int i = 0; i < 3; ++i) {
		ch[i] = 0.0;
		for (int j = 0; j < 3; ++j)
			ch[i] += K[i][j] * v[j];
	}
}

static void o_char_cons(const orc *o, const double ch[3], double c[4], const double r[4])
{
	double u = r[1];
	double a = sqrt(o->gam * r[3] / r[0]);
	double H = o->gam1q * a * a + 0.5 * u * u;
	double K[3][3] = {{1.0, 1.0, 1.0}, {u - a, u, u + a},
			  {H - u * a, 0.5 * u * u, H + u * a}};
	double v[3] = {0.0, 0.0, 0.0};
	for (int i = 0; i < 3; ++i)
		for (int j = 0; j < 3; ++j)
			v[i] += K[i][j] * ch[j];
	c[0] = v[0];
	c[1] = v[1];
	c[3] = v[2];
}

/* ---------------- exact Riemann solver, src/exactRiemann.c:29-214 -------- */
static void o_prefun(const double G[9], double *f, double *fd, double p,
		     double rk, double pk, double ck)
{
	if (p < pk) {
		double q = p / pk;
		*f = G[3] * ck * (pow(q, G[0]) - 1.0);
		*fd = (1.0 / (rk * ck)) * pow(q, -G[1]);
	} else {
		double ak = G[4] / rk, bk = G[5] * pk;
		double qrt = sqrt(ak / (bk + p));
		*f = (p - pk) * qrt;
		*fd = (1.0 - 0.5 * (p - pk) / (bk + p)) * qrt;
	}
}

static void o_riemann(orc *o, double rl, double rr, double *rho, double ul, double ur,
		      double *u, double pl, double pr, double *p, double al, double ar,
		      double s)
{
	double g = o->gam, G[9];
	G[0] = (g - 1.0) / (2.0 * g); G[1] = (g + 1.0) / (2.0 * g);
	G[2] = 2.0 * g / (g - 1.0); G[3] = 2.0 / (g - 1.0); G[4] = 2.0 / (g + 1.0);
	G[5] = (g - 1.0) / (g + 1.0); G[6] = 0.5 * (g - 1.0); G[7] = 1.0 / g;
	G[8] = g - 1.0;
	double du = ur - ul;
	if (G[3] * (al + ar) - du < 0.0) {
		o->vacuum = 1;
		*rho = rl; *u = ul; *p = pl;
		return;
	}
	double tol = 1e-6;
	double pv = 0.5 * (pl + pr) - 0.125 * (ur - ul) * (rl + rr) * (al + ar);
	double pmin = fmin(pl, pr), pmax = fmax(pl, pr);
	if ((pmax / pmin < 2.0) && (pmin < pv) && (pv < pmax)) {
		*p = fmax(tol, pv);
	} else if (pv < pmin) {
		double pnu = al + ar - G[6] * (ur - ul);
		double pde = al / pow(pl, G[0]) + ar / pow(pr, G[0]);
		*p = pow(pnu / pde, G[2]);
	} else {
		double gel = sqrt((G[4] / rl) / (G[5] * pl + fmax(tol, pv)));
		double ger = sqrt((G[4] / rr) / (G[5] * pr + fmax(tol, pv)));
		*p = (gel * pl + ger * pr - (ur - ul)) / (gel + ger);
		*p = fmax(tol, *p);
	}
	double p0 = *p, cha = 2.0 * tol, fr = 0, fl = 0, frd = 0, fld = 0;
	for (int k = 0; cha > tol && k < 1000; ++k) {
		o_prefun(G, &fl, &fld, *p, rl, pl, al);
		o_prefun(G, &fr, &frd, *p, rr, pr, ar);
		*p -= (fl + fr + du) / (fld + frd);
		cha = 2.0 * fabs((*p - p0) / (*p + p0));
		if (*p < 0.0)
			*p = tol;
		p0 = *p;
	}
	*u = 0.5 * (ul + ur + fr - fl);
	double pm = *p, um = *u;
	if (s < um) {
		if (pm < pl) {
			if (s < ul - al) {
				*rho = rl; *u = ul; *p = pl;
			} else if (s > um - al * pow(pm / pl, G[0])) {
				*rho = rl * pow(pm / pl, G[7]); *u = um; *p = pm;
			} else {
				*u = G[4] * (al + G[6] * ul + s);
				double c = G[4] * (al + G[6] * (ul - s));
				*rho = rl * pow(c / al, G[3]);
				*p = pl * pow(c / al, G[2]);
			}
		} else {
			double q = pm / pl;
			if (s < ul - al * sqrt(G[1] * q + G[0])) {
				*rho = rl; *u = ul; *p = pl;
			} else {
				*rho = rl * (q + G[5]) / (q * G[5] + 1.0); *u = um; *p = pm;
			}
		}
	} else {
		if (pm > pr) {
			double q = pm / pr;
			if (s > ur + ar * sqrt(G[1] * q + G[0])) {
				*rho = rr; *u = ur; *p = pr;
			} else {
				*rho = rr * (q + G[5]) / (q * G[5] + 1.0); *u = um; *p = pm;
			}
		} else if (s > ur + ar) {
			*rho = rr; *u = ur; *p = pr;
		} else if (s < um + ar * pow(pm / pr, G[0])) {
			*rho = rr * pow(pm / pr, G[7]); *u = um; *p = pm;
		} else {
			*u = G[4] * (-ar + G[6] * ur + s);
			double c = G[4] * (ar - G[6] * (ur - s));
			*rho = rr * pow(c / ar, G[3]);
			*p = pr * pow(c / ar, G[2]);
		}
	}
}

/* ---------------- exactFunc, src/exactFunction.c:35-183 ------------------ */
static void o_exact(orc *o, int which, const double x[2], double t, double pv[4])
{
	const ccfd_exact *E = &o->cs->exact;
	switch (which) {
	case 1: {
		double xl = E->x_max - E->x_min, yl = E->y_max - E->y_min;
		pv[0] = 1.0; pv[1] = 0.0; pv[2] = 0.0; pv[3] = 1.0;
		if (x[0] >= 0.3 * xl + 1.0 / 30.0 * xl * cos(2.0 * o->pi * 3.0 / yl * x[1]))
			pv[0] = 0.25;
		if ((x[0] <= 0.1 * xl) && (x[0] >= 1.0 / 30.0 * xl)) {
			pv[0] = 4.22; pv[3] = 4.9;
		}
		return;
	}
	case 2: {
		double hw = fmin(E->x_max - E->x_min, E->y_max - E->y_min) / 100.0 * 6.0;
		double xp = E->x_min + 0.5 * (E->x_max - E->x_min);
		double yp = E->y_min + 0.5 * (E->y_max - E->y_min);
		double dr2 = (x[0] - xp) * (x[0] - xp) + (x[1] - yp) * (x[1] - yp);
		pv[0] = 1.0; pv[1] = 0.0; pv[2] = 0.0;
		pv[3] = 1.0 + 1.0 * pow(exp(-log(2.0)), dr2 / (hw * hw));
		return;
	}
	case 3: {
		double r[4];
		r[0] = r[1] = r[2] = 2.0 + 0.1 * sin(o->pi * 1.0 * (x[0] + x[1]) - 2.0 * o->pi * t);
		r[3] = r[0] * r[0];
		o_cons_prim(o, r, pv);
		return;
	}
	case 4: {
		double fac = o->pi / (0.2 * E->dx_ref);
		static const double cs[4] = {9.4, 57.157676649772950686, -33.0, 566.0};
		static const double cd[4] = {6.6, 57.157676649772950686, -33.0, 561.0};
		double c[4];
		for (int i = 0; i < 4; ++i)
			c[i] = 0.5 * (cs[i] - cd[i] * tanh((x[0] - (1.0 / 6.0 + (20.0 * t + x[1]) * o->sqrt3q)) * fac));
		pv[0] = c[0];
		pv[1] = c[1] / c[0];
		pv[2] = c[2] / c[0];
		pv[3] = o->gam1 * (c[3] - 0.5 * (c[1] * c[1] + c[2] * c[2]) / c[0]);
		return;
	}
	case 5: {
		const double *L = E->ref_state[0], *R = E->ref_state[1];
		double cl = sqrt(o->gam * L[3] / L[0]), cr = sqrt(o->gam * R[3] / R[0]);
		if (t == 0.0) {
			const double *S = x[0] <= E->rp1d_interface ? L : R;
			pv[0] = S[0]; pv[1] = S[1]; pv[3] = S[3];
		} else {
			o_riemann(o, L[0], R[0], &pv[0], L[1], R[1], &pv[1], L[3], R[3], &pv[3],
				  cl, cr, (x[0] - E->rp1d_interface) / t);
		}
		pv[2] = 0.0;
		return;
	}
	case 6: {
		double c0v[4] = {1.0, 0.1, 0.0, 1.0}, p0[4];
		o_cons_prim(o, c0v, p0);
		double a0 = sqrt(o->gam * p0[3] / p0[0]);
		double H0 = (c0v[3] + p0[3]) / p0[0];
		double R[4][4] = {{1.0, 1.0, 0.0, 1.0},
				  {p0[1] - a0, p0[1], 0.0, p0[1] + a0},
				  {p0[2], p0[2], 1.0, p0[2]},
				  {H0 - p0[1] * a0, (p0[1] * p0[1] + p0[2] * p0[2]) / 2.0, p0[2], H0 + p0[1] * a0}};
		double vec[4] = {0.0, 0.0, 0.0, 0.00001 * sin(o->pi * 1.0 * (x[0] - (a0 + p0[1]) * t))};
		double r[4];
		for (int i = 0; i < 4; ++i) {
			r[i] = c0v[i];
			for (int j = 0; j < 4; ++j)
				r[i] += R[i][j] * vec[j];
		}
		o_cons_prim(o, r, pv);
		return;
	}
	}
}

/* ---------------- ghost states, src/boundary.c:147-294 ------------------- */
static void o_boundary(orc *o, const ccfd_bc *bc, const double n[2], double t,
		       const double in[4], double gh[4], const double x[2])
{
	switch (bc->type) {
	case CCFD_BC_SLIPWALL:
	case CCFD_BC_WALL: {
		double vn = n[0] * in[1] + n[1] * in[2];
		double vt = -n[1] * in[1] + n[0] * in[2];
		double gn = -vn;
		double gt = (bc->type == CCFD_BC_WALL && o->mu > 0.0) ? -vt : vt;
		gh[1] = n[0] * gn - n[1] * gt;
		gh[2] = n[1] * gn + n[0] * gt;
		gh[0] = in[0];
		gh[3] = in[3];
		return;
	}
	case CCFD_BC_INFLOW:
		memcpy(gh, bc->pvar, sizeof(double) * 4);
		return;
	case CCFD_BC_OUTFLOW:
		memcpy(gh, in, sizeof(double) * 4);
		return;
	case CCFD_BC_CHARACTERISTIC: {
		const double *b = bc->pvar;
		double c = sqrt(o->gam * b[3] / b[0]);
		double v = n[0] * b[1] + n[1] * b[2];
		double il[4] = {in[0], n[0] * in[1] + n[1] * in[2], -n[1] * in[1] + n[0] * in[2], in[3]};
		double gl[4] = {b[0], n[0] * b[1] + n[1] * b[2], -n[1] * b[1] + n[0] * b[2], b[3]};
		double ic[4], gc[4], ich[3], gch[3];
		o_prim_cons(o, il, ic);
		o_prim_cons(o, gl, gc);
		o_cons_char(o, ic, ich, in);
		o_cons_char(o, gc, gch, in);
		if (v + c > 0.0) gch[2] = ich[2];
		if (v > 0.0) gch[1] = ich[1];
		if (v - c > 0.0) gch[0] = ich[0];
		o_char_cons(o, gch, gc, in);
		if (v > 0.0)
			gc[2] = ic[2];
		o_cons_prim(o, gc, gh);
		double a = gh[1], b2 = gh[2];
		gh[1] = n[0] * a - n[1] * b2;
		gh[2] = n[1] * a + n[0] * b2;
		return;
	}
	case CCFD_BC_EXACTSOL:
		o_exact(o, bc->exact_func, x, t, gh);
		return;
	case CCFD_BC_PRESSURE_OUT: {
		double c = sqrt(o->gam * in[3] / in[0]);
		double v = n[0] * in[1] + n[1] * in[2];
		double p = (v / c < 1.0) ? bc->pvar[3] : in[3];
		gh[0] = in[0] * p / in[3];
		gh[1] = in[1];
		gh[2] = in[2];
		gh[3] = p;
		return;
	}
	default:
		memcpy(gh, in, sizeof(double) * 4);
	}
}

/* ---------------- convective fluxes, src/fluxCalculation.c:30-844 -------- */
typedef struct { double rl, rr, ul, ur, vl, vr, pl, pr; } fin;

static double o_energy(const orc *o, double r, double u, double v, double p)
{
	return o->gam1q * p + 0.5 * r * (u * u + v * v);
}

static void o_hll_like(const double arp, const double alm, const double fL[4],
		       const double fR[4], const double uL[4], const double uR[4], double f[4])
{
	double q = 1.0 / (arp - alm);
	for (int i = 0; i < 4; ++i) {
		if (alm > 0.0)
			f[i] = fL[i];
		else if (arp < 0.0)
			f[i] = fR[i];
		else
			f[i] = (arp * fL[i] - alm * fR[i]) * q + (arp * alm) * q * (uR[i] - uL[i]);
	}
}

static void o_flux(orc *o, const fin *s, double f[4])
{
	const double g = o->gam, g1 = o->gam1, g1q = o->gam1q;
	const double rl = s->rl, rr = s->rr, ul = s->ul, ur = s->ur, vl = s->vl, vr = s->vr;
	const double pl = s->pl, pr = s->pr;
	switch (o->flux) {
	case CCFD_FLUX_GODUNOV: {
		double rho, vx, p;
		o_riemann(o, rl, rr, &rho, ul, ur, &vx, pl, pr, &p, sqrt(g * pl / rl),
			  sqrt(g * pr / rr), 0.0);
		double vy = vx > 0.0 ? vl : vr;
		f[0] = rho * vx;
		f[1] = rho * vx * vx + p;
		f[2] = rho * vx * vy;
		f[3] = vx * (g / g1 * p + 0.5 * rho * (vx * vx + vy * vy));
		return;
	}
	case CCFD_FLUX_ROE: {
		double mxl = rl * ul, mxr = rr * ur, myl = rl * vl, myr = rr * vr;
		double er = g1q * pr + 0.5 * rr * (ur * ur + vr * vr);
		double el = g1q * pl + 0.5 * rl * (ul * ul + vl * vl);
		double Hr = (er + pr) / rr, Hl = (el + pl) / rl;
		double sr = sqrt(rr), sl = sqrt(rl), sq = 1.0 / (sl + sr);
		double ub = (sr * ur + sl * ul) * sq, vb = (sr * vr + sl * vl) * sq;
		double Hb = (sr * Hr + sl * Hl) * sq;
		double cb = sqrt(g1 * (Hb - 0.5 * (ub * ub + vb * vb)));
		double lam[4] = {ub - cb, ub, ub, ub + cb};
		double r1[4] = {1.0, lam[0], vb, Hb - ub * cb};
		double r2[4] = {1.0, ub, vb, 0.5 * (ub * ub + vb * vb)};
		double r3[4] = {0.0, 0.0, 1.0, vb};
		double r4[4] = {1.0, lam[3], vb, Hb + ub * cb};
		double dr = rr - rl, dmx = mxr - mxl, dmy = myr - myl, de = er - el;
		double deq = de - (dmy - vb * dr) * vb;
		double cq = 1.0 / cb;
		double a2 = -g1 * cq * cq * (dr * (ub * ub - Hb) + deq - dmx * ub);
		double a1 = -0.5 * cq * (dmx - dr * (ub + cb)) - 0.5 * a2;
		double a4 = dr - a1 - a2;
		double a3 = dmy - vb * dr;
		double fr[4] = {mxr, mxr * ur + pr, mxr * vr, ur * (er + pr)};
		double fl[4] = {mxl, mxl * ul + pl, mxl * vl, ul * (el + pl)};
		double cl = sqrt(g * pl / rl), cr = sqrt(g * pr / rr);
		double lL[4] = {ul - cl, ul, ul, ul + cl}, lR[4] = {ur - cr, ur, ur, ur + cr};
		for (int i = 0; i < 4; ++i) {
			double da = fmax(fmax(0.0, lam[i] - lL[i]), lR[i] - lam[i]);
			lam[i] = fabs(lam[i]) < da ? 0.5 * (lam[i] * lam[i] / da + da) : fabs(lam[i]);
		}
		for (int i = 0; i < 4; ++i)
			f[i] = 0.5 * (fr[i] + fl[i] - a1 * fabs(lam[0]) * r1[i] - a2 * fabs(lam[1]) * r2[i]
				      - a3 * fabs(lam[2]) * r3[i] - a4 * fabs(lam[3]) * r4[i]);
		return;
	}
	case CCFD_FLUX_HLL:
	case CCFD_FLUX_HLLE:
	case CCFD_FLUX_HLLC: {
		double rlq = 1.0 / rl, rrq = 1.0 / rr;
		double sl = sqrt(rl), sr = sqrt(rr), sq = 1.0 / (sl + sr);
		double er = g1q * pr + 0.5 * rr * (ur * ur + vr * vr);
		double el = g1q * pl + 0.5 * rl * (ul * ul + vl * vl);
		double uL[4] = {rl, rl * ul, rl * vl, el}, uR[4] = {rr, rr * ur, rr * vr, er};
		double fL[4] = {uL[1], uL[1] * ul + pl, uL[1] * vl, ul * (el + pl)};
		double fR[4] = {uR[1], uR[1] * ur + pr, uR[1] * vr, ur * (er + pr)};
		double cl = sqrt(g * pl * rlq), cr = sqrt(g * pr * rrq);
		double um = (sr * ur + sl * ul) * sq;
		double arp, alm;
		if (o->flux == CCFD_FLUX_HLLE) {
			double eta2 = 0.5 * sr * sl / (sr + sl) / (sr + sl);
			double d = sqrt((sr * cr * cr + sl * cl * cl) * sq + eta2 * (ur - ul) * (ur - ul));
			arp = fmax(ur + cr, um + d);
			alm = fmin(ul - cl, um - d);
		} else {
			double Hl = (el + pl) * rlq, Hr = (er + pr) * rrq;
			double vm = (sr * vr + sl * vl) * sq;
			double Hm = (sr * Hr + sl * Hl) * sq;
			double cm = sqrt(g1 * (Hm - 0.5 * (um * um + vm * vm)));
			arp = fmax(ur + cr, um + cm);
			alm = fmin(ul - cl, um - cm);
		}
		if (o->flux != CCFD_FLUX_HLLC || alm > 0.0 || arp < 0.0) {
			o_hll_like(arp, alm, fL, fR, uL, uR, f);
			return;
		}
		double as = (pr - pl + uL[1] * (alm - ul) - uR[1] * (arp - ur)) /
			    (rl * (alm - ul) - rr * (arp - ur));
		if ((alm <= 0.0) && (as >= 0.0)) {
			double fac = rl * (alm - ul) / (alm - as);
			double us[4] = {fac, as * fac, vl * fac,
					fac * (el / rl + (as - ul) * (as + pl / (rl * (alm - ul))))};
			for (int i = 0; i < 4; ++i)
				f[i] = fL[i] + alm * (us[i] - uL[i]);
		} else {
			double fac = rr * (arp - ur) / (arp - as);
			double us[4] = {fac, as * fac, vr * fac,
					fac * (er / rr + (as - ur) * (as + pr / (rr * (arp - ur))))};
			for (int i = 0; i < 4; ++i)
				f[i] = fR[i] + arp * (us[i] - uR[i]);
		}
		return;
	}
	case CCFD_FLUX_LXF: {
		double a = fmax(fabs(ur) + sqrt(g * pr / rr), fabs(ul) + sqrt(g * pl / rl));
		double el = g1q * pl + 0.5 * rl * (ul * ul + vl * vl);
		double er = g1q * pr + 0.5 * rr * (ur * ur + vr * vr);
		double du[4] = {rr - rl, rr * ur - rl * ul, rr * vr - rl * vl, er - el};
		double fl[4] = {rl * ul, rl * ul * ul + pl, rl * ul * vl, ul * (el + pl)};
		double fr[4] = {rr * ur, rr * ur * ur + pr, rr * ur * vr, ur * (er + pr)};
		for (int i = 0; i < 4; ++i)
			f[i] = 0.5 * (fr[i] + fl[i]) - 0.5 * a * du[i];
		return;
	}
	case CCFD_FLUX_STEGER_WARMING: {
		double cl = sqrt(g * pl / rl), cr = sqrt(g * pr / rr), h = 0.5 / g;
		double ap[4] = {fmax(ul - cl, 0.0), fmax(ul, 0.0), fmax(ul, 0.0), fmax(ul + cl, 0.0)};
		double am[4] = {fmin(ur - cr, 0.0), fmin(ur, 0.0), fmin(ur, 0.0), fmin(ur + cr, 0.0)};
		double fp[4], fm[4];
		fp[0] = rl * h * (2.0 * g1 * ap[1] + ap[0] + ap[3]);
		fp[1] = fp[0] * ul + (ap[3] - ap[0]) * rl * cl * h;
		fp[2] = fp[0] * vl;
		fp[3] = fp[0] * 0.5 * (ul * ul + vl * vl) + (ap[3] - ap[0]) * rl * cl * ul * h +
			(ap[3] + ap[0]) * rl * cl * cl * h * g1q;
		fm[0] = rr * h * (2.0 * g1 * am[1] + am[0] + am[3]);
		fm[1] = fm[0] * ur + (am[3] - am[0]) * rr * cr * h;
		fm[2] = fm[0] * vr;
		fm[3] = fm[0] * 0.5 * (ur * ur + vr * vr) + (am[3] - am[0]) * rr * cr * ur * h +
			(am[3] + am[0]) * rr * cr * cr * h * g1q;
		for (int i = 0; i < 4; ++i)
			f[i] = fp[i] + fm[i];
		return;
	}
	case CCFD_FLUX_CENTRAL: {
		double el = o_energy(o, rl, ul, vl, pl), er = o_energy(o, rr, ur, vr, pr);
		double fl0 = rl * ul, fr0 = rr * ur;
		double fl[4] = {fl0, fl0 * ul + pl, fl0 * vl, ul * (el + pl)};
		double fr[4] = {fr0, fr0 * ur + pr, fr0 * vr, ur * (er + pr)};
		for (int i = 0; i < 4; ++i)
			f[i] = 0.5 * (fl[i] + fr[i]);
		return;
	}
	case CCFD_FLUX_AUSMD:
	case CCFD_FLUX_AUSMDV: {
		double el = o_energy(o, rl, ul, vl, pl), er = o_energy(o, rr, ur, vr, pr);
		double Hl = (el + pl) / rl, Hr = (er + pr) / rr;
		double cl = sqrt(g * pl / rl), cr = sqrt(g * pr / rr);
		double cm = fmax(cl, cr);
		double al = 2.0 * pl / rl / (pl / rl + pr / rr);
		double ar = 2.0 * pr / rr / (pl / rl + pr / rr);
		double up, pp, um, pm;
		if (o->flux == CCFD_FLUX_AUSMD) {
			if (fabs(ul) < cm) {
				up = 0.25 * al * (ul + cm) * (ul + cm) / cm + 0.5 * (1.0 - al) * (ul + fabs(ul));
				pp = 0.25 * pl * (ul + cm) * (ul + cm) / (cm * cm) * (2.0 - ul / cm);
			} else {
				up = 0.5 * (ul + fabs(ul));
				pp = 0.5 * pl * (ul + fabs(ul)) / ul;
			}
			if (fabs(ur) < cm) {
				um = -0.25 * ar * (ur - cm) * (ur - cm) / cm + 0.5 * (1.0 - ar) * (ur - fabs(ur));
				pm = 0.25 * pr * (ur - cm) * (ur - cm) / (cm * cm) * (2.0 + ur / cm);
			} else {
				um = 0.5 * (ur - fabs(ur));
				pm = 0.5 * pr * (ur - fabs(ur)) / ur;
			}
			double ru = up * rl + um * rr;
			f[0] = ru;
			f[1] = 0.5 * (ru * (ur + ul) - fabs(ru) * (ur - ul)) + (pp + pm);
			f[2] = 0.5 * (ru * (vr + vl) - fabs(ru) * (vr - vl));
			f[3] = 0.5 * (ru * (Hr + Hl) - fabs(ru) * (Hr - Hl));
			return;
		}
		if (fabs(ul) < cm) {
			pp = 0.25 * pl * (ul + cm) * (ul + cm) / (cm * cm) * (2.0 - ul / cm);
			up = ul > 0.0 ? ul + al * (ul - cm) * (ul - cm) : al * (ul + cm) * (ul + cm);
		} else if (ul > 0.0) {
			up = ul; pp = pl;
		} else {
			up = 0.0; pp = 0.0;
		}
		if (fabs(ur) < cm) {
			pm = 0.25 * pr * (ur - cm) * (ur - cm) / (cm * cm) * (2.0 + ur / cm);
			um = ur > 0.0 ? -ar * (ul - cm) * (ul - cm) : ur - ar * (ur + cm) * (ur + cm);
		} else if (ur > 0.0) {
			um = 0.0; pm = 0.0;
		} else {
			um = ur; pm = pr;
		}
		double ru = up * rl + um * rr;
		double sw = fmin(1.0, 10.0 * fabs(pr - pl) / fmin(pr, pl));
		double ru2 = 0.5 * (1.0 + sw) * (rl * ul * up + rr * ur * um);
		ru2 += 0.25 * (1.0 - sw) * (ru * (ur + ul) - fabs(ru) * (ur - ul));
		f[0] = ru;
		f[1] = ru2 + (pp + pm);
		f[2] = 0.5 * (ru * (vr + vl) - fabs(ru) * (vr - vl));
		f[3] = 0.5 * (ru * (Hr + Hl) - fabs(ru) * (Hr - Hl));
		int ta = (ul - cl < 0.0) && (ur - cr > 0.0);
		int tb = (ul + cl < 0.0) && (ur + cr > 0.0);
		double tl[4] = {1.0, ul, vl, Hl}, tr[4] = {1.0, ur, vr, Hr};
		if (ta && !tb)
			for (int i = 0; i < 4; ++i)
				f[i] -= 0.125 * ((ur - cr) - (ul - cl)) * (rr * tr[i] - rl * tl[i]);
		if (!ta && tb)
			for (int i = 0; i < 4; ++i)
				f[i] -= 0.125 * ((ur + cr) - (ul + cl)) * (rr * tr[i] - rl * tl[i]);
		return;
	}
	case CCFD_FLUX_VANLEER: {
		double cl = sqrt(g * pl / rl), cr = sqrt(g * pr / rr);
		double el = o_energy(o, rl, ul, vl, pl), er = o_energy(o, rr, ur, vr, pr);
		double Hl = (el + pl) / rl, Hr = (er + pr) / rr;
		double fp[4] = {0, 0, 0, 0}, fm[4] = {0, 0, 0, 0};
		double ML = ul / cl, MR = ur / cr;
		if (ML > 1.0) {
			fp[0] = rl * ul; fp[1] = fp[0] * ul + pl; fp[2] = fp[0] * vl; fp[3] = fp[0] * Hl;
		} else if ((ML < 1.0) && (ML > -1.0)) {
			double cx = g1 * ul + 2.0 * cl;
			fp[0] = 0.25 * rl * cl * (ML + 1.0) * (ML + 1.0);
			fp[1] = fp[0] * cx / g;
			fp[2] = fp[0] * vl;
			fp[3] = 0.5 * (fp[1] * cx * g / (g * g - 1.0) + fp[2] * vl);
		}
		if (MR < -1.0) {
			fm[0] = rr * ur; fm[1] = fm[0] * ur + pr; fm[2] = fm[0] * vr; fm[3] = fm[0] * Hr;
		} else if ((MR < 1.0) && (MR > -1.0)) {
			double cx = g1 * ur - 2.0 * cr;
			fm[0] = -0.25 * rr * cr * (1.0 - MR) * (1.0 - MR);
			fm[1] = fm[0] * cx / g;
			fm[2] = fm[0] * vr;
			fm[3] = 0.5 * (fm[1] * cx * g / (g * g - 1.0) + fm[2] * vr);
		}
		for (int i = 0; i < 4; ++i)
			f[i] = fp[i] + fm[i];
		return;
	}
	}
}

/* ---------------- residual, src/finiteVolume.c:78-121 -------------------- */
static void o_init(orc *o, const ccfd_case *cs, const double *eps2)
{
	const ccfd_params *p = &cs->params;
	o->gam = p->gamma;
	o->gam1 = p->gamma - 1.0;
	o->gam1q = 1.0 / o->gam1;
	o->eqn = p->eqn;
	o->mu = p->eqn == CCFD_NAVIER_STOKES ? p->mu : 0.0;
	o->Pr = p->eqn == CCFD_NAVIER_STOKES ? p->Pr : 0.72;
	o->pi = acos(-1.0);
	o->sqrt3q = 1 / sqrt(3.0);
	o->order = p->spatial_order;
	o->limiter = p->limiter;
	o->flux = p->flux;
	o->cs = cs;
	o->eps2 = eps2;
	o->vacuum = 0;
}

/* evalSource, source function 1 (src/source.c:22-60): source of the
 * manufactured sine-wave solution (exactFunc 3) */
static void o_source(const orc *o, const double x[2], double t, double s[4])
{
	double freq = 1.0, amp = 0.1;
	double om = o->pi * freq;
	double a = 2.0 * o->pi;
	double tmp1 = cos(om * (x[0] + x[1]) - a * t);
	double tmp2 = sin(2.0 * (om * (x[0] + x[1]) - a * t));
	s[0] = (-a + 2.0 * om) * tmp1;
	s[1] = (-a + om * (o->gam * 3.0 - 1.0)) * tmp1 + amp * om * o->gam1 * tmp2;
	s[2] = s[1];
	if (o->eqn == CCFD_NAVIER_STOKES) {
		double tmp3 = sin(om * (x[0] + x[1]) - a * t);
		s[3] = ((2.0 + o->gam * 6.0) * om - 4.0 * a) * tmp1 + amp * (2.0 * om * o->gam - a) * tmp2 +
		       2.0 * o->mu * o->gam * om * om / o->Pr * tmp3;
	} else {
		s[3] = ((2.0 + o->gam * 6.0) * om - 4.0 * a) * tmp1 + amp * (2.0 * om * o->gam - a) * tmp2;
	}
	for (int v = 0; v < NV; ++v)
		s[v] *= amp;
}

/* element quadrature points and weights (createReconstructionInfo,
 * src/mesh.c:114-161): bary + side GP in side order (area/3 for triangles,
 * area/6 for quads), then a quad's fifth point, the midpoint of nodes 0 and
 * 2, with area/3; returns the point count */
static int o_elem_gp(const ccfd_mesh *m, long c, double x[5][2], double w[5])
{
	long h0 = m->hs_offset[c], h1 = m->hs_offset[c + 1];
	int ns = (int)(h1 - h0);
	double area = m->cell_geo[4 * c];
	const double *b = &m->cell_bary[2 * c];
	for (int k = 0; k < ns; ++k) {
		x[k][0] = b[0] + m->hs_gp[2 * (h0 + k)];
		x[k][1] = b[1] + m->hs_gp[2 * (h0 + k) + 1];
		w[k] = ns == 4 ? area / 6.0 : area / 3.0;
	}
	if (ns == 4) {
		x[4][0] = m->cell_gp5[2 * c];
		x[4][1] = m->cell_gp5[2 * c + 1];
		w[4] = area / 3.0;
		return 5;
	}
	return ns;
}

/* calcSource (src/source.c:66-85) for element c */
static void o_cell_source(const orc *o, const ccfd_mesh *m, long c, double t, double src[4])
{
	double x[5][2], w[5], s[4];
	int n = o_elem_gp(m, c, x, w);
	for (int v = 0; v < NV; ++v)
		src[v] = 0.0;
	for (int k = 0; k < n; ++k) {
		o_source(o, x[k], t, s);
		for (int v = 0; v < NV; ++v)
			src[v] += s[v] * w[k];
	}
}

/* ghost-cell state at the mirrored barycentre of ghost b (setBCatBarys) */
static void o_ghost_bary(orc *o, long b, double t, const double *prim, double out[4])
{
	const ccfd_mesh *m = &o->cs->mesh;
	long f = m->bc_face[b];
	long c = m->face_cells[2 * f];
	o_boundary(o, &o->cs->bc_table[m->bc_index[b]], &m->face_n[2 * f], t, &prim[4 * c], out,
		   &m->bc_ghost_bary[2 * b]);
}

/* Limited least-squares gradient of cell c (spatialReconstruction,
 * src/reconstruction.c:252-275, limiters :25-192): neighbour states from
 * prim, ghost states at the mirrored barycentres from gb; g = (u_x[4],
 * u_y[4]). */
static void o_gradient(const orc *o, const ccfd_mesh *m, const double *prim, const double *gb,
		       long c, double g[8])
{
	const double *q = &prim[4 * c];
	double *ux = g, *uy = g + 4;
	for (int v = 0; v < NV; ++v)
		ux[v] = uy[v] = 0.0;
	for (long h = m->hs_offset[c]; h < m->hs_offset[c + 1]; ++h) {
		long nb = m->hs_nb[h];
		const double *qn = nb >= 0 ? &prim[4 * nb] : &gb[4 * (-1 - nb)];
		for (int v = 0; v < NV; ++v) {
			double d = qn[v] - q[v];
			ux[v] += m->hs_w[2 * h] * d;
			uy[v] += m->hs_w[2 * h + 1] * d;
		}
	}
	double lo[4], hi[4], phi[4] = {1.0, 1.0, 1.0, 1.0};
	memcpy(lo, q, sizeof(lo));
	memcpy(hi, q, sizeof(hi));
	for (long h = m->hs_offset[c]; h < m->hs_offset[c + 1]; ++h) {
		long nb = m->hs_nb[h];
		const double *qn = nb >= 0 ? &prim[4 * nb] : &gb[4 * (-1 - nb)];
		for (int v = 0; v < NV; ++v) {
			lo[v] = fmin(lo[v], qn[v]);
			hi[v] = fmax(hi[v], qn[v]);
		}
	}
	for (long h = m->hs_offset[c]; h < m->hs_offset[c + 1]; ++h) {
		for (int v = 0; v < NV; ++v) {
			double mn = lo[v] - q[v], mx = hi[v] - q[v];
			double d = ux[v] * m->hs_gp[2 * h] + uy[v] * m->hs_gp[2 * h + 1];
			double ph = 1.0;
			if (o->limiter == CCFD_LIM_BARTH_JESPERSEN) {
				/* src/reconstruction.c:25-96 */
				if (d > 0.0)
					ph = fmin(1.0, mx / d);
				else if (d < 0.0)
					ph = fmin(1.0, mn / d);
			} else {
				/* src/reconstruction.c:103-192 */
				double e2 = o->eps2[c], d2 = d * d;
				if (d > 0.0)
					ph = 1.0 / d * (((mx * mx + e2) * d + 2.0 * d2 * mx) /
							(mx * mx + 2.0 * d2 + d * mx + e2));
				else if (d < 0.0)
					ph = 1.0 / d * (((mn * mn + e2) * d + 2.0 * d2 * mn) /
							(mn * mn + 2.0 * d2 + d * mn + e2));
			}
			phi[v] = fmin(phi[v], ph);
		}
	}
	for (int v = 0; v < NV; ++v) {
		ux[v] *= phi[v];
		uy[v] *= phi[v];
	}
}

/* Flux of face f times its length (setBCatSides + fluxCalculation,
 * src/boundary.c:300-314, src/fluxCalculation.c:882-998): gradients g
 * ([N][8], zero in first order), ghost states gb. */
static void o_face_flux(orc *o, const ccfd_case *cs, const double *prim, const double *g,
			const double *gb, long f, double t, double F4[4], double *wall_p)
{
	const ccfd_mesh *m = &cs->mesh;
	long c0 = m->face_cells[2 * f], c1 = m->face_cells[2 * f + 1];
	long h0 = m->face_hs[2 * f], h1 = m->face_hs[2 * f + 1];
	const double *n = &m->face_n[2 * f];
	double L[4], R[4], q1[4] = {0, 0, 0, 0};
	const double *g1x = NULL, *g1y = NULL;
	static const double zero4[4] = {0, 0, 0, 0};
	for (int v = 0; v < NV; ++v)
		L[v] = prim[4 * c0 + v] + m->hs_gp[2 * h0] * g[8 * c0 + v] +
		       m->hs_gp[2 * h0 + 1] * g[8 * c0 + 4 + v];
	if (c1 >= 0) {
		for (int v = 0; v < NV; ++v) {
			R[v] = prim[4 * c1 + v] + m->hs_gp[2 * h1] * g[8 * c1 + v] +
			       m->hs_gp[2 * h1 + 1] * g[8 * c1 + 4 + v];
			q1[v] = prim[4 * c1 + v];
		}
		g1x = &g[8 * c1];
		g1y = &g[8 * c1 + 4];
	} else {
		long b = -1 - c1;
		o_boundary(o, &cs->bc_table[m->bc_index[b]], n, t, L, R, &m->bc_x[2 * b]);
		if (wall_p)
			wall_p[b] = L[3];
		memcpy(q1, &gb[4 * b], sizeof(q1));
		g1x = g1y = zero4;
	}
	fin s = {L[0], R[0], n[0] * L[1] + n[1] * L[2], n[0] * R[1] + n[1] * R[2],
		 -n[1] * L[1] + n[0] * L[2], -n[1] * R[1] + n[0] * R[2], L[3], R[3]};
	double fc[4];
	o_flux(o, &s, fc);
	F4[0] = fc[0];
	F4[1] = n[0] * fc[1] - n[1] * fc[2];
	F4[2] = n[1] * fc[1] + n[0] * fc[2];
	F4[3] = fc[3];
	if (o->eqn == CCFD_NAVIER_STOKES) {
		const double *bb = &m->face_bb[3 * f];
		double bx = bb[0] / bb[2], by = bb[1] / bb[2];
		double st[4], gx[4], gy[4], fx[4], fy[4];
		for (int v = 0; v < NV; ++v) {
			st[v] = 0.5 * (R[v] + L[v]);
			double mx = 0.5 * (g[8 * c0 + v] + g1x[v]);
			double my = 0.5 * (g[8 * c0 + 4 + v] + g1y[v]);
			double corr = mx * bx + my * by - (q1[v] - prim[4 * c0 + v]) / bb[2];
			gx[v] = mx - corr * bx;
			gy[v] = my - corr * by;
		}
		/* diffusionFlux, src/fluxCalculation.c:855-873 */
		double mu = o->mu, k = o->gam / (o->gam1 * o->Pr * st[0] * st[0]);
		fx[0] = fy[0] = 0.0;
		fx[1] = (4.0 / 3.0 * gx[1] - 2.0 / 3.0 * gy[2]) * mu;
		fx[2] = (gy[1] + gx[2]) * mu;
		fx[3] = (4.0 / 3.0 * st[1] * gx[1] - 2.0 / 3.0 * st[1] * gy[2] + (gx[2] + gy[1]) * st[2]
			 + k * (st[0] * gx[3] - st[3] * gx[0])) * mu;
		fy[1] = (gy[1] + gx[2]) * mu;
		fy[2] = (4.0 / 3.0 * gy[2] - 2.0 / 3.0 * gx[1]) * mu;
		fy[3] = (4.0 / 3.0 * st[2] * gy[2] - 2.0 / 3.0 * st[2] * gx[1] + (gy[1] + gx[2]) * st[1]
			 + k * (st[0] * gy[3] - st[3] * gy[0])) * mu;
		for (int v = 0; v < NV; ++v)
			F4[v] -= (fx[v] * n[0] + fy[v] * n[1]);
	}
	for (int v = 0; v < NV; ++v)
		F4[v] *= m->face_len[f];
}

/* u_t of cell c from the face fluxes ff ([F][4]) in side-list order
 * (src/finiteVolume.c:96-120) */
static void o_cell_ut(const orc *o, const ccfd_case *cs, const double *ff, long c, double t,
		      double ut[4])
{
	const ccfd_mesh *m = &cs->mesh;
	double s[4] = {0.0, 0.0, 0.0, 0.0};
	for (long h = m->hs_offset[c]; h < m->hs_offset[c + 1]; ++h) {
		const double *F4 = &ff[4 * m->hs_face[h]];
		for (int v = 0; v < NV; ++v)
			s[v] += m->hs_sign[h] > 0 ? F4[v] : -F4[v];
	}
	double src[4] = {0.0, 0.0, 0.0, 0.0};
	if (cs->params.source_func)
		o_cell_source(o, m, c, t, src);
	for (int v = 0; v < NV; ++v)
		ut[v] = (src[v] - s[v]) * m->cell_geo[4 * c + 1];
}

static double *o_venk_eps2(const ccfd_case *cs)
{
	const ccfd_mesh *m = &cs->mesh;
	if (cs->params.spatial_order != 2 || cs->params.limiter != CCFD_LIM_VENKATAKRISHNAN)
		return NULL;
	double *eps2 = malloc(sizeof(double) * m->n_cells);
	if (!eps2)
		return NULL;
	for (long e = 0; e < m->n_cells; ++e) {
		double a = m->cell_geo[4 * e];
		eps2[e] = (cs->params.venk_k * sqrt(a)) * (cs->params.venk_k * sqrt(a)) *
			  (cs->params.venk_k * sqrt(a));
	}
	return eps2;
}

/* Residual R(U) of primitive state prim at time t.  grad (N x 8) and fflux
 * (F x 4) are optional outputs (limited gradients, face fluxes). */
int oracle_residual(const ccfd_case *cs, const double *prim, double t, double *u_t,
		    double *grad, double *fflux, double *wall_p)
{
	const ccfd_mesh *m = &cs->mesh;
	const long N = m->n_cells, F = m->n_faces, B = m->n_bc;
	orc o;
	double *eps2 = o_venk_eps2(cs);
	o_init(&o, cs, eps2);
	double *g = calloc(8 * N, sizeof(double));
	double *gb = calloc(4 * (B + 1), sizeof(double));
	double *ff = malloc(sizeof(double) * 4 * F);
	if (!g || !gb || !ff) {
		free(g); free(gb); free(ff); free(eps2);
		return CCFD_ERR_NOMEM;
	}
	/* spatialReconstruction, src/reconstruction.c:198-314 */
	if (o.order == 2) {
		for (long b = 0; b < B; ++b)
			o_ghost_bary(&o, b, t, prim, &gb[4 * b]);
		for (long c = 0; c < N; ++c)
			o_gradient(&o, m, prim, gb, c, &g[8 * c]);
	}
	for (long f = 0; f < F; ++f)
		o_face_flux(&o, cs, prim, g, gb, f, t, &ff[4 * f], wall_p);
	for (long c = 0; c < N; ++c)
		o_cell_ut(&o, cs, ff, c, t, &u_t[4 * c]);
	if (grad)
		memcpy(grad, g, sizeof(double) * 8 * N);
	if (fflux)
		memcpy(fflux, ff, sizeof(double) * 4 * F);
	int vac = o.vacuum;
	free(g); free(gb); free(ff); free(eps2);
	return vac ? CCFD_ERR_VACUUM : CCFD_OK;
}

/* calcErrors (src/analyze.c:445-514) of primitive state prim at time t
 * against exact function `which`: out = {L1[4], L2[4], Linf[4]}, summed in
 * element order */
int oracle_errors(const ccfd_case *cs, const double *prim, double t, int which, double out[12])
{
	const ccfd_mesh *m = &cs->mesh;
	const long N = m->n_cells;
	double *ut = malloc(sizeof(double) * 4 * N);
	double *g = calloc(8 * N, sizeof(double));
	if (!ut || !g) {
		free(ut); free(g);
		return CCFD_ERR_NOMEM;
	}
	int st = CCFD_OK;
	if (cs->params.spatial_order == 2)
		st = oracle_residual(cs, prim, t, ut, g, NULL, NULL);
	orc o;
	o_init(&o, cs, NULL);
	double L1[4] = {0, 0, 0, 0}, L2[4] = {0, 0, 0, 0}, Li[4] = {0, 0, 0, 0};
	for (long c = 0; c < N && st == CCFD_OK; ++c) {
		double x[5][2], w[5];
		int n = o_elem_gp(m, c, x, w);
		const double *b = &m->cell_bary[2 * c];
		for (int k = 0; k < n; ++k) {
			double ex[4];
			o_exact(&o, which, x[k], t, ex);
			double dx[2] = {x[k][0] - b[0], x[k][1] - b[1]};
			for (int v = 0; v < NV; ++v) {
				double q = prim[4 * c + v] + dx[0] * g[8 * c + v] + dx[1] * g[8 * c + 4 + v];
				double err = fabs(ex[v] - q);
				Li[v] = fmax(Li[v], err);
				L1[v] += err * w[k];
				L2[v] += err * err * w[k];
			}
		}
	}
	for (int v = 0; v < NV; ++v) {
		out[v] = L1[v] * m->total_area_q;
		out[4 + v] = sqrt(L2[v] * m->total_area_q);
		out[8 + v] = Li[v];
	}
	free(ut); free(g);
	return st;
}

/* ---------------- time loop, src/timeDiscretization.c:249-731 ----------- */
static const double rk_tab[3][3][5] = {
	{{0.1418, 0.4, 1.0}, {0.1918, 0.4929, 1.0}, {0.2884, 0.5010, 1.0}},
	{{0.0833, 0.2069, 0.4265, 1.0}, {0.1084, 0.2602, 0.5052, 1.0}, {0.1666, 0.3027, 0.5275, 1.0}},
	{{0.0533, 0.1263, 0.2375, 0.4414, 1.0}, {0.0695, 0.1602, 0.2898, 0.5060, 1.0},
	 {0.1067, 0.1979, 0.3232, 0.5201, 1.0}}};

/* calcTimeStep, src/timeDiscretization.c:249-329 */
int oracle_time_step(const ccfd_case *cs, const double *prim, double t, double print_time,
		     double *dt_out)
{
	const ccfd_params *p = &cs->params;
	const ccfd_mesh *m = &cs->mesh;
	double gam = p->gamma;
	double mu = p->eqn == CCFD_NAVIER_STOKES ? p->mu : 0.0;
	double Pr = p->eqn == CCFD_NAVIER_STOKES ? p->Pr : 0.72;
	double dt;
	if (p->time_step_1d) {
		double mx = 1e150;
		for (long c = 0; c < m->n_cells; ++c) {
			const double *q = &prim[4 * c];
			double a = sqrt(gam * q[3] / q[0]);
			double d = p->cfl * m->cell_geo[4 * c + 3] / (fabs(q[1]) + a);
			if (!isfinite(d))
				return CCFD_ERR_DT;
			mx = fmin(mx, d);
		}
		dt = mx;
	} else {
		double gpm = fmax(4.0 / 3.0, gam / Pr), dc = 1e150, dv = 1e150;
		for (long c = 0; c < m->n_cells; ++c) {
			const double *q = &prim[4 * c], *geo = &m->cell_geo[4 * c];
			double a = sqrt(gam * q[3] / q[0]);
			double d = p->cfl * geo[0] / ((fabs(q[1]) + a) * geo[2] + (fabs(q[2]) + a) * geo[3]);
			if (!isfinite(d))
				return CCFD_ERR_DT;
			dc = fmin(dc, d);
			if (mu > 1e-10) {
				double sr = gpm * mu * geo[2] * geo[2] + gpm * mu * geo[3] * geo[3];
				double v = p->dfl * q[0] * q[0] * geo[0] * geo[0] / (4.0 * sr);
				if (!isfinite(v))
					return CCFD_ERR_DT;
				dv = fmin(dv, v);
			}
		}
		dt = fmin(dc, dv);
	}
	if ((t + dt > print_time) || (t + dt > p->t_end))
		dt = fmin(print_time, p->t_end) - t;
	else if ((t + 1.5 * dt > print_time) || (t + 1.5 * dt > p->t_end))
		dt = 0.5 * (fmin(print_time, p->t_end) - t);
	*dt_out = dt;
	return CCFD_OK;
}

/* Explicit time loop of timeDisc (Euler / low-storage RK, globalResidual,
 * stop tests).  prim is updated in place; info[0..7] = t, iterations,
 * res[0..3], finished, converged. */
int oracle_run_explicit(const ccfd_case *cs, double *prim, long nsteps, double *info)
{
	const ccfd_params *p = &cs->params;
	const ccfd_mesh *m = &cs->mesh;
	const long N = m->n_cells;
	orc o;
	o_init(&o, cs, NULL);
	double rk[6] = {0, 0, 0, 0, 0, 0};
	int nrk;
	if (p->n_rk_stages == 1 && p->time_order == 1) {
		rk[1] = 1.0;
		nrk = 1;
	} else {
		nrk = p->n_rk_stages;
		for (int s = 0; s < nrk; ++s)
			rk[s + 1] = rk_tab[nrk - 3][p->time_order - 1][s];
	}
	double *cons = malloc(sizeof(double) * 4 * N), *cons0 = malloc(sizeof(double) * 4 * N);
	double *ut = malloc(sizeof(double) * 4 * N);
	if (!cons || !cons0 || !ut) {
		free(cons); free(cons0); free(ut);
		return CCFD_ERR_NOMEM;
	}
	for (long c = 0; c < N; ++c)
		o_prim_cons(&o, &prim[4 * c], &cons[4 * c]);
	double t = 0.0;
	double print_time = (floor(0.0 / p->io_time_interval) + 1) * p->io_time_interval;
	long io_iter = p->io_iter_interval > 0 ? p->io_iter_interval : 1;
	long print_iter = io_iter;
	double res[4] = {0, 0, 0, 0};
	int finished = 0, converged = 0, st = CCFD_OK;
	long iter;
	for (iter = 1; iter <= p->max_iter; ++iter) {
		if (nsteps > 0 && iter > nsteps) {
			iter--;
			break;
		}
		double dt;
		if ((st = oracle_time_step(cs, prim, t, print_time, &dt)) != CCFD_OK)
			break;
		memcpy(cons0, cons, sizeof(double) * 4 * N);
		for (int s = 1; s <= nrk; ++s) {
			if ((st = oracle_residual(cs, prim, t + rk[s - 1] * dt, ut, NULL, NULL, NULL)) != CCFD_OK)
				goto out;
			for (long c = 0; c < N; ++c) {
				for (int v = 0; v < NV; ++v)
					cons[4 * c + v] = cons0[4 * c + v] + rk[s] * dt * ut[4 * c + v];
				o_cons_prim(&o, &cons[4 * c], &prim[4 * c]);
			}
		}
		/* globalResidual, src/analyze.c:521-539 */
		double acc[4] = {0, 0, 0, 0};
		for (long c = 0; c < N; ++c)
			for (int v = 0; v < NV; ++v)
				acc[v] += m->cell_geo[4 * c] * ut[4 * c + v] * ut[4 * c + v];
		for (int v = 0; v < NV; ++v)
			res[v] = sqrt(acc[v] * m->total_area_q);
		t += dt;
		if (p->t_end - t <= 1e-15) {
			finished = 1;
			break;
		}
		if (p->stationary && fabs(res[p->abort_variable]) <= p->abort_residual) {
			converged = 1;
			break;
		}
		if ((print_time - t <= 1e-15) || (iter == print_iter)) {
			if (print_time - t <= 1e-15)
				print_time += p->io_time_interval;
			if (iter == print_iter)
				print_iter += io_iter;
		}
	}
out:
	if (iter > p->max_iter)
		iter = p->max_iter;
	info[0] = t;
	info[1] = (double)iter;
	for (int v = 0; v < 4; ++v)
		info[2 + v] = res[v];
	info[6] = finished;
	info[7] = converged;
	free(cons); free(cons0); free(ut);
	return st;
}

/* ======================================================================
 * Implicit path, restated: buildMatrix / calcDinv / LUSGS
 * (src/linearSolver.c:136-333) in block-sparse storage, and
 * implicitTimeStep / GMRES_M / matrixVector (src/timeDiscretization.c:
 * 412-552, src/linearSolver.c:343-510).
 *
 * The reference stores dRdU densely, (4N)^2 doubles, and obtains its
 * columns from 4N residual evaluations over the whole mesh; both are out of
 * reach beyond a few thousand cells.  Here a column (cell i, variable v)
 * is evaluated on the stencil it reaches: the residuals of cell i and of
 * its face neighbours, from the fluxes of their faces, the gradients of the
 * cells on those faces and the ghost states those gradients read -- the
 * same per-cell and per-face arithmetic as oracle_residual, so every
 * recorded residual equals the one a whole-mesh evaluation gives.
 * Columns run in the reference's order (cells, then variables); with
 * in_place the perturbation is undone by subtracting the step again, as
 * the reference does (pVar += rEps0 ... pVar -= rEps0), so the state and
 * every later column carry that rounding exactly as there.
 * ==================================================================== */

typedef struct {
	double *g, *gb, *ff;
	long *stamp_f, *stamp_c, *stamp_b, *faces, *cells;
	long stamp;
} olocal;

static void o_local_free(olocal *L)
{
	free(L->g); free(L->gb); free(L->ff);
	free(L->stamp_f); free(L->stamp_c); free(L->stamp_b); free(L->faces); free(L->cells);
}

static int o_local_init(olocal *L, const ccfd_mesh *m)
{
	const long N = m->n_cells, F = m->n_faces, B = m->n_bc;
	memset(L, 0, sizeof(*L));
	L->g = calloc(8 * N, sizeof(double));
	L->gb = calloc(4 * (B + 1), sizeof(double));
	L->ff = calloc(4 * F, sizeof(double));
	L->stamp_f = calloc(F, sizeof(long));
	L->stamp_c = calloc(N, sizeof(long));
	L->stamp_b = calloc(B + 1, sizeof(long));
	L->faces = malloc(sizeof(long) * F);
	L->cells = malloc(sizeof(long) * N);
	if (!L->g || !L->gb || !L->ff || !L->stamp_f || !L->stamp_c || !L->stamp_b || !L->faces ||
	    !L->cells) {
		o_local_free(L);
		return CCFD_ERR_NOMEM;
	}
	return CCFD_OK;
}

/* u_t (rows of ut) of the nt cells tgt at state prim and time t */
static void o_local_ut(orc *o, const ccfd_case *cs, olocal *L, const double *prim, double t,
		       const long *tgt, int nt, double *ut)
{
	const ccfd_mesh *m = &cs->mesh;
	long nf = 0, nc = 0, st = ++L->stamp;
	for (int k = 0; k < nt; ++k)
		for (long h = m->hs_offset[tgt[k]]; h < m->hs_offset[tgt[k] + 1]; ++h) {
			long f = m->hs_face[h];
			if (L->stamp_f[f] != st) {
				L->stamp_f[f] = st;
				L->faces[nf++] = f;
			}
		}
	if (o->order == 2) {
		for (long k = 0; k < nf; ++k)
			for (int s = 0; s < 2; ++s) {
				long c = m->face_cells[2 * L->faces[k] + s];
				if (c >= 0 && L->stamp_c[c] != st) {
					L->stamp_c[c] = st;
					L->cells[nc++] = c;
				}
			}
		for (long k = 0; k < nc; ++k)
			for (long h = m->hs_offset[L->cells[k]]; h < m->hs_offset[L->cells[k] + 1]; ++h) {
				long nb = m->hs_nb[h];
				if (nb >= 0 || L->stamp_b[-1 - nb] == st)
					continue;
				L->stamp_b[-1 - nb] = st;
				o_ghost_bary(o, -1 - nb, t, prim, &L->gb[4 * (-1 - nb)]);
			}
		for (long k = 0; k < nc; ++k)
			o_gradient(o, m, prim, L->gb, L->cells[k], &L->g[8 * L->cells[k]]);
	}
	for (long k = 0; k < nf; ++k)
		o_face_flux(o, cs, prim, L->g, L->gb, L->faces[k], t, &L->ff[4 * L->faces[k]], NULL);
	for (int k = 0; k < nt; ++k)
		o_cell_ut(o, cs, L->ff, tgt[k], t, &ut[4 * k]);
}

/* 4x4 inverse by Laplace expansion in complementary 2x2 minors of the first
 * two and the last two rows; 0 if |det| <= DBL_EPSILON (the singularity test
 * of calcDinv, src/linearSolver.c:155-157) */
static int o_inv4(const double *a, double *r)
{
	double s0 = a[0] * a[5] - a[4] * a[1], s1 = a[0] * a[6] - a[4] * a[2];
	double s2 = a[0] * a[7] - a[4] * a[3], s3 = a[1] * a[6] - a[5] * a[2];
	double s4 = a[1] * a[7] - a[5] * a[3], s5 = a[2] * a[7] - a[6] * a[3];
	double c5 = a[10] * a[15] - a[14] * a[11], c4 = a[9] * a[15] - a[13] * a[11];
	double c3 = a[9] * a[14] - a[13] * a[10], c2 = a[8] * a[15] - a[12] * a[11];
	double c1 = a[8] * a[14] - a[12] * a[10], c0 = a[8] * a[13] - a[12] * a[9];
	double det = s0 * c5 - s1 * c4 + s2 * c3 + s3 * c2 - s4 * c1 + s5 * c0;
	if (fabs(det) <= 2.220446049250313e-16)
		return 0;
	double q = 1.0 / det;
	r[0] = (a[5] * c5 - a[6] * c4 + a[7] * c3) * q;
	r[1] = (-a[1] * c5 + a[2] * c4 - a[3] * c3) * q;
	r[2] = (a[13] * s5 - a[14] * s4 + a[15] * s3) * q;
	r[3] = (-a[9] * s5 + a[10] * s4 - a[11] * s3) * q;
	r[4] = (-a[4] * c5 + a[6] * c2 - a[7] * c1) * q;
	r[5] = (a[0] * c5 - a[2] * c2 + a[3] * c1) * q;
	r[6] = (-a[12] * s5 + a[14] * s2 - a[15] * s1) * q;
	r[7] = (a[8] * s5 - a[10] * s2 + a[11] * s1) * q;
	r[8] = (a[4] * c4 - a[5] * c2 + a[7] * c0) * q;
	r[9] = (-a[0] * c4 + a[1] * c2 - a[3] * c0) * q;
	r[10] = (a[12] * s4 - a[13] * s2 + a[15] * s0) * q;
	r[11] = (-a[8] * s4 + a[9] * s2 - a[11] * s0) * q;
	r[12] = (-a[4] * c3 + a[5] * c1 - a[6] * c0) * q;
	r[13] = (a[0] * c3 - a[1] * c1 + a[2] * c0) * q;
	r[14] = (-a[12] * s3 + a[13] * s1 - a[14] * s0) * q;
	r[15] = (a[8] * s3 - a[9] * s1 + a[10] * s0) * q;
	return 1;
}

/* buildMatrix + calcDinv (src/linearSolver.c:136-252).  prim: primitive
 * state (perturbed and restored in place), r_xk: residual at the state
 * (R_XK), t: evaluation time of the perturbed residuals (the reference
 * passes the step's start time), dt: time step.  Out: D, Dinv [N][16] and
 * O [H][16] (row-major 4x4 blocks: rows = residual variables, columns =
 * perturbed primitive variables; O[h] is the block of the row cell of
 * half-side h and the column cell across it, zero at boundary sides).
 * in_place: restore by subtraction (the reference's rounding) instead of
 * the saved value. */
int oracle_build_matrix(const ccfd_case *cs, double *prim, const double *r_xk, double t, double dt,
			int in_place, double *D, double *Dinv, double *O)
{
	const ccfd_mesh *m = &cs->mesh;
	const long N = m->n_cells, H = m->n_half_sides;
	const double rEps0 = sqrt(2.220446049250313e-16), srEps0 = 1.0 / rEps0;
	orc o;
	double *eps2 = o_venk_eps2(cs);
	o_init(&o, cs, eps2);
	olocal L;
	if (o_local_init(&L, m) != CCFD_OK) {
		free(eps2);
		return CCFD_ERR_NOMEM;
	}
	memset(D, 0, sizeof(double) * 16 * N);
	memset(O, 0, sizeof(double) * 16 * H);
	long tgt[64];
	double ut[4 * 64];
	for (long i = 0; i < N; ++i) {
		int nt = 0;
		tgt[nt++] = i;
		for (long h = m->hs_offset[i]; h < m->hs_offset[i + 1] && nt < 64; ++h)
			if (m->hs_nb[h] >= 0)
				tgt[nt++] = m->hs_nb[h];
		for (int iv = 0; iv < NV; ++iv) {
			const double save = prim[4 * i + iv];
			prim[4 * i + iv] += rEps0;
			o_local_ut(&o, cs, &L, prim, t, tgt, nt, ut);
			if (in_place)
				prim[4 * i + iv] -= rEps0;
			else
				prim[4 * i + iv] = save;
			for (int jv = 0; jv < NV; ++jv)
				D[16 * i + 4 * jv + iv] += (ut[jv] - r_xk[4 * i + jv]) * srEps0;
			/* column of cell i in the rows of its face neighbours j: the
			 * block (j, i), kept at every half-side of j that faces i */
			int k = 1;
			for (long h = m->hs_offset[i]; h < m->hs_offset[i + 1]; ++h) {
				long j = m->hs_nb[h];
				if (j < 0)
					continue;
				const double *uj = &ut[4 * k++];
				for (long h2 = m->hs_offset[j]; h2 < m->hs_offset[j + 1]; ++h2) {
					if (m->hs_nb[h2] != i)
						continue;
					for (int jv = 0; jv < NV; ++jv)
						O[16 * h2 + 4 * jv + iv] += (uj[jv] - r_xk[4 * j + jv]) * srEps0;
				}
			}
		}
	}
	/* I - dt dR/dU (src/linearSolver.c:226-233) and the inverses */
	int st = CCFD_OK;
	for (long k = 0; k < 16 * H; ++k)
		O[k] *= -dt;
	for (long i = 0; i < N; ++i) {
		for (int k = 0; k < 16; ++k)
			D[16 * i + k] *= -dt;
		for (int a = 0; a < NV; ++a)
			D[16 * i + 5 * a] += 1.0;
		if (!o_inv4(&D[16 * i], &Dinv[16 * i]))
			st = CCFD_ERR_SINGULAR;
	}
	o_local_free(&L);
	free(eps2);
	if (o.vacuum && st == CCFD_OK)
		st = CCFD_ERR_VACUUM;
	return st;
}

/* LUSGS (src/linearSolver.c:261-333): forward and backward sweeps in cell
 * order; x = M^-1 b, xs ([N][4]) is the intermediate vector. */
void oracle_lusgs(const ccfd_case *cs, const double *Dinv, const double *O, const double *b,
		  double *x, double *xs)
{
	const ccfd_mesh *m = &cs->mesh;
	const long N = m->n_cells;
	memset(x, 0, sizeof(double) * 4 * N);
	memset(xs, 0, sizeof(double) * 4 * N);
	for (long i = 0; i < N; ++i) {
		double s[4] = {0.0, 0.0, 0.0, 0.0};
		for (long h = m->hs_offset[i]; h < m->hs_offset[i + 1]; ++h) {
			long j = m->hs_nb[h];
			if (j < 0 || j >= i)
				continue;
			for (int a = 0; a < NV; ++a)
				for (int c = 0; c < NV; ++c)
					s[a] += O[16 * h + 4 * a + c] * xs[4 * j + c];
		}
		for (int a = 0; a < NV; ++a) {
			double r = 0.0;
			for (int c = 0; c < NV; ++c)
				r += Dinv[16 * i + 4 * a + c] * (b[4 * i + c] - s[c]);
			xs[4 * i + a] = r;
		}
	}
	for (long i = N - 1; i >= 0; --i) {
		double s[4] = {0.0, 0.0, 0.0, 0.0};
		for (long h = m->hs_offset[i]; h < m->hs_offset[i + 1]; ++h) {
			long j = m->hs_nb[h];
			if (j <= i)
				continue;
			for (int a = 0; a < NV; ++a)
				for (int c = 0; c < NV; ++c)
					s[a] += O[16 * h + 4 * a + c] * x[4 * j + c];
		}
		for (int a = 0; a < NV; ++a) {
			double r = 0.0;
			for (int c = 0; c < NV; ++c)
				r += Dinv[16 * i + 4 * a + c] * s[c];
			x[4 * i + a] = xs[4 * i + a] - r;
		}
	}
}

/* vectorDotProduct (src/linearSolver.c:115-128), element order */
static double o_dot(long N, const double *a, const double *b)
{
	double r = 0.0;
	for (long i = 0; i < N; ++i)
		for (int v = 0; v < NV; ++v)
			r += a[4 * i + v] * b[4 * i + v];
	return r;
}

/* implicit-step work arrays */
typedef struct {
	long N;
	int K;
	double *Q, *FX0, *FXK, *XK, *RXK, *dX, *R0, *W, *V, *Z, *U, *ut, *xs;
	double *D, *Dinv, *O, *prim_m;
	double *wall_p;
	long newton, gmres;
} oimp;

static void o_imp_free(oimp *I)
{
	free(I->Q); free(I->FX0); free(I->FXK); free(I->XK); free(I->RXK); free(I->dX);
	free(I->R0); free(I->W); free(I->V); free(I->Z); free(I->U); free(I->ut); free(I->xs);
	free(I->D); free(I->Dinv); free(I->O); free(I->prim_m); free(I->wall_p);
}

static int o_imp_init(oimp *I, const ccfd_case *cs)
{
	const ccfd_mesh *m = &cs->mesh;
	const long N = m->n_cells;
	memset(I, 0, sizeof(*I));
	I->N = N;
	I->K = cs->params.n_kdim > 0 ? cs->params.n_kdim : 1;
	size_t v = sizeof(double) * 4 * N;
	I->Q = malloc(v); I->FX0 = malloc(v); I->FXK = malloc(v); I->XK = malloc(v);
	I->RXK = malloc(v); I->dX = malloc(v); I->R0 = malloc(v); I->W = malloc(v);
	I->U = malloc(v); I->ut = malloc(v); I->xs = malloc(v); I->prim_m = malloc(v);
	I->V = malloc(v * (I->K + 1));
	I->Z = malloc(v * I->K);
	I->wall_p = calloc(m->n_bc + 1, sizeof(double));
	if (cs->params.precond) {
		I->D = malloc(sizeof(double) * 16 * N);
		I->Dinv = malloc(sizeof(double) * 16 * N);
		I->O = malloc(sizeof(double) * 16 * (m->n_half_sides + 1));
	}
	if (!I->Q || !I->FX0 || !I->FXK || !I->XK || !I->RXK || !I->dX || !I->R0 || !I->W || !I->U ||
	    !I->ut || !I->xs || !I->prim_m || !I->V || !I->Z || !I->wall_p ||
	    (cs->params.precond && (!I->D || !I->Dinv || !I->O))) {
		o_imp_free(I);
		return CCFD_ERR_NOMEM;
	}
	return CCFD_OK;
}

/* matrixVector (src/linearSolver.c:343-373): res = v - alpha dt
 * (R(XK + eps v) - R_XK) / eps, eps = rEps0 / |v|; prim is left at the
 * perturbed state (as the reference leaves pVar) */
static int o_matvec(orc *o, const ccfd_case *cs, oimp *I, double *prim, double time, double dt,
		    double alpha, const double *v, double *res)
{
	const long N = I->N;
	const double rEps0 = sqrt(2.220446049250313e-16);
	double epsFD = o_dot(N, v, v);
	epsFD = rEps0 / sqrt(epsFD);
	for (long i = 0; i < N; ++i) {
		for (int k = 0; k < NV; ++k)
			I->U[4 * i + k] = I->XK[4 * i + k] + epsFD * v[4 * i + k];
		o_cons_prim(o, &I->U[4 * i], &prim[4 * i]);
	}
	int st = oracle_residual(cs, prim, time, I->ut, NULL, NULL, I->wall_p);
	for (long i = 0; i < N; ++i)
		for (int k = 0; k < NV; ++k)
			res[4 * i + k] = v[4 * i + k] - alpha * dt * (I->ut[4 * i + k] - I->RXK[4 * i + k]) / epsFD;
	return st;
}

/* GMRES_M (src/linearSolver.c:385-510); t0: step start (buildMatrix time) */
static int o_gmres(orc *o, const ccfd_case *cs, oimp *I, double *prim, double time, double t0,
		   double dt, double alpha, const double *B, double normB, double *abortCrit,
		   int in_place)
{
	const long N = I->N;
	const int K = I->K;
	const size_t VS = 4 * N;
	*abortCrit = cs->params.eps_gmres * normB;
	double normR0 = normB;
	for (long i = 0; i < 4 * N; ++i) {
		I->R0[i] = -B[i];
		I->dX[i] = 0.0;
		I->V[i] = I->R0[i] / normR0;
	}
	double gam[K + 1], H[K + 1][K + 1], C[K], S[K];
	gam[0] = normR0;
	int st = CCFD_OK;
	if (cs->params.precond) {
		/* buildMatrix runs at the state pVar holds (consPrim of XK) */
		if ((st = oracle_build_matrix(cs, prim, I->RXK, t0, dt, in_place, I->D, I->Dinv, I->O)))
			return st;
	}
	for (int m = 0; m < K; ++m) {
		I->gmres++;
		double *Vm = I->V + VS * m, *Zm = I->Z + VS * m;
		if (cs->params.precond)
			oracle_lusgs(cs, I->Dinv, I->O, Vm, Zm, I->xs);
		else
			memcpy(Zm, Vm, sizeof(double) * VS);
		if ((st = o_matvec(o, cs, I, prim, time, dt, alpha, Zm, I->W)))
			return st;
		for (int nn = 0; nn <= m; ++nn) {
			H[nn][m] = o_dot(N, I->V + VS * nn, I->W);
			for (long i = 0; i < 4 * N; ++i)
				I->W[i] -= H[nn][m] * I->V[VS * nn + i];
		}
		double res = o_dot(N, I->W, I->W);
		H[m + 1][m] = sqrt(res);
		for (int nn = 0; nn <= m - 1; ++nn) {
			double tmp = C[nn] * H[nn][m] + S[nn] * H[nn + 1][m];
			H[nn + 1][m] = -S[nn] * H[nn][m] + C[nn] * H[nn + 1][m];
			H[nn][m] = tmp;
		}
		double bet = sqrt(H[m][m] * H[m][m] + H[m + 1][m] * H[m + 1][m]);
		S[m] = H[m + 1][m] / bet;
		C[m] = H[m][m] / bet;
		H[m][m] = bet;
		gam[m + 1] = -S[m] * gam[m];
		gam[m] = C[m] * gam[m];
		if ((fabs(gam[m + 1]) <= *abortCrit) || (m == K - 1)) {
			double alp[K];
			for (int nn = m; nn >= 0; --nn) {
				alp[nn] = gam[nn];
				for (int q = nn + 1; q <= m; ++q)
					alp[nn] -= H[nn][q] * alp[q];
				alp[nn] /= H[nn][nn];
			}
			for (int nn = 0; nn <= m; ++nn)
				for (long i = 0; i < 4 * N; ++i)
					I->dX[i] += alp[nn] * I->Z[VS * nn + i];
			return CCFD_OK;
		}
		for (long i = 0; i < 4 * N; ++i)
			I->V[VS * (m + 1) + i] = I->W[i] / H[m + 1][m];
	}
	return CCFD_ERR_GMRES;
}

/* implicitTimeStep (src/timeDiscretization.c:412-552) from the step start
 * time t: cons / prim are the state (updated), ut the residual of the last
 * evaluation; res (4) = globalResidual of it */
static int o_implicit_step(orc *o, const ccfd_case *cs, oimp *I, double *cons, double *prim,
			   double t, double dt, int in_place, double res[4])
{
	const ccfd_params *p = &cs->params;
	const ccfd_mesh *m = &cs->mesh;
	const long N = I->N;
	const double alpha = 1.0, beta = 1.0;
	const double eps2newton = p->eps_newton * p->eps_newton, eps2newton_sq = sqrt(eps2newton);
	int st;
	for (long i = 0; i < N; ++i) {
		memcpy(&I->Q[4 * i], &cons[4 * i], sizeof(double) * 4);
		o_cons_prim(o, &cons[4 * i], &prim[4 * i]);
	}
	double time = t + beta * dt;
	if ((st = oracle_residual(cs, prim, time, I->ut, NULL, NULL, I->wall_p)))
		return st;
	for (long i = 0; i < 4 * N; ++i) {
		I->FX0[i] = cons[i] - I->Q[i] - alpha * dt * I->ut[i];
		I->XK[i] = cons[i];
		I->RXK[i] = I->ut[i];
		I->FXK[i] = I->FX0[i];
	}
	double norm2_F_X0 = o_dot(N, I->FX0, I->FX0);
	double eps2newtonLoc = fmax(1e-8 * 1e-8 * N * eps2newton / norm2_F_X0, eps2newton);
	double norm2_F_XK = norm2_F_X0;
	int nInner = 0;
	double abortCrit = 0.0, norm2_old = norm2_F_XK, gamA, gamB;
	while ((norm2_F_XK > eps2newtonLoc * norm2_F_X0) && (nInner < p->n_newton_iter)) {
		if (nInner == 0) {
			abortCrit = 0.999;
			norm2_old = norm2_F_XK;
		} else {
			gamA = p->gamma_ew * norm2_F_XK / norm2_old;
			if (p->gamma_ew * abortCrit * abortCrit < 0.1)
				gamB = fmin(0.999, gamA);
			else
				gamB = fmin(0.999, fmax(gamA, p->gamma_ew * abortCrit * abortCrit));
			abortCrit = fmin(0.999, fmax(gamB, 0.5 * eps2newton_sq / sqrt(norm2_F_XK)));
			norm2_old = norm2_F_XK;
		}
		nInner++;
		if ((st = o_gmres(o, cs, I, prim, time, t, dt, alpha, I->FXK, sqrt(norm2_F_XK), &abortCrit,
				  in_place)))
			return st;
		for (long i = 0; i < N; ++i) {
			for (int k = 0; k < NV; ++k) {
				I->XK[4 * i + k] += I->dX[4 * i + k];
				cons[4 * i + k] = I->XK[4 * i + k];
			}
			o_cons_prim(o, &cons[4 * i], &prim[4 * i]);
		}
		if ((st = oracle_residual(cs, prim, time, I->ut, NULL, NULL, I->wall_p)))
			return st;
		for (long i = 0; i < 4 * N; ++i) {
			I->RXK[i] = I->ut[i];
			I->FXK[i] = cons[i] - I->Q[i] - alpha * dt * I->ut[i];
		}
		norm2_F_XK = o_dot(N, I->FXK, I->FXK);
	}
	I->newton += nInner;
	if (nInner == p->n_newton_iter)
		return CCFD_ERR_NEWTON;
	double acc[4] = {0, 0, 0, 0};
	for (long c = 0; c < N; ++c)
		for (int v = 0; v < NV; ++v)
			acc[v] += m->cell_geo[4 * c] * I->ut[4 * c + v] * I->ut[4 * c + v];
	for (int v = 0; v < NV; ++v)
		res[v] = sqrt(acc[v] * m->total_area_q);
	return CCFD_OK;
}

/* lift and drag of calcCoef (src/analyze.c:292-387) from the interior face
 * pressures at the wall faces (BC code wall_id), summed in BCside order */
static void o_clcd(const ccfd_case *cs, const double *wall_p, double *cl_out, double *cd_out)
{
	const ccfd_mesh *m = &cs->mesh;
	const ccfd_params *p = &cs->params;
	const double pi = acos(-1.0);
	double v = cs->exact.ref_state[0][1] / cos(cs->exact.alpha * pi / 180.0);
	double qInfQ = 1.0 / (cs->exact.ref_state[0][0] * 0.5 * v * v);
	double qInfLq = qInfQ / p->ref_length;
	double cl = 0.0, cd = 0.0;
	for (long b = 0; b < m->n_bc; ++b) {
		const ccfd_bc *bc = &cs->bc_table[m->bc_index[b]];
		if (bc->type * 100 + bc->id != p->wall_id)
			continue;
		long f = m->bc_face[b];
		cl += m->face_n[2 * f + 1] * wall_p[b] * m->face_len[f];
		cd += m->face_n[2 * f] * wall_p[b] * m->face_len[f];
	}
	cl *= qInfLq;
	cd *= qInfLq;
	double a = cs->exact.alpha * pi / 180.0;
	*cl_out = cl * cos(a) - cd * sin(a);
	*cd_out = cd * cos(a) + cl * sin(a);
}

/* Implicit time loop of timeDisc: per step calcTimeStep, implicitTimeStep,
 * the wing coefficients, the reference's absolute stop test and the
 * relative one (params.rel_abort_residual).  ser_cfl_max > 0 turns on
 * switched evolution relaxation of the CFL number (Mulder and van Leer,
 * 1985): before step n >= 2, CFL = min(ser_cfl_max, CFL_0 * r_1 / r_{n-1}),
 * r the abort variable's global residual after a step, and the viscous
 * number follows, DFL = DFL_0 * CFL / CFL_0.  in_place: the
 * reference's in-place restore in buildMatrix.  prim is updated in place;
 * info[0..11] = t, steps, res[0..3], finished, converged, Newton and GMRES
 * iterations, cl, cd; hist (optional, nsteps x 8): t, dt, res[0..3], cl, cd
 * per step. */
int oracle_run_implicit(const ccfd_case *cs, double *prim, long nsteps, double ser_cfl_max,
			int in_place, double *info, double *hist)
{
	ccfd_case c2 = *cs;
	ccfd_params *p = &c2.params;
	const ccfd_mesh *m = &cs->mesh;
	const long N = m->n_cells;
	const double cfl0 = p->cfl, dfl0 = p->dfl;
	orc o;
	o_init(&o, cs, NULL);
	oimp I;
	if (o_imp_init(&I, cs) != CCFD_OK)
		return CCFD_ERR_NOMEM;
	double *cons = malloc(sizeof(double) * 4 * N);
	if (!cons) {
		o_imp_free(&I);
		return CCFD_ERR_NOMEM;
	}
	for (long c = 0; c < N; ++c)
		o_prim_cons(&o, &prim[4 * c], &cons[4 * c]);
	double t = 0.0;
	double print_time = (floor(0.0 / p->io_time_interval) + 1) * p->io_time_interval;
	long io_iter = p->io_iter_interval > 0 ? p->io_iter_interval : 1;
	long print_iter = io_iter;
	double res[4] = {0, 0, 0, 0}, r_first = 0.0, r_prev = 0.0, cl = 0.0, cd = 0.0;
	int finished = 0, converged = 0, st = CCFD_OK;
	long iter, done = 0;
	for (iter = 1; iter <= p->max_iter; ++iter) {
		if (nsteps > 0 && iter > nsteps)
			break;
		if (ser_cfl_max > 0.0 && iter >= 2 && r_prev > 0.0) {
			p->cfl = fmin(ser_cfl_max, cfl0 * r_first / r_prev);
			p->dfl = dfl0 * p->cfl / cfl0;
		}
		double dt;
		if ((st = oracle_time_step(&c2, prim, t, print_time, &dt)) != CCFD_OK)
			break;
		o.vacuum = 0;
		if ((st = o_implicit_step(&o, &c2, &I, cons, prim, t, dt, in_place, res)) != CCFD_OK)
			break;
		double cl_old = cl, cd_old = cd, rcl = 0.0, rcd = 0.0;
		if (p->calc_wing) {
			o_clcd(cs, I.wall_p, &cl, &cd);
			rcl = fabs(cl_old - cl) / dt;
			rcd = fabs(cd_old - cd) / dt;
		}
		t += dt;
		if (hist) {
			double *h = &hist[8 * done];
			h[0] = t; h[1] = dt;
			for (int v = 0; v < 4; ++v)
				h[2 + v] = res[v];
			h[6] = cl; h[7] = cd;
		}
		done++;
		double ra = res[p->abort_variable];
		if (iter == 1)
			r_first = ra;
		r_prev = ra;
		if (p->t_end - t <= 1e-15) {
			finished = 1;
			break;
		}
		if (p->stationary) {
			int conv = 0;
			if (fabs(ra) <= p->abort_residual) {
				if (p->cl_abort_residual > 0.0)
					conv = fabs(rcl) <= p->cl_abort_residual;
				else if (p->cd_abort_residual > 0.0)
					conv = fabs(rcd) <= p->cd_abort_residual;
				else
					conv = 1;
			}
			if (p->rel_abort_residual > 0.0 && ra <= p->rel_abort_residual * r_first)
				conv = 1;
			if (conv) {
				converged = 1;
				break;
			}
		}
		if ((print_time - t <= 1e-15) || (iter == print_iter)) {
			if (print_time - t <= 1e-15)
				print_time += p->io_time_interval;
			if (iter == print_iter)
				print_iter += io_iter;
		}
	}
	info[0] = t;
	info[1] = (double)done;
	for (int v = 0; v < 4; ++v)
		info[2 + v] = res[v];
	info[6] = finished;
	info[7] = converged;
	info[8] = (double)I.newton;
	info[9] = (double)I.gmres;
	info[10] = cl;
	info[11] = cd;
	free(cons);
	o_imp_free(&I);
	return st;
}
