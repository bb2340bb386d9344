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

/* Residual R(U) of primitive state prim at time t.  grad (N x 8) and fflux
 * (F x 4) are optional outputs (limited gradients, face fluxes). */
int oracle_residual(const ccfd_case *cs, const double *prim, double t, double *u_t,
		    double *grad, double *fflux, double *wall_p)
{
	const ccfd_mesh *m = &cs->mesh;
	const long N = m->n_cells, F = m->n_faces, B = m->n_bc;
	orc o;
	double *eps2 = NULL;
	if (cs->params.spatial_order == 2 && cs->params.limiter == CCFD_LIM_VENKATAKRISHNAN) {
		eps2 = malloc(sizeof(double) * N);
		for (long e = 0; e < N; ++e) {
			double a = m->cell_geo[4 * e];
			eps2[e] = (cs->params.venk_k * sqrt(a)) * (cs->params.venk_k * sqrt(a)) *
				  (cs->params.venk_k * sqrt(a));
		}
	}
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
		for (long c = 0; c < N; ++c) {
			const double *q = &prim[4 * c];
			double *ux = &g[8 * c], *uy = &g[8 * c + 4];
			for (long h = m->hs_offset[c]; h < m->hs_offset[c + 1]; ++h) {
				long nb = m->hs_nb[h];
				const double *qn = nb >= 0 ? &prim[4 * nb] : &gb[4 * (-1 - nb)];
				for (int v = 0; v < NV; ++v) {
					double d = qn[v] - q[v];
					ux[v] += m->hs_w[2 * h] * d;
					uy[v] += m->hs_w[2 * h + 1] * d;
				}
			}
		}
		for (long c = 0; c < N; ++c) {
			const double *q = &prim[4 * c];
			double *ux = &g[8 * c], *uy = &g[8 * c + 4];
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
					if (o.limiter == CCFD_LIM_BARTH_JESPERSEN) {
						/* src/reconstruction.c:25-96 */
						if (d > 0.0)
							ph = fmin(1.0, mx / d);
						else if (d < 0.0)
							ph = fmin(1.0, mn / d);
					} else {
						/* src/reconstruction.c:103-192 */
						double e2 = eps2[c], d2 = d * d;
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
	}
	/* setBCatSides + fluxCalculation, src/boundary.c:300-314,
	 * src/fluxCalculation.c:882-998 */
	for (long f = 0; f < F; ++f) {
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
			o_boundary(&o, &cs->bc_table[m->bc_index[b]], n, t, L, R, &m->bc_x[2 * b]);
			if (wall_p)
				wall_p[b] = L[3];
			memcpy(q1, &gb[4 * b], sizeof(q1));
			g1x = g1y = zero4;
		}
		fin s = {L[0], R[0], n[0] * L[1] + n[1] * L[2], n[0] * R[1] + n[1] * R[2],
			 -n[1] * L[1] + n[0] * L[2], -n[1] * R[1] + n[0] * R[2], L[3], R[3]};
		double fc[4], *F4 = &ff[4 * f];
		o_flux(&o, &s, fc);
		F4[0] = fc[0];
		F4[1] = n[0] * fc[1] - n[1] * fc[2];
		F4[2] = n[1] * fc[1] + n[0] * fc[2];
		F4[3] = fc[3];
		if (o.eqn == CCFD_NAVIER_STOKES) {
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
			double mu = o.mu, k = o.gam / (o.gam1 * o.Pr * st[0] * st[0]);
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
	/* per-cell sum in side-list order, src/finiteVolume.c:96-120 */
	for (long c = 0; c < N; ++c) {
		double s[4] = {0.0, 0.0, 0.0, 0.0};
		for (long h = m->hs_offset[c]; h < m->hs_offset[c + 1]; ++h) {
			const double *F4 = &ff[4 * m->hs_face[h]];
			for (int v = 0; v < NV; ++v)
				s[v] += m->hs_sign[h] > 0 ? F4[v] : -F4[v];
		}
		double src[4] = {0.0, 0.0, 0.0, 0.0};
		if (cs->params.source_func)
			o_cell_source(&o, m, c, t, src);
		for (int v = 0; v < NV; ++v)
			u_t[4 * c + v] = (src[v] - s[v]) * m->cell_geo[4 * c + 1];
	}
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
