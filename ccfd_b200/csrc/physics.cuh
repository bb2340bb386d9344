// Device physics of the residual path: equation of state, ghost states,
// exact functions, the eleven convective fluxes and the viscous flux.
//
// Every expression keeps the operand order and association of the
// reference's C code (file:line cited per function), and the library is
// compiled without contraction of multiply-adds (-fmad=false), so in FP64 the
// device results equal the reference's bit for bit wherever both use
// correctly rounded operations (+ - * / sqrt); pow / tanh / exp / sin / cos
// follow CUDA's implementations.
//
// The flux and reconstruction helpers are templated on the arithmetic type
// (double for the FP64 path, float for the mixed-precision face fluxes).
#pragma once

#include <cuda_runtime.h>
#include <math.h>

namespace ccfd {

constexpr int kMaxBC = 20;

struct DevBC {
    int type;        // enum ccfd_bc_type
    int exact_func;  // BCexactFunc
    double pvar[4];  // rho, vx, vy, p
};

struct DevExact {
    double ref_state[2][4];
    double rp1d_interface;
    double x_min, x_max, y_min, y_max, dx_ref;
};

// Physics constants, passed by value to every kernel (constant bank).
struct Phys {
    double gam, gam1, gam1q, mu, Pr, pi, sqrt3q;
    int nbc;
    int order;      // spatial order 1 / 2
    int eqn;        // 0 Euler, 1 Navier-Stokes
    int source_func;  // calcSource / sourceFunction, 0: no source term
    DevBC bc[kMaxBC];
    DevExact ex;
};

// status bits raised by kernels (host maps them to ccfd_status)
enum DevFlag : unsigned {
    FLAG_DT = 1u,        // non-finite time step
    FLAG_VACUUM = 2u,    // vacuum in the exact Riemann solver
    FLAG_STATE = 4u,     // non-finite residual
    FLAG_SINGULAR = 8u,  // singular LU-SGS block
    FLAG_GMRES = 16u,
    FLAG_NEWTON = 32u,   // Newton not converged (set by the host driver)
};

template <typename T>
struct V4 {
    T v[4];
};

// evalSource, source function 1 (src/source.c:22-60): the source of the
// manufactured sine-wave solution (exact function 3); adds source * w to q.
// The operation order is the reference's; cos / sin are CUDA's and may
// differ from the C library's in the last bit.
__device__ __forceinline__ void add_source(const Phys& P, double x, double y, double time, double w,
                                           double q[4]) {
    const double freq = 1.0, amp = 0.1;
    const double om = P.pi * freq;
    const double a = 2.0 * P.pi;
    const double tmp1 = cos(om * (x + y) - a * time);
    const double tmp2 = sin(2.0 * (om * (x + y) - a * time));
    double s0 = (-a + 2.0 * om) * tmp1;
    double s1 = (-a + om * (P.gam * 3.0 - 1.0)) * tmp1 + amp * om * P.gam1 * tmp2;
    double s3 = ((2.0 + P.gam * 6.0) * om - 4.0 * a) * tmp1 + amp * (2.0 * om * P.gam - a) * tmp2;
    if (P.eqn == 1) {
        const double tmp3 = sin(om * (x + y) - a * time);
        s3 = s3 + 2.0 * P.mu * P.gam * om * om / P.Pr * tmp3;
    }
    s0 *= amp;
    s1 *= amp;
    s3 *= amp;
    q[0] += s0 * w;
    q[1] += s1 * w;
    q[2] += s1 * w;
    q[3] += s3 * w;
}

// calcSource (src/source.c:66-85) for one cell: side quadrature points
// bary + GP in side order (weight area/3 for triangles, area/6 for quads),
// then the quad's fifth point, the midpoint of its nodes 0 and 2
// (src/mesh.c:117-161).  xq = (bary.x, bary.y, gp5.x, gp5.y).
__device__ __forceinline__ double4 cell_source(const Phys& P, const double4* __restrict__ hs_gw, int h0, int h1,
                                               double4 xq, double area, double time) {
    double q[4] = {0.0, 0.0, 0.0, 0.0};
    const bool quad = h1 - h0 == 4;
    const double w = quad ? area / 6.0 : area / 3.0;
    for (int h = h0; h < h1; ++h) {
        double4 gw = hs_gw[h];
        add_source(P, xq.x + gw.x, xq.y + gw.y, time, w, q);
    }
    if (quad) add_source(P, xq.z, xq.w, time, area / 3.0, q);
    return make_double4(q[0], q[1], q[2], q[3]);
}

// primCons, src/equationOfState.c:19-26
__device__ __forceinline__ void prim_cons(double gam1q, const double p[4], double c[4]) {
    c[0] = p[0];
    c[1] = p[1] * p[0];
    c[2] = p[2] * p[0];
    c[3] = gam1q * p[3] + 0.5 * (c[1] * p[1] + c[2] * p[2]);
}

// consPrim with the density / pressure floor, src/equationOfState.c:37-52
__device__ __forceinline__ void cons_prim(double gam1, const double c[4], double p[4]) {
    p[0] = c[0];
    p[1] = c[1] / c[0];
    p[2] = c[2] / c[0];
    p[3] = gam1 * (c[3] - 0.5 * (c[1] * p[1] + c[2] * p[2]));
    if (p[0] < 1e-19) p[0] = 1e-10;
    if (p[3] < 1e-19) p[3] = 1e-10;
}

// consChar, src/equationOfState.c:60-88 (reference state: the unrotated
// interior state, as the reference passes it)
__device__ __forceinline__ void cons_char(const Phys& P, const double c[4], double ch[3],
                                          const double ref[4]) {
    double cs = sqrt(P.gam * ref[3] / ref[0]);
    double u = ref[1];
    double H = P.gam1q * cs * cs + 0.5 * u * u;
    double phi = u * u - 2.0 * H;
    double a1 = 1.0 / (2.0 * cs * phi);
    double a2 = 1.0 / phi;
    double a3 = u * cs;
    double c1d[3] = {c[0], c[1], c[3]};
    double K[3][3] = {{a1 * u * (phi - a3), -a1 * (phi - 2.0 * a3), -a2},
                      {a2 * (u * u + phi), -2.0 * u * a2, 2.0 * a2},
                      {-a1 * u * (a3 + phi), a1 * (phi + 2.0 * a3), -a2}};
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        double s = 0.0;
#pragma unroll
        for (int j = 0; j < 3; ++j) s += K[i][j] * c1d[j];
        ch[i] = s;
    }
}

// charCons, src/equationOfState.c:90-110 (sets rho, m_x, E only)
__device__ __forceinline__ void char_cons(const Phys& P, const double ch[3], double c[4],
                                          const double ref[4]) {
    double u = ref[1];
    double cs = sqrt(P.gam * ref[3] / ref[0]);
    double H = P.gam1q * cs * cs + 0.5 * u * u;
    double K[3][3] = {{1.0, 1.0, 1.0}, {u - cs, u, u + cs}, {H - u * cs, 0.5 * u * u, H + u * cs}};
    double c1d[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) c1d[i] += K[i][j] * ch[j];
    c[0] = c1d[0];
    c[1] = c1d[1];
    c[3] = c1d[2];
}

// ---------------------------------------------------------------- exactRiemann
// Exact Riemann solver (Newton iteration on the star pressure) and sampling,
// src/exactRiemann.c:29-214.  Vacuum raises FLAG_VACUUM instead of exit(1).
__device__ __forceinline__ void riemann_pre(double G0, double G1, double G3, double G4,
                                            double G5, double* f, double* fd, double p,
                                            double rhok, double pk, double ck) {
    if (p < pk) {
        double pRat = p / pk;
        *f = G3 * ck * (pow(pRat, G0) - 1.0);
        *fd = (1.0 / (rhok * ck)) * pow(pRat, -G1);
    } else {
        double ak = G4 / rhok;
        double bk = G5 * pk;
        double qrt = sqrt(ak / (bk + p));
        *f = (p - pk) * qrt;
        *fd = (1.0 - 0.5 * (p - pk) / (bk + p)) * qrt;
    }
}

__device__ inline void exact_riemann(double gam, double rhol, double rhor, double* rho,
                                     double ul, double ur, double* u, double pl, double pr,
                                     double* p, double al, double ar, double s,
                                     unsigned* flags) {
    const double G0 = (gam - 1.0) / (2.0 * gam), G1 = (gam + 1.0) / (2.0 * gam),
                 G2 = 2.0 * gam / (gam - 1.0), G3 = 2.0 / (gam - 1.0), G4 = 2.0 / (gam + 1.0),
                 G5 = (gam - 1.0) / (gam + 1.0), G6 = 0.5 * (gam - 1.0), G7 = 1.0 / gam;
    const double tol = 1e-6;
    double du = ur - ul;
    double duCrit = G3 * (al + ar) - du;
    if (duCrit < 0.0) {
        if (flags) atomicOr(flags, (unsigned)FLAG_VACUUM);
        *rho = rhol;
        *u = ul;
        *p = pl;
        return;
    }
    double qMax = 2.0;
    double pv = 0.5 * (pl + pr) - 0.125 * (ur - ul) * (rhol + rhor) * (al + ar);
    double pMin = fmin(pl, pr);
    double pMax = fmax(pl, pr);
    double qRat = pMax / pMin;
    if ((qRat < qMax) && (pMin < pv) && (pv < pMax)) {
        *p = fmax(tol, pv);
    } else {
        if (pv < pMin) {
            double pnu = al + ar - G6 * (ur - ul);
            double pde = al / pow(pl, G0) + ar / pow(pr, G0);
            *p = pow(pnu / pde, G2);
        } else {
            double gel = sqrt((G4 / rhol) / (G5 * pl + fmax(tol, pv)));
            double ger = sqrt((G4 / rhor) / (G5 * pr + fmax(tol, pv)));
            *p = (gel * pl + ger * pr - (ur - ul)) / (gel + ger);
            *p = fmax(tol, *p);
        }
    }
    double p0 = *p;
    double cha = 2.0 * tol;
    int KK = 0;
    double fr = 0.0, fl = 0.0, frd = 0.0, fld = 0.0;
    while ((cha > tol) && (KK < 1000)) {
        riemann_pre(G0, G1, G3, G4, G5, &fl, &fld, *p, rhol, pl, al);
        riemann_pre(G0, G1, G3, G4, G5, &fr, &frd, *p, rhor, pr, ar);
        *p -= (fl + fr + du) / (fld + frd);
        cha = 2.0 * fabs((*p - p0) / (*p + p0));
        if (*p < 0.0) *p = tol;
        p0 = *p;
        KK++;
    }
    *u = 0.5 * (ul + ur + fr - fl);
    double pm = *p;
    double um = *u;
    if (s < um) {
        if (pm < pl) {
            if (s < ul - al) {
                *rho = rhol; *u = ul; *p = pl;
            } else {
                double cml = al * pow(pm / pl, G0);
                double stl = um - cml;
                if (s > stl) {
                    *rho = rhol * pow(pm / pl, G7); *u = um; *p = pm;
                } else {
                    *u = G4 * (al + G6 * ul + s);
                    double c = G4 * (al + G6 * (ul - s));
                    *rho = rhol * pow(c / al, G3);
                    *p = pl * pow(c / al, G2);
                }
            }
        } else {
            double pml = pm / pl;
            double sl = ul - al * sqrt(G1 * pml + G0);
            if (s < sl) {
                *rho = rhol; *u = ul; *p = pl;
            } else {
                *rho = rhol * (pml + G5) / (pml * G5 + 1.0); *u = um; *p = pm;
            }
        }
    } else {
        if (pm > pr) {
            double pmr = pm / pr;
            double sr = ur + ar * sqrt(G1 * pmr + G0);
            if (s > sr) {
                *rho = rhor; *u = ur; *p = pr;
            } else {
                *rho = rhor * (pmr + G5) / (pmr * G5 + 1.0); *u = um; *p = pm;
            }
        } else {
            double shr = ur + ar;
            if (s > shr) {
                *rho = rhor; *u = ur; *p = pr;
            } else {
                double cmr = ar * pow(pm / pr, G0);
                double str = um + cmr;
                if (s < str) {
                    *rho = rhor * pow(pm / pr, G7); *u = um; *p = pm;
                } else {
                    *u = G4 * (-ar + G6 * ur + s);
                    double c = G4 * (ar - G6 * (ur - s));
                    *rho = rhor * pow(c / ar, G3);
                    *p = pr * pow(c / ar, G2);
                }
            }
        }
    }
}

// ---------------------------------------------------------------- exactFunc
// src/exactFunction.c:35-183, used by EXACTSOL ghost states
__device__ inline void exact_func(const Phys& P, int which, const double x[2], double time,
                                  double pv[4], unsigned* flags) {
    const DevExact& E = P.ex;
    switch (which) {
    case 1: {
        pv[0] = 1.0; pv[1] = 0.0; pv[2] = 0.0; pv[3] = 1.0;
        double xLen = E.x_max - E.x_min, yLen = E.y_max - E.y_min;
        if (x[0] >= 0.3 * xLen + 1.0 / 30.0 * xLen * cos(2.0 * P.pi * 3.0 / yLen * x[1])) pv[0] = 0.25;
        if ((x[0] <= 0.1 * xLen) && (x[0] >= 1.0 / 30.0 * xLen)) { pv[0] = 4.22; pv[3] = 4.9; }
        break;
    }
    case 2: {
        pv[0] = 1.0; pv[1] = 0.0; pv[2] = 0.0;
        double hWidth = fmin((E.x_max - E.x_min), (E.y_max - E.y_min)) / 100.0 * 6.0;
        double xPeak = E.x_min + 0.5 * (E.x_max - E.x_min);
        double yPeak = E.y_min + 0.5 * (E.y_max - E.y_min);
        double expLog = exp(-log(2.0));
        double hWidth2 = hWidth * hWidth;
        double dr2 = (x[0] - xPeak) * (x[0] - xPeak) + (x[1] - yPeak) * (x[1] - yPeak);
        pv[3] = 1.0 + 1.0 * pow(expLog, dr2 / hWidth2);
        break;
    }
    case 3: {
        double omega = P.pi * 1.0, a = 2.0 * P.pi, r[4];
        r[0] = r[1] = r[2] = 2.0 + 0.1 * sin(omega * (x[0] + x[1]) - a * time);
        r[3] = r[0] * r[0];
        cons_prim(P.gam1, r, pv);
        break;
    }
    case 4: {
        // double Mach reflection, src/exactFunction.c:92-116
        double factor = P.pi / (0.2 * E.dx_ref);
        const double cSum[4] = {9.4, 57.157676649772950686, -33.0, 566.0};
        const double cDiff[4] = {6.6, 57.157676649772950686, -33.0, 561.0};
        double th = tanh((x[0] - (1.0 / 6.0 + (20.0 * time + x[1]) * P.sqrt3q)) * factor);
        double cv[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) cv[i] = 0.5 * (cSum[i] - cDiff[i] * th);
        pv[0] = cv[0];
        pv[1] = cv[1] / cv[0];
        pv[2] = cv[2] / cv[0];
        pv[3] = P.gam1 * (cv[3] - 0.5 * (cv[1] * cv[1] + cv[2] * cv[2]) / cv[0]);
        break;
    }
    case 5: {
        double rl = E.ref_state[0][0], ul = E.ref_state[0][1], pl = E.ref_state[0][3];
        double rr = E.ref_state[1][0], ur = E.ref_state[1][1], pr = E.ref_state[1][3];
        double cl = sqrt(P.gam * pl / rl), cr = sqrt(P.gam * pr / rr);
        if (time == 0.0) {
            if (x[0] <= E.rp1d_interface) { pv[0] = rl; pv[1] = ul; pv[3] = pl; }
            else { pv[0] = rr; pv[1] = ur; pv[3] = pr; }
        } else {
            double s = (x[0] - E.rp1d_interface) / time;
            exact_riemann(P.gam, rl, rr, &pv[0], ul, ur, &pv[1], pl, pr, &pv[3], cl, cr, s, flags);
        }
        pv[2] = 0.0;
        break;
    }
    case 6: {
        double omega = P.pi * 1.0, amplitude = 0.00001;
        double cons0[4] = {1.0, 0.1, 0.0, 1.0}, p0[4];
        cons_prim(P.gam1, cons0, p0);
        double c0 = sqrt(P.gam * p0[3] / p0[0]);
        double H0 = (cons0[3] + p0[3]) / p0[0];
        double R[4][4] = {{1.0, 1.0, 0.0, 1.0},
                          {p0[1] - c0, p0[1], 0.0, p0[1] + c0},
                          {p0[2], p0[2], 1.0, p0[2]},
                          {H0 - p0[1] * c0, (p0[1] * p0[1] + p0[2] * p0[2]) / 2.0, p0[2], H0 + p0[1] * c0}};
        double vec[4] = {0.0, 0.0, 0.0, amplitude * sin(omega * (x[0] - (c0 + p0[1]) * time))};
        double r[4];
        for (int i = 0; i < 4; ++i) {
            r[i] = cons0[i];
            for (int j = 0; j < 4; ++j) r[i] += R[i][j] * vec[j];
        }
        cons_prim(P.gam1, r, pv);
        break;
    }
    default:
        pv[0] = pv[1] = pv[2] = pv[3] = 0.0;
    }
}

// ---------------------------------------------------------------- boundary
// Ghost state for one boundary side, src/boundary.c:147-294.  n is the outward
// normal of the interior cell, q the interior state (cell or face), x the
// point at which an exact solution is evaluated.
__device__ inline void boundary_state(const Phys& P, const DevBC& bc, double nx, double ny,
                                      double time, const double q[4], double g[4],
                                      const double x[2], unsigned* flags) {
    switch (bc.type) {
    case 1: {  // SLIPWALL
        double vxl = nx * q[1] + ny * q[2];
        double vyl = -ny * q[1] + nx * q[2];
        double vxg = -vxl, vyg = vyl;
        g[1] = nx * vxg - ny * vyg;
        g[2] = ny * vxg + nx * vyg;
        g[0] = q[0];
        g[3] = q[3];
        break;
    }
    case 2: {  // WALL (Navier-Stokes)
        double vxl = nx * q[1] + ny * q[2];
        double vyl = -ny * q[1] + nx * q[2];
        double vxg = -vxl;
        double vyg = P.mu > 0.0 ? -vyl : vyl;
        g[1] = nx * vxg - ny * vyg;
        g[2] = ny * vxg + nx * vyg;
        g[0] = q[0];
        g[3] = q[3];
        break;
    }
    case 3:  // INFLOW
        g[0] = bc.pvar[0]; g[1] = bc.pvar[1]; g[2] = bc.pvar[2]; g[3] = bc.pvar[3];
        break;
    case 4:  // OUTFLOW
        g[0] = q[0]; g[1] = q[1]; g[2] = q[2]; g[3] = q[3];
        break;
    case 5: {  // CHARACTERISTIC
        double c = sqrt(P.gam * bc.pvar[3] / bc.pvar[0]);
        double v = nx * bc.pvar[1] + ny * bc.pvar[2];
        double il[4], gl[4];
        il[0] = q[0];
        il[1] = nx * q[1] + ny * q[2];
        il[2] = -ny * q[1] + nx * q[2];
        il[3] = q[3];
        gl[0] = bc.pvar[0];
        gl[1] = nx * bc.pvar[1] + ny * bc.pvar[2];
        gl[2] = -ny * bc.pvar[1] + nx * bc.pvar[2];
        gl[3] = bc.pvar[3];
        double ic[4], gc[4];
        prim_cons(P.gam1q, il, ic);
        prim_cons(P.gam1q, gl, gc);
        double ich[3], gch[3];
        cons_char(P, ic, ich, q);
        cons_char(P, gc, gch, q);
        if (v + c > 0.0) gch[2] = ich[2];
        if (v > 0.0) gch[1] = ich[1];
        if (v - c > 0.0) gch[0] = ich[0];
        char_cons(P, gch, gc, q);
        if (v > 0.0) gc[2] = ic[2];
        cons_prim(P.gam1, gc, g);
        double vxl = g[1], vyl = g[2];
        g[1] = nx * vxl - ny * vyl;
        g[2] = ny * vxl + nx * vyl;
        break;
    }
    case 6:  // EXACTSOL
        exact_func(P, bc.exact_func, x, time, g, flags);
        break;
    case 8: {  // PRESSURE_OUT
        double c = sqrt(P.gam * q[3] / q[0]);
        double v = nx * q[1] + ny * q[2];
        double p = (v / c < 1.0) ? bc.pvar[3] : q[3];
        g[0] = q[0] * p / q[3];
        g[1] = q[1];
        g[2] = q[2];
        g[3] = p;
        break;
    }
    default:
        g[0] = q[0]; g[1] = q[1]; g[2] = q[2]; g[3] = q[3];
    }
}

// ---------------------------------------------------------------- fluxes
// All fluxes take the left / right primitive states rotated into the face
// normal frame and return the flux in that frame.

template <typename T>
struct FluxIn {
    T rL, rR, uL, uR, vL, vR, pL, pR;
};

// flux_god, src/fluxCalculation.c:30-53 (FP64 only)
__device__ inline void flux_god(const Phys& P, const FluxIn<double>& s, double f[4],
                                unsigned* flags) {
    double cL = sqrt(P.gam * s.pL / s.rL);
    double cR = sqrt(P.gam * s.pR / s.rR);
    double rho, vx, p;
    exact_riemann(P.gam, s.rL, s.rR, &rho, s.uL, s.uR, &vx, s.pL, s.pR, &p, cL, cR, 0.0, flags);
    double vy = vx > 0.0 ? s.vL : s.vR;
    f[0] = rho * vx;
    f[1] = rho * vx * vx + p;
    f[2] = rho * vx * vy;
    f[3] = vx * (P.gam / P.gam1 * p + 0.5 * rho * (vx * vx + vy * vy));
}

// flux_roe with Harten-type entropy fix, src/fluxCalculation.c:67-147
template <typename T>
__device__ __forceinline__ void flux_roe(T gam, T gam1, T gam1q, const FluxIn<T>& s, T f[4]) {
    T mxL = s.rL * s.uL, mxR = s.rR * s.uR, myL = s.rL * s.vL, myR = s.rR * s.vR;
    T eR = gam1q * s.pR + T(0.5) * s.rR * (s.uR * s.uR + s.vR * s.vR);
    T eL = gam1q * s.pL + T(0.5) * s.rL * (s.uL * s.uL + s.vL * s.vL);
    T HR = (eR + s.pR) / s.rR;
    T HL = (eL + s.pL) / s.rL;
    T rhoSqR = sqrt(s.rR), rhoSqL = sqrt(s.rL);
    T rhoSqQsum = T(1.0) / (rhoSqL + rhoSqR);
    T vxBar = (rhoSqR * s.uR + rhoSqL * s.uL) * rhoSqQsum;
    T vyBar = (rhoSqR * s.vR + rhoSqL * s.vL) * rhoSqQsum;
    T Hbar = (rhoSqR * HR + rhoSqL * HL) * rhoSqQsum;
    T cBar = sqrt(gam1 * (Hbar - T(0.5) * (vxBar * vxBar + vyBar * vyBar)));
    T a[4] = {vxBar - cBar, vxBar, vxBar, vxBar + cBar};
    T r1[4] = {T(1.0), a[0], vyBar, Hbar - vxBar * cBar};
    T r2[4] = {T(1.0), vxBar, vyBar, T(0.5) * (vxBar * vxBar + vyBar * vyBar)};
    T r3[4] = {T(0.0), T(0.0), T(1.0), vyBar};
    T r4[4] = {T(1.0), a[3], vyBar, Hbar + vxBar * cBar};
    T delRho = s.rR - s.rL, delMx = mxR - mxL, delMy = myR - myL, delE = eR - eL;
    T delEq = delE - (delMy - vyBar * delRho) * vyBar;
    T cBarQ = T(1.0) / cBar;
    // wave strengths (the reference names them gam1..gam4)
    T w2 = -gam1 * cBarQ * cBarQ * (delRho * (vxBar * vxBar - Hbar) + delEq - delMx * vxBar);
    T w1 = -T(0.5) * cBarQ * (delMx - delRho * (vxBar + cBar)) - T(0.5) * w2;
    T w4 = delRho - w1 - w2;
    T w3 = delMy - vyBar * delRho;
    T fR[4] = {mxR, mxR * s.uR + s.pR, mxR * s.vR, s.uR * (eR + s.pR)};
    T fL[4] = {mxL, mxL * s.uL + s.pL, mxL * s.vL, s.uL * (eL + s.pL)};
    T cL = sqrt(gam * s.pL / s.rL), cR = sqrt(gam * s.pR / s.rR);
    T al[4] = {s.uL - cL, s.uL, s.uL, s.uL + cL};
    T ar[4] = {s.uR - cR, s.uR, s.uR, s.uR + cR};
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        T da = fmax(fmax(T(0.0), a[i] - al[i]), ar[i] - a[i]);
        if (fabs(a[i]) < da) a[i] = T(0.5) * (a[i] * a[i] / da + da);
        else a[i] = fabs(a[i]);
    }
#pragma unroll
    for (int i = 0; i < 4; ++i)
        f[i] = T(0.5) * (fR[i] + fL[i] - w1 * fabs(a[0]) * r1[i] - w2 * fabs(a[1]) * r2[i] -
                         w3 * fabs(a[2]) * r3[i] - w4 * fabs(a[3]) * r4[i]);
}

// HLL / HLLE shared tail, src/fluxCalculation.c:206-225 and :281-300
template <typename T>
__device__ __forceinline__ void hll_tail(T arp, T alm, const T fL[4], const T fR[4],
                                         const T uL[4], const T uR[4], T f[4]) {
    T arpAlmQ = T(1.0) / (arp - alm);
    if (alm > T(0.0)) {
#pragma unroll
        for (int i = 0; i < 4; ++i) f[i] = fL[i];
    } else if (arp < T(0.0)) {
#pragma unroll
        for (int i = 0; i < 4; ++i) f[i] = fR[i];
    } else {
#pragma unroll
        for (int i = 0; i < 4; ++i)
            f[i] = (arp * fL[i] - alm * fR[i]) * arpAlmQ + (arp * alm) * arpAlmQ * (uR[i] - uL[i]);
    }
}

// flux_hll, src/fluxCalculation.c:161-226
template <typename T>
__device__ __forceinline__ void flux_hll(T gam, T gam1, T gam1q, const FluxIn<T>& s, T f[4]) {
    T rhoLq = T(1.0) / s.rL, rhoRq = T(1.0) / s.rR;
    T rhoSqL = sqrt(s.rL), rhoSqR = sqrt(s.rR);
    T rhoSqQsum = T(1.0) / (rhoSqL + rhoSqR);
    T eR = gam1q * s.pR + T(0.5) * s.rR * (s.uR * s.uR + s.vR * s.vR);
    T eL = gam1q * s.pL + T(0.5) * s.rL * (s.uL * s.uL + s.vL * s.vL);
    T uL[4] = {s.rL, s.rL * s.uL, s.rL * s.vL, eL};
    T uR[4] = {s.rR, s.rR * s.uR, s.rR * s.vR, eR};
    T fL[4] = {uL[1], uL[1] * s.uL + s.pL, uL[1] * s.vL, s.uL * (eL + s.pL)};
    T fR[4] = {uR[1], uR[1] * s.uR + s.pR, uR[1] * s.vR, s.uR * (eR + s.pR)};
    T cL = sqrt(gam * s.pL * rhoLq), cR = sqrt(gam * s.pR * rhoRq);
    T HL = (eL + s.pL) * rhoLq, HR = (eR + s.pR) * rhoRq;
    T uM = (rhoSqR * s.uR + rhoSqL * s.uL) * rhoSqQsum;
    T vM = (rhoSqR * s.vR + rhoSqL * s.vL) * rhoSqQsum;
    T HM = (rhoSqR * HR + rhoSqL * HL) * rhoSqQsum;
    T cM = sqrt(gam1 * (HM - T(0.5) * (uM * uM + vM * vM)));
    T arp = fmax(s.uR + cR, uM + cM);
    T alm = fmin(s.uL - cL, uM - cM);
    hll_tail(arp, alm, fL, fR, uL, uR, f);
}

// flux_hlle (Einfeldt signal speeds), src/fluxCalculation.c:240-301
template <typename T>
__device__ __forceinline__ void flux_hlle(T gam, T gam1, T gam1q, const FluxIn<T>& s, T f[4]) {
    T rhoLq = T(1.0) / s.rL, rhoRq = T(1.0) / s.rR;
    T rhoSqL = sqrt(s.rL), rhoSqR = sqrt(s.rR);
    T rhoSqQsum = T(1.0) / (rhoSqL + rhoSqR);
    T eR = gam1q * s.pR + T(0.5) * s.rR * (s.uR * s.uR + s.vR * s.vR);
    T eL = gam1q * s.pL + T(0.5) * s.rL * (s.uL * s.uL + s.vL * s.vL);
    T uL[4] = {s.rL, s.rL * s.uL, s.rL * s.vL, eL};
    T uR[4] = {s.rR, s.rR * s.uR, s.rR * s.vR, eR};
    T fL[4] = {uL[1], uL[1] * s.uL + s.pL, uL[1] * s.vL, s.uL * (eL + s.pL)};
    T fR[4] = {uR[1], uR[1] * s.uR + s.pR, uR[1] * s.vR, s.uR * (eR + s.pR)};
    T cL = sqrt(gam * s.pL * rhoLq), cR = sqrt(gam * s.pR * rhoRq);
    T uM = (rhoSqR * s.uR + rhoSqL * s.uL) * rhoSqQsum;
    T eta2 = T(0.5) * rhoSqR * rhoSqL / (rhoSqR + rhoSqL) / (rhoSqR + rhoSqL);
    T d = sqrt((rhoSqR * cR * cR + rhoSqL * cL * cL) * rhoSqQsum +
               eta2 * (s.uR - s.uL) * (s.uR - s.uL));
    T arp = fmax(s.uR + cR, uM + d);
    T alm = fmin(s.uL - cL, uM - d);
    hll_tail(arp, alm, fL, fR, uL, uR, f);
}

// flux_hllc, src/fluxCalculation.c:315-396
template <typename T>
__device__ __forceinline__ void flux_hllc(T gam, T gam1, T gam1q, const FluxIn<T>& s, T f[4]) {
    T rhoLq = T(1.0) / s.rL, rhoRq = T(1.0) / s.rR;
    T rhoSqL = sqrt(s.rL), rhoSqR = sqrt(s.rR);
    T rhoSqQsum = T(1.0) / (rhoSqL + rhoSqR);
    T eR = gam1q * s.pR + T(0.5) * s.rR * (s.uR * s.uR + s.vR * s.vR);
    T eL = gam1q * s.pL + T(0.5) * s.rL * (s.uL * s.uL + s.vL * s.vL);
    T uL[4] = {s.rL, s.rL * s.uL, s.rL * s.vL, eL};
    T uR[4] = {s.rR, s.rR * s.uR, s.rR * s.vR, eR};
    T fL[4] = {uL[1], uL[1] * s.uL + s.pL, uL[1] * s.vL, s.uL * (eL + s.pL)};
    T fR[4] = {uR[1], uR[1] * s.uR + s.pR, uR[1] * s.vR, s.uR * (eR + s.pR)};
    T cL = sqrt(gam * s.pL * rhoLq), cR = sqrt(gam * s.pR * rhoRq);
    T HL = (eL + s.pL) * rhoLq, HR = (eR + s.pR) * rhoRq;
    T uM = (rhoSqR * s.uR + rhoSqL * s.uL) * rhoSqQsum;
    T vM = (rhoSqR * s.vR + rhoSqL * s.vL) * rhoSqQsum;
    T HM = (rhoSqR * HR + rhoSqL * HL) * rhoSqQsum;
    T cM = sqrt(gam1 * (HM - T(0.5) * (uM * uM + vM * vM)));
    T arp = fmax(s.uR + cR, uM + cM);
    T alm = fmin(s.uL - cL, uM - cM);
    if (alm > T(0.0)) {
#pragma unroll
        for (int i = 0; i < 4; ++i) f[i] = fL[i];
    } else if (arp < T(0.0)) {
#pragma unroll
        for (int i = 0; i < 4; ++i) f[i] = fR[i];
    } else {
        T as = (s.pR - s.pL + uL[1] * (alm - s.uL) - uR[1] * (arp - s.uR)) /
               (s.rL * (alm - s.uL) - s.rR * (arp - s.uR));
        if ((alm <= T(0.0)) && (as >= T(0.0))) {
            T fac = s.rL * (alm - s.uL) / (alm - as);
            T us[4] = {fac, as * fac, s.vL * fac,
                       fac * (eL / s.rL + (as - s.uL) * (as + s.pL / (s.rL * (alm - s.uL))))};
#pragma unroll
            for (int i = 0; i < 4; ++i) f[i] = fL[i] + alm * (us[i] - uL[i]);
        } else {
            T fac = s.rR * (arp - s.uR) / (arp - as);
            T us[4] = {fac, as * fac, s.vR * fac,
                       fac * (eR / s.rR + (as - s.uR) * (as + s.pR / (s.rR * (arp - s.uR))))};
#pragma unroll
            for (int i = 0; i < 4; ++i) f[i] = fR[i] + arp * (us[i] - uR[i]);
        }
    }
}

// flux_lxf (local Lax-Friedrichs), src/fluxCalculation.c:410-446
template <typename T>
__device__ __forceinline__ void flux_lxf(T gam, T gam1, T gam1q, const FluxIn<T>& s, T f[4]) {
    T cL = sqrt(gam * s.pL / s.rL), cR = sqrt(gam * s.pR / s.rR);
    T a = fmax(fabs(s.uR) + cR, fabs(s.uL) + cL);
    T eL = gam1q * s.pL + T(0.5) * s.rL * (s.uL * s.uL + s.vL * s.vL);
    T eR = gam1q * s.pR + T(0.5) * s.rR * (s.uR * s.uR + s.vR * s.vR);
    T delU[4] = {s.rR - s.rL, s.rR * s.uR - s.rL * s.uL, s.rR * s.vR - s.rL * s.vL, eR - eL};
    T fL[4] = {s.rL * s.uL, s.rL * s.uL * s.uL + s.pL, s.rL * s.uL * s.vL, s.uL * (eL + s.pL)};
    T fR[4] = {s.rR * s.uR, s.rR * s.uR * s.uR + s.pR, s.rR * s.uR * s.vR, s.uR * (eR + s.pR)};
#pragma unroll
    for (int i = 0; i < 4; ++i) f[i] = T(0.5) * (fR[i] + fL[i]) - T(0.5) * a * delU[i];
}

// flux_stw (Steger-Warming), src/fluxCalculation.c:460-509
template <typename T>
__device__ __forceinline__ void flux_stw(T gam, T gam1, T gam1q, const FluxIn<T>& s, T f[4]) {
    T cL = sqrt(gam * s.pL / s.rL), cR = sqrt(gam * s.pR / s.rR);
    T gam2q = T(0.5) / gam;
    T aL[4] = {s.uL - cL, s.uL, s.uL, s.uL + cL};
    T aR[4] = {s.uR - cR, s.uR, s.uR, s.uR + cR};
    T ap[4] = {fmax(aL[0], T(0.0)), fmax(aL[1], T(0.0)), fmax(aL[2], T(0.0)), fmax(aL[3], T(0.0))};
    T am[4] = {fmin(aR[0], T(0.0)), fmin(aR[1], T(0.0)), fmin(aR[2], T(0.0)), fmin(aR[3], T(0.0))};
    T fp[4], fm[4];
    fp[0] = s.rL * gam2q * (T(2.0) * gam1 * ap[1] + ap[0] + ap[3]);
    fp[1] = fp[0] * s.uL + (ap[3] - ap[0]) * s.rL * cL * gam2q;
    fp[2] = fp[0] * s.vL;
    fp[3] = fp[0] * T(0.5) * (s.uL * s.uL + s.vL * s.vL) + (ap[3] - ap[0]) * s.rL * cL * s.uL * gam2q +
            (ap[3] + ap[0]) * s.rL * cL * cL * gam2q * gam1q;
    fm[0] = s.rR * gam2q * (T(2.0) * gam1 * am[1] + am[0] + am[3]);
    fm[1] = fm[0] * s.uR + (am[3] - am[0]) * s.rR * cR * gam2q;
    fm[2] = fm[0] * s.vR;
    fm[3] = fm[0] * T(0.5) * (s.uR * s.uR + s.vR * s.vR) + (am[3] - am[0]) * s.rR * cR * s.uR * gam2q +
            (am[3] + am[0]) * s.rR * cR * cR * gam2q * gam1q;
#pragma unroll
    for (int i = 0; i < 4; ++i) f[i] = fp[i] + fm[i];
}

// flux_cen (central), src/fluxCalculation.c:524-551
template <typename T>
__device__ __forceinline__ void flux_cen(T gam, T gam1, T gam1q, const FluxIn<T>& s, T f[4]) {
    T eL = gam1q * s.pL + T(0.5) * s.rL * (s.uL * s.uL + s.vL * s.vL);
    T eR = gam1q * s.pR + T(0.5) * s.rR * (s.uR * s.uR + s.vR * s.vR);
    T fL[4], fR[4];
    fL[0] = s.rL * s.uL; fL[1] = fL[0] * s.uL + s.pL; fL[2] = fL[0] * s.vL; fL[3] = s.uL * (eL + s.pL);
    fR[0] = s.rR * s.uR; fR[1] = fR[0] * s.uR + s.pR; fR[2] = fR[0] * s.vR; fR[3] = s.uR * (eR + s.pR);
#pragma unroll
    for (int i = 0; i < 4; ++i) f[i] = T(0.5) * (fL[i] + fR[i]);
}

// flux_ausmd, src/fluxCalculation.c:565-611
template <typename T>
__device__ __forceinline__ void flux_ausmd(T gam, T gam1, T gam1q, const FluxIn<T>& s, T f[4]) {
    T eL = gam1q * s.pL + T(0.5) * s.rL * (s.uL * s.uL + s.vL * s.vL);
    T eR = gam1q * s.pR + T(0.5) * s.rR * (s.uR * s.uR + s.vR * s.vR);
    T HL = (eL + s.pL) / s.rL, HR = (eR + s.pR) / s.rR;
    T cm = fmax(sqrt(gam * s.pL / s.rL), sqrt(gam * s.pR / s.rR));
    T alphaL = T(2.0) * s.pL / s.rL / (s.pL / s.rL + s.pR / s.rR);
    T alphaR = T(2.0) * s.pR / s.rR / (s.pL / s.rL + s.pR / s.rR);
    T uPlus, pPlus, uMinus, pMinus;
    if (fabs(s.uL) < cm) {
        uPlus = T(0.25) * alphaL * (s.uL + cm) * (s.uL + cm) / cm + T(0.5) * (T(1.0) - alphaL) * (s.uL + fabs(s.uL));
        pPlus = T(0.25) * s.pL * (s.uL + cm) * (s.uL + cm) / (cm * cm) * (T(2.0) - s.uL / cm);
    } else {
        uPlus = T(0.5) * (s.uL + fabs(s.uL));
        pPlus = T(0.5) * s.pL * (s.uL + fabs(s.uL)) / s.uL;
    }
    if (fabs(s.uR) < cm) {
        uMinus = -T(0.25) * alphaR * (s.uR - cm) * (s.uR - cm) / cm + T(0.5) * (T(1.0) - alphaR) * (s.uR - fabs(s.uR));
        pMinus = T(0.25) * s.pR * (s.uR - cm) * (s.uR - cm) / (cm * cm) * (T(2.0) + s.uR / cm);
    } else {
        uMinus = T(0.5) * (s.uR - fabs(s.uR));
        pMinus = T(0.5) * s.pR * (s.uR - fabs(s.uR)) / s.uR;
    }
    T rhoU = uPlus * s.rL + uMinus * s.rR;
    f[0] = rhoU;
    f[1] = T(0.5) * (rhoU * (s.uR + s.uL) - fabs(rhoU) * (s.uR - s.uL)) + (pPlus + pMinus);
    f[2] = T(0.5) * (rhoU * (s.vR + s.vL) - fabs(rhoU) * (s.vR - s.vL));
    f[3] = T(0.5) * (rhoU * (HR + HL) - fabs(rhoU) * (HR - HL));
}

// flux_ausmdv, src/fluxCalculation.c:627-713 (the reference marks it buggy at
// :615-616; restated as written, including the vxL in the uMinus branch)
template <typename T>
__device__ __forceinline__ void flux_ausmdv(T gam, T gam1, T gam1q, const FluxIn<T>& s, T f[4]) {
    T eL = gam1q * s.pL + T(0.5) * s.rL * (s.uL * s.uL + s.vL * s.vL);
    T eR = gam1q * s.pR + T(0.5) * s.rR * (s.uR * s.uR + s.vR * s.vR);
    T HL = (eL + s.pL) / s.rL, HR = (eR + s.pR) / s.rR;
    T cL = sqrt(gam * s.pL / s.rL), cR = sqrt(gam * s.pR / s.rR);
    T cm = fmax(cL, cR);
    T alphaL = T(2.0) * s.pL / s.rL / (s.pL / s.rL + s.pR / s.rR);
    T alphaR = T(2.0) * s.pR / s.rR / (s.pL / s.rL + s.pR / s.rR);
    T uPlus, pPlus, uMinus, pMinus;
    if (fabs(s.uL) < cm) {
        pPlus = T(0.25) * s.pL * (s.uL + cm) * (s.uL + cm) / (cm * cm) * (T(2.0) - s.uL / cm);
        if (s.uL > T(0.0)) uPlus = s.uL + alphaL * (s.uL - cm) * (s.uL - cm);
        else uPlus = alphaL * (s.uL + cm) * (s.uL + cm);
    } else {
        if (s.uL > T(0.0)) { uPlus = s.uL; pPlus = s.pL; }
        else { uPlus = T(0.0); pPlus = T(0.0); }
    }
    if (fabs(s.uR) < cm) {
        pMinus = T(0.25) * s.pR * (s.uR - cm) * (s.uR - cm) / (cm * cm) * (T(2.0) + s.uR / cm);
        if (s.uR > T(0.0)) uMinus = -alphaR * (s.uL - cm) * (s.uL - cm);
        else uMinus = s.uR - alphaR * (s.uR + cm) * (s.uR + cm);
    } else {
        if (s.uR > T(0.0)) { uMinus = T(0.0); pMinus = T(0.0); }
        else { uMinus = s.uR; pMinus = s.pR; }
    }
    T rhoU = uPlus * s.rL + uMinus * s.rR;
    T sw = fmin(T(1.0), T(10.0) * fabs(s.pR - s.pL) / fmin(s.pR, s.pL));
    T rhoUsq = T(0.5) * (T(1.0) + sw) * (s.rL * s.uL * uPlus + s.rR * s.uR * uMinus);
    rhoUsq += T(0.25) * (T(1.0) - sw) * (rhoU * (s.uR + s.uL) - fabs(rhoU) * (s.uR - s.uL));
    f[0] = rhoU;
    f[1] = rhoUsq + (pPlus + pMinus);
    f[2] = T(0.5) * (rhoU * (s.vR + s.vL) - fabs(rhoU) * (s.vR - s.vL));
    f[3] = T(0.5) * (rhoU * (HR + HL) - fabs(rhoU) * (HR - HL));
    bool tmpa = (s.uL - cL < T(0.0)) && (s.uR - cR > T(0.0));
    bool tmpb = (s.uL + cL < T(0.0)) && (s.uR + cR > T(0.0));
    T tL[4] = {T(1.0), s.uL, s.vL, HL};
    T tR[4] = {T(1.0), s.uR, s.vR, HR};
    if (tmpa && !tmpb) {
#pragma unroll
        for (int i = 0; i < 4; ++i)
            f[i] -= T(0.125) * ((s.uR - cR) - (s.uL - cL)) * (s.rR * tR[i] - s.rL * tL[i]);
    }
    if (!tmpa && tmpb) {
#pragma unroll
        for (int i = 0; i < 4; ++i)
            f[i] -= T(0.125) * ((s.uR + cR) - (s.uL + cL)) * (s.rR * tR[i] - s.rL * tL[i]);
    }
}

// flux_vanleer, src/fluxCalculation.c:727-789
template <typename T>
__device__ __forceinline__ void flux_vanleer(T gam, T gam1, T gam1q, const FluxIn<T>& s, T f[4]) {
    T cL = sqrt(gam * s.pL / s.rL), cR = sqrt(gam * s.pR / s.rR);
    T eL = gam1q * s.pL + T(0.5) * s.rL * (s.uL * s.uL + s.vL * s.vL);
    T eR = gam1q * s.pR + T(0.5) * s.rR * (s.uR * s.uR + s.vR * s.vR);
    T HL = (eL + s.pL) / s.rL, HR = (eR + s.pR) / s.rR;
    T fp[4], fm[4];
    T ML = s.uL / cL;
    if (ML > T(1.0)) {
        fp[0] = s.rL * s.uL; fp[1] = fp[0] * s.uL + s.pL; fp[2] = fp[0] * s.vL; fp[3] = fp[0] * HL;
    } else if ((ML < T(1.0)) && (ML > -T(1.0))) {
        T cx = gam1 * s.uL + T(2.0) * cL;
        fp[0] = T(0.25) * s.rL * cL * (ML + T(1.0)) * (ML + T(1.0));
        fp[1] = fp[0] * cx / gam;
        fp[2] = fp[0] * s.vL;
        fp[3] = T(0.5) * (fp[1] * cx * gam / (gam * gam - T(1.0)) + fp[2] * s.vL);
    } else {
        fp[0] = fp[1] = fp[2] = fp[3] = T(0.0);
    }
    T MR = s.uR / cR;
    if (MR < -T(1.0)) {
        fm[0] = s.rR * s.uR; fm[1] = fm[0] * s.uR + s.pR; fm[2] = fm[0] * s.vR; fm[3] = fm[0] * HR;
    } else if ((MR < T(1.0)) && (MR > -T(1.0))) {
        T cx = gam1 * s.uR - T(2.0) * cR;
        fm[0] = -T(0.25) * s.rR * cR * (T(1.0) - MR) * (T(1.0) - MR);
        fm[1] = fm[0] * cx / gam;
        fm[2] = fm[0] * s.vR;
        fm[3] = T(0.5) * (fm[1] * cx * gam / (gam * gam - T(1.0)) + fm[2] * s.vR);
    } else {
        fm[0] = fm[1] = fm[2] = fm[3] = T(0.0);
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) f[i] = fp[i] + fm[i];
}

// convectiveFlux dispatch, src/fluxCalculation.c:803-844 (FLUX is a template
// constant, so each kernel instantiation carries exactly one flux)
template <int FLUX, typename T>
__device__ __forceinline__ void convective_flux(const Phys& P, const FluxIn<T>& s, T f[4],
                                                unsigned* flags) {
    const T gam = T(P.gam), gam1 = T(P.gam1), gam1q = T(P.gam1q);
    if constexpr (FLUX == 1) {
        FluxIn<double> sd{double(s.rL), double(s.rR), double(s.uL), double(s.uR),
                          double(s.vL), double(s.vR), double(s.pL), double(s.pR)};
        double fd[4];
        flux_god(P, sd, fd, flags);
        for (int i = 0; i < 4; ++i) f[i] = T(fd[i]);
    } else if constexpr (FLUX == 2) {
        flux_roe(gam, gam1, gam1q, s, f);
    } else if constexpr (FLUX == 3) {
        flux_hll(gam, gam1, gam1q, s, f);
    } else if constexpr (FLUX == 4) {
        flux_hlle(gam, gam1, gam1q, s, f);
    } else if constexpr (FLUX == 5) {
        flux_hllc(gam, gam1, gam1q, s, f);
    } else if constexpr (FLUX == 6) {
        flux_lxf(gam, gam1, gam1q, s, f);
    } else if constexpr (FLUX == 7) {
        flux_stw(gam, gam1, gam1q, s, f);
    } else if constexpr (FLUX == 8) {
        flux_cen(gam, gam1, gam1q, s, f);
    } else if constexpr (FLUX == 9) {
        flux_ausmd(gam, gam1, gam1q, s, f);
    } else if constexpr (FLUX == 10) {
        flux_ausmdv(gam, gam1, gam1q, s, f);
    } else {
        flux_vanleer(gam, gam1, gam1q, s, f);
    }
}

// diffusionFlux, src/fluxCalculation.c:855-873 (state: mean primitive state,
// gx / gy: face gradients of the primitive variables); f[0] = g[0] = 0
template <typename T>
__device__ __forceinline__ void diffusion_flux(const Phys& P, const T st[4], const T gx[4],
                                               const T gy[4], T f[4], T g[4]) {
    const T mu = T(P.mu), c43 = T(4.0 / 3.0), c23 = T(2.0 / 3.0);
    const T gam = T(P.gam), gam1 = T(P.gam1), Pr = T(P.Pr);
    f[0] = T(0.0);
    f[1] = (c43 * gx[1] - c23 * gy[2]) * mu;
    f[2] = (gy[1] + gx[2]) * mu;
    f[3] = (c43 * st[1] * gx[1] - c23 * st[1] * gy[2] + (gx[2] + gy[1]) * st[2] +
            gam / (gam1 * Pr * st[0] * st[0]) * (st[0] * gx[3] - st[3] * gx[0])) * mu;
    g[0] = T(0.0);
    g[1] = (gy[1] + gx[2]) * mu;
    g[2] = (c43 * gy[2] - c23 * gx[1]) * mu;
    g[3] = (c43 * st[2] * gy[2] - c23 * st[2] * gx[1] + (gy[1] + gx[2]) * st[1] +
            gam / (gam1 * Pr * st[0] * st[0]) * (st[0] * gy[3] - st[3] * gy[0])) * mu;
}

}  // namespace ccfd
