/*
 * CPU oracle for the collapse-table generator: homogeneous-ellipsoid collapse with the
 * reference's fixed-step "funny RK4" (EllipsoidalCollapse.jl:192-198 rk4_homel!,
 * :200-290 get_derivs!, :492-590 evolve_ellipse_full with solver = :rk4) and the table
 * sweep of CollapseTable.jl:22-76.
 *
 * TEST INFRASTRUCTURE ONLY: the checker of the CUDA generator (ht_collapse.cu) and the
 * timed CPU baseline.  Nothing in the product library links or calls it.
 *
 * FP64 throughout, every operation in the reference's order (Julia evaluates a + b + c
 * as (a + b) + c and x^3 for a literal 3 as x * x * x); built with -ffp-contract=off so
 * that no product is fused into an addition, as in Julia.
 */
#include <math.h>
#include <string.h>

#include "ht_oracle.h"

#define OR_RD_MAXIT 200

/* _hunt (Cosmology.jl:117-132): 1-based jlo of x in the ascending table. */
static int or_hunt(const double* xx, int n, double x) {
    const int ascnd = xx[n - 1] > xx[0];
    int jlo = 0, jhi = n + 1;
    while (jhi - jlo > 1) {
        const int jm = (jhi + jlo) / 2;
        if ((x > xx[jm - 1]) == ascnd) jlo = jm;
        else jhi = jm;
    }
    return jlo;
}

/* Lagrange weights of _lagrint_one / _lagrint_2col (Cosmology.jl:80-115) over
 * xa[0 .. nl-1]. */
static void or_lagr_weights(const double* xa, int nl, double x, double* w) {
    if (nl == 4) {
        w[0] = (x - xa[1]) / (xa[0] - xa[1]) * (x - xa[2]) / (xa[0] - xa[2]) * (x - xa[3]) / (xa[0] - xa[3]);
        w[1] = (x - xa[0]) / (xa[1] - xa[0]) * (x - xa[2]) / (xa[1] - xa[2]) * (x - xa[3]) / (xa[1] - xa[3]);
        w[2] = (x - xa[0]) / (xa[2] - xa[0]) * (x - xa[1]) / (xa[2] - xa[1]) * (x - xa[3]) / (xa[2] - xa[3]);
        w[3] = (x - xa[0]) / (xa[3] - xa[0]) * (x - xa[1]) / (xa[3] - xa[1]) * (x - xa[2]) / (xa[3] - xa[2]);
    } else {
        w[0] = (x - xa[1]) / (xa[0] - xa[1]);
        w[1] = 1.0 - w[0];
    }
}

/* The interpolation window of Dlinear_ab / Dfnofa (Cosmology.jl:289-300): 0-based first
 * entry and point count.  A 4-point window that would start before the first entry starts
 * at it (the reference would index out of bounds there, at a ~ 1/1000, which the collapse
 * never reaches: it starts at a = 1 / (zinit_fac Frho)). */
static void or_window(const or_growth* g, double ai, int* k0, int* nl) {
    const int kk = or_hunt(g->atab, g->ntab, ai);
    if (kk < 2 || kk >= g->ntab) {
        *nl = 2;
        *k0 = (kk - 1 > 1 ? kk - 1 : 1) - 1;
    } else {
        *nl = 4;
        *k0 = (kk - 2 > 1 ? kk - 2 : 1) - 1;
    }
}

/* Dlinear_ab (Cosmology.jl:287-307): (D(a), dlnD/dlna). */
void or_dlinear_ab(const or_growth* g, double ai, double* dlin, double* hd_ha) {
    if (ai > g->amintab && ai < g->amaxtab) {
        int k0, nl;
        double w[4];
        or_window(g, ai, &k0, &nl);
        or_lagr_weights(g->atab + k0, nl, ai, w);
        double p1, p2;
        if (nl == 4) {
            p1 = w[0] * g->D_atab[k0] + w[1] * g->D_atab[k0 + 1] + w[2] * g->D_atab[k0 + 2] +
                 w[3] * g->D_atab[k0 + 3];
            p2 = w[0] * g->dlnD[k0] + w[1] * g->dlnD[k0 + 1] + w[2] * g->dlnD[k0 + 2] +
                 w[3] * g->dlnD[k0 + 3];
        } else {
            p1 = w[0] * g->D_atab[k0] + w[1] * g->D_atab[k0 + 1];
            p2 = w[0] * g->dlnD[k0] + w[1] * g->dlnD[k0 + 1];
        }
        *dlin = p1 * ai;
        *hd_ha = p2;
    } else if (ai >= g->amaxtab) {
        *dlin = g->D_a0 * ai;
        *hd_ha = g->HD_Ha0;
    } else {
        *dlin = g->D_ainfty * ai;
        *hd_ha = g->HD_Hainfty;
    }
}

/* Dfnofa (Cosmology.jl:310-330): D(a) normalised to D(1) = 1. */
double or_dfnofa(const or_growth* g, double ai) {
    if (ai > g->amintab && ai < g->amaxtab) {
        int k0, nl;
        double w[4];
        or_window(g, ai, &k0, &nl);
        or_lagr_weights(g->atab + k0, nl, ai, w);
        const double p = nl == 4 ? w[0] * g->D_atab[k0] + w[1] * g->D_atab[k0 + 1] +
                                       w[2] * g->D_atab[k0 + 2] + w[3] * g->D_atab[k0 + 3]
                                 : w[0] * g->D_atab[k0] + w[1] * g->D_atab[k0 + 1];
        return ai * p;
    }
    if (ai >= g->amaxtab) return ai * g->D_a0;
    return ai * g->D_ainfty;
}

/* Carlson's RD(x, y, z) (EllipsoidalCollapse.jl:62-106, the Numerical Recipes form with
 * ERRTOL 0.05).  The duplication loop stops after OR_RD_MAXIT rounds at the latest (finite
 * positive arguments converge in a few dozen; the reference loops for ever on NaN). */
double or_elliptic_rd(double x, double y, double z) {
    const double ERRTOL = 0.05, C1 = 3.0 / 14.0, C2 = 1.0 / 6.0, C3 = 9.0 / 22.0,
                 C4 = 3.0 / 26.0, C5 = 0.25 * C3, C6 = 1.5 * C4;
    double xt = x, yt = y, zt = z, sum = 0.0, fac = 1.0, delx = 0.0, dely = 0.0, delz = 0.0,
           ave = 0.0;
    for (int it = 0; it < OR_RD_MAXIT; ++it) {
        const double sqrtx = sqrt(xt), sqrty = sqrt(yt), sqrtz = sqrt(zt);
        const double alamb = sqrtx * (sqrty + sqrtz) + sqrty * sqrtz;
        sum += fac / (sqrtz * (zt + alamb));
        fac *= 0.25;
        xt = 0.25 * (xt + alamb);
        yt = 0.25 * (yt + alamb);
        zt = 0.25 * (zt + alamb);
        ave = 0.2 * (xt + yt + 3.0 * zt);
        delx = (ave - xt) / ave;
        dely = (ave - yt) / ave;
        delz = (ave - zt) / ave;
        if (fmax(fmax(fabs(delx), fabs(dely)), fabs(delz)) <= ERRTOL) break;
    }
    const double ea = delx * dely, eb = delz * delz, ec = ea - eb, ed = ea - 6.0 * eb,
                 ee = ed + ec + ec;
    return 3.0 * sum + fac * (1.0 + ed * (-C1 + C5 * ed - C6 * delz * ee) +
                              delz * (C2 * ee + delz * (-C3 * ec + delz * C4 * ea))) /
                           (ave * sqrt(ave));
}

/* Natural log of a finite x > 0 from a series: x = m 2^e with m in [1/sqrt 2, sqrt 2),
 * log x = e ln 2 + 2 atanh(s), s = (m - 1)/(m + 1) (|s| < 0.172), the atanh series summed to
 * s^23 (truncation below 1e-20).  Plain arithmetic in a fixed order, so that the CUDA
 * generator, which carries the same function, rounds alike (the library logs of the host
 * and the device may differ in the last bit, which the adaptive path would amplify into a
 * different step sequence).  Also returns log2 x through *log2x when non-NULL. */
static double or_log_series(double x, double* log2x) {
    int e;
    double m = frexp(x, &e);
    if (m < 0.7071067811865476) { m *= 2.0; e -= 1; }
    const double s = (m - 1.0) / (m + 1.0), s2 = s * s;
    double t = 1.0 / 23.0;
    for (int k = 21; k >= 1; k -= 2) t = 1.0 / (double)k + s2 * t;
    const double lnm = 2.0 * s * t;
    if (log2x) *log2x = (double)e + lnm * 1.4426950408889634;
    return (double)e * 0.6931471805599453 + lnm;
}

/* Shape integrals b_i (EllipsoidalCollapse.jl:108-146, iwant_rd = 1); sum(b) = 1. */
void or_get_b_2(double a1, double a2, double a3, double b[3]) {
    const double third = 1.0 / 3.0;
    const double r_2 = a2 / a1, r_3 = a3 / a1;
    if (r_3 >= r_2) {
        if (r_3 >= 0.999) {
            b[0] = b[1] = b[2] = third;
            return;
        }
        double b3;
        if (r_3 <= 0.001) {
            const double ecc2 = 1.0 - r_3 * r_3, one_ecc2 = r_3 * r_3,
                         one_ecc = 0.5 * (r_3 * r_3), ecc = sqrt(ecc2);
            b3 = 0.5 * (one_ecc2 / ecc2 *
                        (1.0 / one_ecc2 - or_log_series((1.0 + ecc) / one_ecc, NULL) * 0.5 / ecc));
        } else {
            const double ecc2 = 1.0 - r_3 * r_3, ecc = sqrt(ecc2);
            b3 = 0.5 * ((1.0 - ecc2) / ecc2 *
                        (1.0 / (1.0 - ecc2) -
                         or_log_series((1.0 + ecc) / (1.0 - ecc), NULL) * 0.5 / ecc));
        }
        b[0] = 1.0 - 2.0 * b3;
        b[1] = b3;
        b[2] = b3;
        return;
    }
    const double r_22 = r_2 * r_2, r_32 = r_3 * r_3, qrat = third * r_2 * r_3;
    const double b3 = qrat * or_elliptic_rd(r_22, 1.0, r_32);
    const double b2 = qrat * or_elliptic_rd(r_32, 1.0, r_22);
    b[0] = 1.0 - (b2 + b3);
    b[1] = b2;
    b[2] = b3;
}

/* Mutable state of the RK4 path (EllipsoidalCollapse.jl:168-191 DerivState). */
typedef struct {
    int lvirv[3];
    double a_3eq, a_2eq, a_1eq, a_3eq2, a_3eq1, Ha_b_nr_val;
    double aLam[3], Frho_3;
} or_derivstate;

/* a H / (H0 sqrt(Om)) (EllipsoidalCollapse.jl:57-59). */
static double or_ha_b_nr(double a_b, double Rvac, double Rcurv) {
    return sqrt((1.0 + Rvac * (a_b * a_b * a_b) + Rcurv * a_b) / a_b);
}

/* get_derivs! (EllipsoidalCollapse.jl:200-290): dy at (t, y); freezes the virialised
 * axes in y and advances the virialisation flags, as the Fortran does. */
static void or_get_derivs(const or_ellipsoid* ep, double Rvac, double Rcurv, double t,
                          double* y, double* dy, or_derivstate* ds) {
    for (int i = 0; i < 6; ++i) dy[i] = 0.0;
    const double a_b = t, a_b3 = a_b * a_b * a_b;
    const double Ha = or_ha_b_nr(a_b, Rvac, Rcurv);
    ds->Ha_b_nr_val = Ha;
    const double Ha_inv = 1.0 / Ha;
    if (ds->lvirv[2] == 0 && y[2] <= ep->fcoll[2] * a_b) {
        ds->lvirv[2] = 1;
        ds->a_3eq = ep->fcoll[2] * a_b;
        if (ep->ivir_strat == 1) {
            ds->a_3eq2 = ds->a_3eq * 1.001;
            ds->a_3eq1 = ds->a_3eq * 1.0003;
        }
    }
    if (ep->ivir_strat == 2 && ds->lvirv[1] == 0) ds->a_3eq2 = ep->fcoll[1] * a_b;
    if (ep->ivir_strat == 2 && ds->lvirv[0] == 0) ds->a_3eq1 = ep->fcoll[0] * a_b;
    if (ds->lvirv[2] == 1 && y[1] <= ds->a_3eq2 && ds->lvirv[1] == 0) {
        ds->lvirv[1] = 1;
        ds->a_2eq = ds->a_3eq2;
    }
    if (ds->lvirv[2] == 1 && y[0] <= ds->a_3eq1 && ds->lvirv[0] == 0) {
        ds->lvirv[0] = 1;
        ds->a_1eq = ds->a_3eq1;
    }
    if (ds->lvirv[2] == 1) { y[2] = ds->a_3eq; y[5] = 0.0; dy[2] = 0.0; dy[5] = 0.0; }
    if (ds->lvirv[1] == 1) { y[1] = ds->a_2eq; y[4] = 0.0; dy[1] = 0.0; dy[4] = 0.0; }
    if (ds->lvirv[0] == 1) { y[0] = ds->a_1eq; y[3] = 0.0; dy[0] = 0.0; dy[3] = 0.0; }

    const double a1 = y[0], a2 = y[1], a3 = y[2];
    const double delta1_e = a_b3 / (a1 * a2 * a3);
    double d0, d1_int, d1_ext = 0.0;
    const int fs = ep->iforce_strat;
    if (fs == 0) {
        d0 = -Rvac * Ha_inv;
        d1_int = 1.5 * delta1_e / a_b3 * Ha_inv;
    } else {
        d0 = (0.5 / a_b3 - Rvac) * Ha_inv;
        d1_int = 1.5 * (delta1_e - 1.0) / a_b3 * Ha_inv;
        if (fs == 4 || fs == 5 || fs == 6) {
            double dlin, hd;
            or_dlinear_ab(&ep->growth, a_b, &dlin, &hd);
            d1_ext = 1.5 / a_b3 * Ha_inv * dlin;
        } else if (fs == 3) {
            d1_ext = 1.5 * 2.5 / a_b3 * Ha_inv;
        }
    }
    double b[3] = {0.0, 0.0, 0.0};
    if (fs != 5 && fs != 6) or_get_b_2(a1, a2, a3, b);
    const double third = 1.0 / 3.0;
    /* axes in the reference's order: 3, 2, 1 */
    for (int ax = 2; ax >= 0; --ax) {
        if (ds->lvirv[ax] != 0) continue;
        dy[ax] = y[ax + 3] * Ha_inv;
        double f;
        if (fs == 0) f = -y[ax] * d1_int * b[ax];
        else if (fs == 1) f = -y[ax] * (d1_int * b[ax] + d0);
        else if (fs == 3) f = -y[ax] * (d1_int * b[ax] + d0 + d1_ext * (b[ax] - third));
        else if (fs == 4 || fs == 6)
            f = -y[ax] * (d1_int * b[ax] + d0 + d1_ext * (ds->aLam[ax] - ds->Frho_3));
        else if (fs == 5) f = -y[ax] * d0 - d1_ext * a_b * ds->aLam[ax];
        else f = dy[ax + 3];
        dy[ax + 3] = f;
    }
}

/* rk4_homel! (EllipsoidalCollapse.jl:149-172); dy holds the derivatives at (t, y). */
static void or_rk4(const or_ellipsoid* ep, double Rvac, double Rcurv, const double* y,
                   const double* dy, double t, double h, double* yout, or_derivstate* ds) {
    double yt[6], dyt[6], dym[6];
    const double hh = h * 0.5, h6 = h / 6.0, xh = t + hh;
    for (int i = 0; i < 6; ++i) yt[i] = y[i] + hh * dy[i];
    or_get_derivs(ep, Rvac, Rcurv, xh, yt, dyt, ds);
    for (int i = 0; i < 6; ++i) yt[i] = y[i] + hh * dyt[i];
    or_get_derivs(ep, Rvac, Rcurv, xh, yt, dym, ds);
    for (int i = 0; i < 6; ++i) {
        yt[i] = y[i] + h * dym[i];
        dym[i] = dyt[i] + dym[i];
    }
    or_get_derivs(ep, Rvac, Rcurv, t + h, yt, dyt, ds);
    for (int i = 0; i < 6; ++i) yout[i] = y[i] + h6 * (dy[i] + dyt[i] + 2.0 * dym[i]);
}

/* ---- solver = :diffeq: adaptive Tsit5 (EllipsoidalCollapse.jl:333-485) ---- */

/* x^y for finite x > 0 as 2^(y log2 x): log2 x from or_log_series, 2^v = 2^n exp(f ln 2)
 * with n the nearest integer to v and the Taylor series to f^16.  About 1e-15 relative,
 * ample for a step-size controller, and made of operations that round alike on the host
 * and on the device (the CUDA generator carries the same function), so both take the same
 * steps. */
double or_pow_pos(double x, double y) {
    double l2;
    or_log_series(x, &l2);
    const double v = y * l2;
    const double n = floor(v + 0.5);
    const double f = (v - n) * 0.6931471805599453;
    double p = 1.0;
    for (int k = 16; k >= 1; --k) p = 1.0 + f * p / (double)k;
    return ldexp(p, (int)n);
}

/* VirState (EllipsoidalCollapse.jl:327-333). */
typedef struct {
    int lvirv[3];
    double a_eq[3], zdynv[3];
} or_virstate;

/* _diffeq_rhs! (EllipsoidalCollapse.jl:344-438): du at (t, u).  Like get_derivs! it
 * freezes the virialised axes in u (the caller's vector) and advances the virialisation
 * flags at every evaluation, accepted step or not, recording 1/a at the evaluation that
 * sets each flag.  aLam[3] is Frho / 3.  iforce_strat 2 (no reference branch) keeps the
 * velocities constant. */
static void or_diffeq_rhs(const or_ellipsoid* ep, double Rvac, double Rcurv,
                          const double* aLam, double t, double* u, double* du,
                          or_virstate* v) {
    const double a_b = t, a_b3 = a_b * a_b * a_b;
    const double Ha = or_ha_b_nr(a_b, Rvac, Rcurv);
    const double Ha_inv = 1.0 / Ha;
    if (v->lvirv[2] == 0 && u[2] <= ep->fcoll[2] * a_b) {
        v->lvirv[2] = 1;
        v->a_eq[2] = ep->fcoll[2] * a_b;
        v->zdynv[2] = 1.0 / a_b;
    }
    double a_3eq2 = 0.0, a_3eq1 = 0.0;
    if (ep->ivir_strat == 2 && v->lvirv[1] == 0) a_3eq2 = ep->fcoll[1] * a_b;
    else if (ep->ivir_strat == 1 && v->lvirv[2] == 1) a_3eq2 = v->a_eq[2] * 1.001;
    if (ep->ivir_strat == 2 && v->lvirv[0] == 0) a_3eq1 = ep->fcoll[0] * a_b;
    else if (ep->ivir_strat == 1 && v->lvirv[2] == 1) a_3eq1 = v->a_eq[2] * 1.0003;
    if (v->lvirv[2] == 1 && v->lvirv[1] == 0 && u[1] <= a_3eq2) {
        v->lvirv[1] = 1;
        v->a_eq[1] = a_3eq2;
        v->zdynv[1] = 1.0 / a_b;
    }
    if (v->lvirv[2] == 1 && v->lvirv[0] == 0 && u[0] <= a_3eq1) {
        v->lvirv[0] = 1;
        v->a_eq[0] = a_3eq1;
        v->zdynv[0] = 1.0 / a_b;
    }
    for (int ax = 2; ax >= 0; --ax)
        if (v->lvirv[ax] == 1) { u[ax] = v->a_eq[ax]; u[ax + 3] = 0.0; }

    const double a1 = u[0], a2 = u[1], a3 = u[2];
    const double delta1_e = a_b3 / (a1 * a2 * a3);
    const double Frho_3 = aLam[3];
    double d0, d1_int, d1_ext = 0.0;
    const int fs = ep->iforce_strat;
    if (fs == 0) {
        d0 = -Rvac * Ha_inv;
        d1_int = 1.5 * delta1_e / a_b3 * Ha_inv;
    } else {
        d0 = (0.5 / a_b3 - Rvac) * Ha_inv;
        d1_int = 1.5 * (delta1_e - 1.0) / a_b3 * Ha_inv;
        if (fs == 4 || fs == 5 || fs == 6) {
            double dlin, hd;
            or_dlinear_ab(&ep->growth, a_b, &dlin, &hd);
            d1_ext = 1.5 / a_b3 * Ha_inv * dlin;
        } else if (fs == 3) {
            d1_ext = 1.5 * 2.5 / a_b3 * Ha_inv;
        }
    }
    double b[3] = {0.0, 0.0, 0.0};
    if (fs != 5 && fs != 6) or_get_b_2(a1, a2, a3, b);
    const double third = 1.0 / 3.0;
    for (int ax = 0; ax < 3; ++ax) {
        if (v->lvirv[ax] == 1) { du[ax] = 0.0; du[ax + 3] = 0.0; continue; }
        du[ax] = u[ax + 3] * Ha_inv;
        double f = 0.0;
        if (fs == 0) f = -u[ax] * d1_int * b[ax];
        else if (fs == 1) f = -u[ax] * (d1_int * b[ax] + d0);
        else if (fs == 3) f = -u[ax] * (d1_int * b[ax] + d0 + d1_ext * (b[ax] - third));
        else if (fs == 4 || fs == 6)
            f = -u[ax] * (d1_int * b[ax] + d0 + d1_ext * (aLam[ax] - Frho_3));
        else if (fs == 5) f = -u[ax] * d0 - d1_ext * a_b * aLam[ax];
        du[ax + 3] = f;
    }
}

/* Tsitouras' 5(4) pair (Ch. Tsitouras, Comput. Math. Appl. 62 (2011) 770-775), first same
 * as last, in the tabulation of OrdinaryDiffEq's Tsit5: nodes, stage weights and the
 * weights of the embedded error estimate. */
static const double TS_C[7] = {0.0, 0.161, 0.327, 0.9, 0.9800255409045097, 1.0, 1.0};
static const double TS_A[7][6] = {
    {0, 0, 0, 0, 0, 0},
    {0.161, 0, 0, 0, 0, 0},
    {-0.008480655492356989, 0.335480655492357, 0, 0, 0, 0},
    {2.897153057105493, -6.359448489975075, 4.3622954328695815, 0, 0, 0},
    {5.325864828439257, -11.748883564062828, 7.4955393428898365, -0.09249506636175525, 0, 0},
    {5.86145544294642, -12.92096931784711, 8.159367898576159, -0.071584973281401,
     -0.028269050394068383, 0},
    {0.09646076681806523, 0.01, 0.4798896504144996, 1.379008574103742, -3.290069515436081,
     2.324710524099774}};
static const double TS_E[7] = {-0.00178001105222577714, -0.0008164344596567469,
                               0.007880878010261995, -0.1447110071732629,
                               0.5823571654525552, -0.45808210592918697,
                               0.015151515151515152};

/* Root mean square of six values, summed in order. */
static double or_rms6(const double* v) {
    double s = 0.0;
    for (int i = 0; i < 6; ++i) s += v[i] * v[i];
    return sqrt(s / 6.0);
}

/* _evolve_diffeq (EllipsoidalCollapse.jl:440-485): the same initial state as the RK4 path,
 * integrated over a in [1/(zinit_fac Frho), 2] by Tsit5 with abstol 1e-8, reltol 1e-6,
 * at most 100,000 iterations, stopping after the first accepted step at which axis 1 has
 * virialised (the DiscreteCallback).  The integrator restates the published method as
 * OrdinaryDiffEq runs it: the starting step of Hairer, Norsett & Wanner (Solving ODEs I,
 * II.4), the error norm RMS(err_i / (abstol + max(|u_i|, |unew_i|) reltol)), and the PI
 * step-size controller with beta1 = 7/50, beta2 = 2/25, safety 9/10, step ratio within
 * [1/10, 5] after an accepted step and the new step dt / min(5, EEst^beta1 / 0.9) after a
 * rejected one (qold starts at 1e-4).  idynax 1-3 (axis virialisation: the reference's
 * VirState keeps no turnaround events).  Returns the iterations taken. */
static int or_evolve_tsit5(const or_ellipsoid* ep, double Frho, double e_v, double p_v,
                           int idynax, double out[3]) {
    const double Omnr = ep->Om, Omvac = ep->OL, Omcurv = 1.0 - ep->Om - ep->OL;
    const double Rvac = Omvac / Omnr, Rcurv = Omcurv / Omnr;
    const double abstol = 1e-8, reltol = 1e-6, tend = 2.0;
    const int maxiters = 100000;
    double aLam[4];
    aLam[2] = Frho / 3.0 * (1.0 + 3.0 * e_v + p_v);
    aLam[1] = Frho / 3.0 * (1.0 - 2.0 * p_v);
    aLam[0] = Frho / 3.0 * (1.0 - 3.0 * e_v + p_v);
    aLam[3] = Frho / 3.0;
    or_virstate vs;
    memset(&vs, 0, sizeof vs);
    for (int i = 0; i < 3; ++i) vs.zdynv[i] = -1.0;
    const double zinit = ep->zinit_fac * Frho;
    const double a_b = 1.0 / zinit;
    double dlin, HD_Ha;
    or_dlinear_ab(&ep->growth, a_b, &dlin, &HD_Ha);
    const double Ha = or_ha_b_nr(a_b, Rvac, Rcurv);
    double u[6];
    for (int ax = 2; ax >= 0; --ax) u[ax] = a_b * (1.0 - dlin * aLam[ax]);
    for (int ax = 2; ax >= 0; --ax) u[ax + 3] = Ha * (1.0 - (1.0 + HD_Ha) * dlin * aLam[ax]);
    double t = a_b;

    /* starting step */
    double k[7][6], tmp[6], sc[6];
    or_diffeq_rhs(ep, Rvac, Rcurv, aLam, t, u, k[0], &vs);
    for (int i = 0; i < 6; ++i) sc[i] = abstol + fabs(u[i]) * reltol;
    for (int i = 0; i < 6; ++i) tmp[i] = u[i] / sc[i];
    const double d0 = or_rms6(tmp);
    for (int i = 0; i < 6; ++i) tmp[i] = k[0][i] / sc[i];
    const double d1 = or_rms6(tmp);
    double dt0 = (d0 < 1e-5 || d1 < 1e-5) ? 1e-6 : 0.01 * (d0 / d1);
    if (dt0 > tend - t) dt0 = tend - t;
    double u1[6];
    for (int i = 0; i < 6; ++i) u1[i] = u[i] + dt0 * k[0][i];
    or_diffeq_rhs(ep, Rvac, Rcurv, aLam, t + dt0, u1, k[1], &vs);
    for (int i = 0; i < 6; ++i) tmp[i] = (k[1][i] - k[0][i]) / sc[i];
    const double d2 = or_rms6(tmp) / dt0;
    const double dmax = d1 > d2 ? d1 : d2;
    double dt1 = dmax <= 1e-15 ? (1e-6 > dt0 * 1e-3 ? 1e-6 : dt0 * 1e-3)
                               : or_pow_pos(0.01 / dmax, 0.2);
    double dt = 100.0 * dt0 < dt1 ? 100.0 * dt0 : dt1;
    if (dt > tend - t) dt = tend - t;
    or_diffeq_rhs(ep, Rvac, Rcurv, aLam, t, u, k[0], &vs);   /* the first FSAL stage */

    double qold = 1e-4;
    int iter = 0;
    while (iter < maxiters && t < tend) {
        ++iter;
        if (dt > tend - t) dt = tend - t;
        if (!(dt > 1e-14 * t)) break;   /* step size underflow: give up */
        for (int st = 1; st < 7; ++st) {
            for (int i = 0; i < 6; ++i) {
                double acc = 0.0;
                for (int j = 0; j < st; ++j) acc += TS_A[st][j] * k[j][i];
                tmp[i] = u[i] + dt * acc;
            }
            or_diffeq_rhs(ep, Rvac, Rcurv, aLam, t + TS_C[st] * dt, tmp, k[st], &vs);
            if (st == 6) memcpy(u1, tmp, sizeof u1);   /* the step's end, after the RHS froze it */
        }
        double r[6];
        for (int i = 0; i < 6; ++i) {
            double acc = 0.0;
            for (int j = 0; j < 7; ++j) acc += TS_E[j] * k[j][i];
            const double au = fabs(u[i]), an = fabs(u1[i]);
            r[i] = (dt * acc) / (abstol + (au > an ? au : an) * reltol);
        }
        const double EEst = or_rms6(r);
        if (EEst <= 1.0) {
            double q;
            if (EEst == 0.0) {
                q = 0.1;
            } else {
                q = or_pow_pos(EEst, 0.14) / or_pow_pos(qold, 0.08) / 0.9;
                q = q < 5.0 ? q : 5.0;
                q = q > 0.1 ? q : 0.1;
            }
            t = t + dt;
            if (tend - t <= 1e-13 * tend) t = tend;
            memcpy(u, u1, sizeof u);
            memcpy(k[0], k[6], sizeof k[0]);
            qold = EEst > 1e-4 ? EEst : 1e-4;
            dt = dt / q;
            if (vs.lvirv[0] == 1) break;   /* the terminating callback */
        } else {
            /* rejected (EEst > 1 or NaN): shrink by EEst^beta1 / 0.9, at most 5x */
            double q11 = EEst == EEst ? or_pow_pos(EEst, 0.14) / 0.9 : 5.0;
            dt = dt / (q11 < 5.0 ? q11 : 5.0);
        }
    }
    const double z = idynax >= 1 && idynax <= 3 ? vs.zdynv[idynax - 1] : -1.0;
    if (z == -1.0) {
        out[0] = out[1] = out[2] = -1.0;
    } else {
        const double D = or_dfnofa(&ep->growth, 1.0 / z);
        out[0] = z;
        out[1] = D;
        out[2] = Frho * D;
    }
    return iter;
}

/* evolve_ellipse_full (EllipsoidalCollapse.jl:492-590): out[0] = 1/a at event idynax (1-3
 * axis virialisation, 4-6 axis turnaround with the RK4), out[1] = D there, out[2] = Frho D;
 * all -1 if the event does not happen before a = 2 (or nstepmax RK4 steps).  solver 1 runs
 * the :diffeq path (or_evolve_tsit5).  Returns the number of steps (iterations) taken. */
int or_evolve_ellipse(const or_ellipsoid* ep, double Frho, double e_v, double p_v,
                      int idynax, double out[3]) {
    if (ep->solver == 1) return or_evolve_tsit5(ep, Frho, e_v, p_v, idynax, out);
    const double Omnr = ep->Om, Omvac = ep->OL, Omcurv = 1.0 - ep->Om - ep->OL;
    const double Rvac = Omvac / Omnr, Rcurv = Omcurv / Omnr;
    or_derivstate ds;
    memset(&ds, 0, sizeof ds);
    ds.aLam[2] = Frho / 3.0 * (1.0 + 3.0 * e_v + p_v);
    ds.aLam[1] = Frho / 3.0 * (1.0 - 2.0 * p_v);
    ds.aLam[0] = Frho / 3.0 * (1.0 - 3.0 * e_v + p_v);
    ds.Frho_3 = Frho / 3.0;
    const double zinit = ep->zinit_fac * Frho;
    const double a_b = 1.0 / zinit;
    double t = a_b, dlin, HD_Ha;
    or_dlinear_ab(&ep->growth, a_b, &dlin, &HD_Ha);
    const double Ha = or_ha_b_nr(a_b, Rvac, Rcurv);
    ds.Ha_b_nr_val = Ha;
    double y[6], dy[6], yout[6];
    for (int ax = 2; ax >= 0; --ax) y[ax] = a_b * (1.0 - dlin * ds.aLam[ax]);
    for (int ax = 2; ax >= 0; --ax) y[ax + 3] = Ha * (1.0 - (1.0 + HD_Ha) * dlin * ds.aLam[ax]);
    double zdynv[7], aturnv[3] = {0.0, 0.0, 0.0};
    int ldynv[7];
    for (int i = 0; i < 7; ++i) { zdynv[i] = -1.0; ldynv[i] = 0; }
    int istep = 0;
    for (;;) {
        ++istep;
        const double a_3 = y[2];
        const double dtstep = ep->tfac * a_3 * sqrt(a_3) * ds.Ha_b_nr_val;
        or_get_derivs(ep, Rvac, Rcurv, t, y, dy, &ds);
        or_rk4(ep, Rvac, Rcurv, y, dy, t, dtstep, yout, &ds);
        memcpy(y, yout, sizeof y);
        t += dtstep;
        for (int ii = 0; ii < 3; ++ii) {
            if (ds.lvirv[ii] != ldynv[ii]) {
                zdynv[ii] = 1.0 / t;
                ldynv[ii] = 1;
            }
        }
        for (int ii = 3; ii < 6; ++ii) {
            if (ldynv[ii] != 1) {
                const int iax = ii - 3;
                if (y[iax] < aturnv[iax]) {
                    zdynv[ii] = 1.0 / t;
                    ldynv[ii] = 1;
                } else {
                    aturnv[iax] = y[iax];
                }
            }
        }
        if (ds.lvirv[0] == 1 || istep >= ep->nstepmax || t >= 2.0) {
            const double z = zdynv[idynax - 1];
            if (z == -1.0) {
                out[0] = out[1] = out[2] = -1.0;
            } else {
                const double D = or_dfnofa(&ep->growth, 1.0 / z);
                out[0] = z;
                out[1] = D;
                out[2] = Frho * D;
            }
            return istep;
        }
    }
}

/* make_table (CollapseTable.jl:29-50) with evolve_ellipse_function (:22-27): table[i, j, k]
 * = Float32(zvir(10^x_i, y_j, z_k y_j)), x_i = X1 + (i - 1) dX and so on, column-major.
 * Entries are independent; OpenMP over them. */
void or_make_table(const or_ellipsoid* ep, int nx, int ny, int nz, double X1, double X2,
                   double Y1, double Y2, double Z1, double Z2, float* table) {
    const double dX = (X2 - X1) / (nx - 1), dY = (Y2 - Y1) / (ny - 1),
                 dZ = (Z2 - Z1) / (nz - 1);
    const long long n = (long long)nx * ny * nz;
#pragma omp parallel for schedule(dynamic, 16)
    for (long long e = 0; e < n; ++e) {
        const int i = (int)(e % nx), j = (int)((e / nx) % ny), k = (int)(e / ((long long)nx * ny));
        const double x = X1 + i * dX, y = Y1 + j * dY, z = Z1 + k * dZ;
        double out[3];
        or_evolve_ellipse(ep, pow(10.0, x), y, z * y, 1, out);
        table[e] = (float)out[0];
    }
}
