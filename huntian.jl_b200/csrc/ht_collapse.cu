// Collapse-table generation on the device: homogeneous-ellipsoid collapse with the
// reference's fixed-step "funny RK4" (EllipsoidalCollapse.jl:149-590 with solver = :rk4,
// the port of the Fortran HomogeneousEllipsoid.f90) or its adaptive Tsit5 path (solver =
// :diffeq, :333-485) for many (Frho, e_v, p_v) at once, and the zvir table of
// CollapseTable.jl:22-76 built from either.
//
// One thread integrates one ellipsoid in FP64; the entries are independent (20,000 for the
// 50 x 20 x 20 table).  The integration is a dependent chain of ~10^3 RK4 steps, each four
// right-hand sides with two Carlson RD evaluations (square-root chains): latency bound, so
// the launch uses small CTAs to spread the threads over every SM.  This file is compiled
// with -fmad=false: no product is fused into an addition, the operations run in the
// reference's order, and the one logarithm on the path (the oblate shape branch) is a
// series both sides carry, so the results follow the CPU restatement to the last bit.
#include <cmath>
#include <vector>

#include "ht_internal.cuh"

namespace {

constexpr int kRdMaxIt = 200;   // Carlson RD: rounds before the loop gives up (see below)
constexpr int kEvolveThreads = 64;

struct GrowthDev {
    const double* atab;
    const double* Da;
    const double* f;
    int ntab;
    double amin, amax, D_inf, D_a0, HD_inf, HD_a0;
};

struct EllDev {
    double Rvac, Rcurv;   // Omvac / Omnr, Omcurv / Omnr (EllipsoidalCollapse.jl:47-55)
    int fs, vs;           // iforce_strat, ivir_strat
    double fcoll[3];
    double tfac;
    int nstepmax;
    double zinit_fac;
};

// _hunt (Cosmology.jl:117-132): 1-based jlo.
__device__ int hunt(const double* xx, int n, double x) {
    const bool ascnd = xx[n - 1] > xx[0];
    int jlo = 0, jhi = n + 1;
    while (jhi - jlo > 1) {
        const int jm = (jhi + jlo) / 2;
        if ((x > xx[jm - 1]) == ascnd) jlo = jm;
        else jhi = jm;
    }
    return jlo;
}

// The same index from a starting guess: jlo is the number of entries below x (0 when x
// is NaN), which any search returns; the integration's a only grows, so a walk from the
// previous call's index takes a step or none instead of eleven dependent loads.
__device__ int hunt_from(const double* xx, int n, double x, int j) {
    while (j < n && x > xx[j]) ++j;
    while (j > 0 && !(x > xx[j - 1])) --j;
    return j;
}

// Interpolation window and Lagrange weights of Dlinear_ab / Dfnofa (Cosmology.jl:80-115,
// 287-330); a 4-point window never starts before the first entry.  *hint (nullable) holds
// the previous call's table index.
__device__ int growth_weights(const GrowthDev& g, double x, int* k0, double* w,
                              int* hint = nullptr) {
    const int kk = hint ? (*hint = hunt_from(g.atab, g.ntab, x, *hint)) : hunt(g.atab, g.ntab, x);
    int nl;
    if (kk < 2 || kk >= g.ntab) {
        nl = 2;
        *k0 = (kk - 1 > 1 ? kk - 1 : 1) - 1;
    } else {
        nl = 4;
        *k0 = (kk - 2 > 1 ? kk - 2 : 1) - 1;
    }
    const double* xa = g.atab + *k0;
    if (nl == 4) {
        w[0] = (x - xa[1]) / (xa[0] - xa[1]) * (x - xa[2]) / (xa[0] - xa[2]) * (x - xa[3]) / (xa[0] - xa[3]);
        w[1] = (x - xa[0]) / (xa[1] - xa[0]) * (x - xa[2]) / (xa[1] - xa[2]) * (x - xa[3]) / (xa[1] - xa[3]);
        w[2] = (x - xa[0]) / (xa[2] - xa[0]) * (x - xa[1]) / (xa[2] - xa[1]) * (x - xa[3]) / (xa[2] - xa[3]);
        w[3] = (x - xa[0]) / (xa[3] - xa[0]) * (x - xa[1]) / (xa[3] - xa[1]) * (x - xa[2]) / (xa[3] - xa[2]);
    } else {
        w[0] = (x - xa[1]) / (xa[0] - xa[1]);
        w[1] = 1.0 - w[0];
    }
    return nl;
}

__device__ double lagr(const double* v, int nl, const double* w) {
    return nl == 4 ? w[0] * v[0] + w[1] * v[1] + w[2] * v[2] + w[3] * v[3]
                   : w[0] * v[0] + w[1] * v[1];
}

// Dlinear_ab (Cosmology.jl:287-307): D(a) and dlnD/dlna.
__device__ void dlinear_ab(const GrowthDev& g, double ai, double* dlin, double* hd,
                           int* hint = nullptr) {
    if (ai > g.amin && ai < g.amax) {
        int k0;
        double w[4];
        const int nl = growth_weights(g, ai, &k0, w, hint);
        *dlin = lagr(g.Da + k0, nl, w) * ai;
        *hd = lagr(g.f + k0, nl, w);
    } else if (ai >= g.amax) {
        *dlin = g.D_a0 * ai;
        *hd = g.HD_a0;
    } else {
        *dlin = g.D_inf * ai;
        *hd = g.HD_inf;
    }
}

// Dfnofa (Cosmology.jl:310-330).
__device__ double dfnofa(const GrowthDev& g, double ai) {
    if (ai > g.amin && ai < g.amax) {
        int k0;
        double w[4];
        const int nl = growth_weights(g, ai, &k0, w);
        return ai * lagr(g.Da + k0, nl, w);
    }
    if (ai >= g.amax) return ai * g.D_a0;
    return ai * g.D_inf;
}

// Carlson's RD (EllipsoidalCollapse.jl:62-106), two argument sets side by side: each set
// runs its own duplication rounds until its own stopping test holds (a finished set stops
// changing) and then the final formula, so both results are those of two separate calls,
// while the two square-root / division chains overlap.  Finite positive arguments converge
// in a few dozen rounds; a set stops after kRdMaxIt rounds at the latest (the reference
// loops for ever on NaN arguments), as the CPU restatement does.
struct RdState {
    double xt, yt, zt, sum, fac, delx, dely, delz, ave;
    bool done;
};

__device__ __forceinline__ void rd_init(RdState& r, double x, double y, double z) {
    r.xt = x; r.yt = y; r.zt = z; r.sum = 0.0; r.fac = 1.0;
    r.delx = r.dely = r.delz = r.ave = 0.0;
    r.done = false;
}

__device__ __forceinline__ void rd_round(RdState& r) {
    const double ERRTOL = 0.05;
    const double sqrtx = sqrt(r.xt), sqrty = sqrt(r.yt), sqrtz = sqrt(r.zt);
    const double alamb = sqrtx * (sqrty + sqrtz) + sqrty * sqrtz;
    r.sum += r.fac / (sqrtz * (r.zt + alamb));
    r.fac *= 0.25;
    r.xt = 0.25 * (r.xt + alamb);
    r.yt = 0.25 * (r.yt + alamb);
    r.zt = 0.25 * (r.zt + alamb);
    r.ave = 0.2 * (r.xt + r.yt + 3.0 * r.zt);
    r.delx = (r.ave - r.xt) / r.ave;
    r.dely = (r.ave - r.yt) / r.ave;
    r.delz = (r.ave - r.zt) / r.ave;
    r.done = fmax(fmax(fabs(r.delx), fabs(r.dely)), fabs(r.delz)) <= ERRTOL;
}

__device__ __forceinline__ double rd_final(const RdState& r) {
    const double C1 = 3.0 / 14.0, C2 = 1.0 / 6.0, C3 = 9.0 / 22.0, C4 = 3.0 / 26.0,
                 C5 = 0.25 * C3, C6 = 1.5 * C4;
    const double delx = r.delx, dely = r.dely, delz = r.delz, ave = r.ave;
    const double ea = delx * dely, eb = delz * delz, ec = ea - eb, ed = ea - 6.0 * eb,
                 ee = ed + ec + ec;
    return 3.0 * r.sum + r.fac * (1.0 + ed * (-C1 + C5 * ed - C6 * delz * ee) +
                                  delz * (C2 * ee + delz * (-C3 * ec + delz * C4 * ea))) /
                             (ave * sqrt(ave));
}

__device__ void elliptic_rd2(double x1, double y1, double z1, double x2, double y2, double z2,
                             double* r1, double* r2) {
    RdState a, b;
    rd_init(a, x1, y1, z1);
    rd_init(b, x2, y2, z2);
    for (int it = 0; it < kRdMaxIt && !(a.done && b.done); ++it) {
        if (!a.done) rd_round(a);
        if (!b.done) rd_round(b);
    }
    *r1 = rd_final(a);
    *r2 = rd_final(b);
}

// Natural log of a finite x > 0 (and log2 x through log2x when non-null): x = m 2^e with m
// in [1/sqrt 2, sqrt 2), log x = e ln 2 + 2 atanh((m - 1)/(m + 1)), the atanh series summed
// to the 23rd power.  The CPU restatement carries the same function, operation for
// operation, so that both round alike (library logs may differ in the last bit, which the
// adaptive path would amplify into a different step sequence).
__device__ double log_series(double x, double* log2x) {
    int ex;
    double m = frexp(x, &ex);
    if (m < 0.7071067811865476) { m *= 2.0; ex -= 1; }
    const double s = (m - 1.0) / (m + 1.0), s2 = s * s;
    double t = 1.0 / 23.0;
    for (int k = 21; k >= 1; k -= 2) t = 1.0 / (double)k + s2 * t;
    const double lnm = 2.0 * s * t;
    if (log2x) *log2x = (double)ex + lnm * 1.4426950408889634;
    return (double)ex * 0.6931471805599453 + lnm;
}

// Shape integrals (EllipsoidalCollapse.jl:108-146, iwant_rd = 1).
__device__ void get_b_2(double a1, double a2, double a3, double* b) {
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
                        (1.0 / one_ecc2 - log_series((1.0 + ecc) / one_ecc, nullptr) * 0.5 / ecc));
        } else {
            const double ecc2 = 1.0 - r_3 * r_3, ecc = sqrt(ecc2);
            b3 = 0.5 * ((1.0 - ecc2) / ecc2 *
                        (1.0 / (1.0 - ecc2) -
                         log_series((1.0 + ecc) / (1.0 - ecc), nullptr) * 0.5 / ecc));
        }
        b[0] = 1.0 - 2.0 * b3;
        b[1] = b3;
        b[2] = b3;
        return;
    }
    const double r_22 = r_2 * r_2, r_32 = r_3 * r_3, qrat = third * r_2 * r_3;
    double rd3, rd2;
    elliptic_rd2(r_22, 1.0, r_32, r_32, 1.0, r_22, &rd3, &rd2);
    const double b3 = qrat * rd3;
    const double b2 = qrat * rd2;
    b[0] = 1.0 - (b2 + b3);
    b[1] = b2;
    b[2] = b3;
}

// DerivState (EllipsoidalCollapse.jl:174-191).
struct DState {
    int lvirv[3];
    int hint;             // growth-table index of the last lookup
    double a_3eq, a_2eq, a_1eq, a_3eq2, a_3eq1, Ha;
    double aLam[3], Frho_3;
};

__device__ double ha_b_nr(double a_b, const EllDev& e) {
    return sqrt((1.0 + e.Rvac * (a_b * a_b * a_b) + e.Rcurv * a_b) / a_b);
}

// get_derivs! (EllipsoidalCollapse.jl:200-290): dy at (t, y); freezes the virialised axes
// in y and advances the flags (also from the intermediate RK4 stages, as the Fortran does).
__device__ void get_derivs(const EllDev& e, const GrowthDev& g, double t, double* y,
                           double* dy, DState& ds) {
#pragma unroll
    for (int i = 0; i < 6; ++i) dy[i] = 0.0;
    const double a_b = t, a_b3 = a_b * a_b * a_b;
    const double Ha = ha_b_nr(a_b, e);
    ds.Ha = Ha;
    const double Ha_inv = 1.0 / Ha;
    if (ds.lvirv[2] == 0 && y[2] <= e.fcoll[2] * a_b) {
        ds.lvirv[2] = 1;
        ds.a_3eq = e.fcoll[2] * a_b;
        if (e.vs == 1) {
            ds.a_3eq2 = ds.a_3eq * 1.001;
            ds.a_3eq1 = ds.a_3eq * 1.0003;
        }
    }
    if (e.vs == 2 && ds.lvirv[1] == 0) ds.a_3eq2 = e.fcoll[1] * a_b;
    if (e.vs == 2 && ds.lvirv[0] == 0) ds.a_3eq1 = e.fcoll[0] * a_b;
    if (ds.lvirv[2] == 1 && y[1] <= ds.a_3eq2 && ds.lvirv[1] == 0) {
        ds.lvirv[1] = 1;
        ds.a_2eq = ds.a_3eq2;
    }
    if (ds.lvirv[2] == 1 && y[0] <= ds.a_3eq1 && ds.lvirv[0] == 0) {
        ds.lvirv[0] = 1;
        ds.a_1eq = ds.a_3eq1;
    }
    if (ds.lvirv[2] == 1) { y[2] = ds.a_3eq; y[5] = 0.0; dy[2] = 0.0; dy[5] = 0.0; }
    if (ds.lvirv[1] == 1) { y[1] = ds.a_2eq; y[4] = 0.0; dy[1] = 0.0; dy[4] = 0.0; }
    if (ds.lvirv[0] == 1) { y[0] = ds.a_1eq; y[3] = 0.0; dy[0] = 0.0; dy[3] = 0.0; }

    const double a1 = y[0], a2 = y[1], a3 = y[2];
    const double delta1_e = a_b3 / (a1 * a2 * a3);
    double d0, d1_int, d1_ext = 0.0;
    if (e.fs == 0) {
        d0 = -e.Rvac * Ha_inv;
        d1_int = 1.5 * delta1_e / a_b3 * Ha_inv;
    } else {
        d0 = (0.5 / a_b3 - e.Rvac) * Ha_inv;
        d1_int = 1.5 * (delta1_e - 1.0) / a_b3 * Ha_inv;
        if (e.fs == 4 || e.fs == 5 || e.fs == 6) {
            double dlin, hd;
            dlinear_ab(g, a_b, &dlin, &hd, &ds.hint);
            d1_ext = 1.5 / a_b3 * Ha_inv * dlin;
        } else if (e.fs == 3) {
            d1_ext = 1.5 * 2.5 / a_b3 * Ha_inv;
        }
    }
    double b[3] = {0.0, 0.0, 0.0};
    if (e.fs != 5 && e.fs != 6) get_b_2(a1, a2, a3, b);
    const double third = 1.0 / 3.0;
#pragma unroll
    for (int ax = 2; ax >= 0; --ax) {   // the reference's order: axes 3, 2, 1
        if (ds.lvirv[ax] != 0) continue;
        dy[ax] = y[ax + 3] * Ha_inv;
        double f = 0.0;
        if (e.fs == 0) f = -y[ax] * d1_int * b[ax];
        else if (e.fs == 1) f = -y[ax] * (d1_int * b[ax] + d0);
        else if (e.fs == 3) f = -y[ax] * (d1_int * b[ax] + d0 + d1_ext * (b[ax] - third));
        else if (e.fs == 4 || e.fs == 6)
            f = -y[ax] * (d1_int * b[ax] + d0 + d1_ext * (ds.aLam[ax] - ds.Frho_3));
        else if (e.fs == 5) f = -y[ax] * d0 - d1_ext * a_b * ds.aLam[ax];
        dy[ax + 3] = f;
    }
}

// One step of rk4_homel! (EllipsoidalCollapse.jl:149-172); dy holds the derivatives at
// (t, y).
__device__ void rk4_step(const EllDev& e, const GrowthDev& g, const double* y,
                         const double* dy, double t, double h, double* yout, DState& ds) {
    double yt[6], dyt[6], dym[6];
    const double hh = h * 0.5, h6 = h / 6.0, xh = t + hh;
#pragma unroll
    for (int i = 0; i < 6; ++i) yt[i] = y[i] + hh * dy[i];
    get_derivs(e, g, xh, yt, dyt, ds);
#pragma unroll
    for (int i = 0; i < 6; ++i) yt[i] = y[i] + hh * dyt[i];
    get_derivs(e, g, xh, yt, dym, ds);
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        yt[i] = y[i] + h * dym[i];
        dym[i] = dyt[i] + dym[i];
    }
    get_derivs(e, g, t + h, yt, dyt, ds);
#pragma unroll
    for (int i = 0; i < 6; ++i) yout[i] = y[i] + h6 * (dy[i] + dyt[i] + 2.0 * dym[i]);
}

// evolve_ellipse_full, solver = :rk4 (EllipsoidalCollapse.jl:492-590), one ellipsoid per
// thread: zvir = 1/a at event idynax (1-3 axis virialisation, 4-6 axis turnaround), D(a)
// there and Frho D; -1 for all three if the event does not happen before a = 2 or nstepmax
// steps.
__global__ void __launch_bounds__(kEvolveThreads) evolve_kernel(
    const EllDev e, const GrowthDev g, long long n, const double* __restrict__ Frho_in,
    const double* __restrict__ ev_in, const double* __restrict__ pv_in, int idynax,
    double* __restrict__ zout, double* __restrict__ Dout, double* __restrict__ fcout,
    int32_t* __restrict__ steps_out) {
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    const double Frho = Frho_in[q], e_v = ev_in[q], p_v = pv_in[q];
    DState ds;
    ds.lvirv[0] = ds.lvirv[1] = ds.lvirv[2] = 0;
    ds.hint = 0;
    ds.a_3eq = ds.a_2eq = ds.a_1eq = ds.a_3eq2 = ds.a_3eq1 = 0.0;
    ds.aLam[2] = Frho / 3.0 * (1.0 + 3.0 * e_v + p_v);
    ds.aLam[1] = Frho / 3.0 * (1.0 - 2.0 * p_v);
    ds.aLam[0] = Frho / 3.0 * (1.0 - 3.0 * e_v + p_v);
    ds.Frho_3 = Frho / 3.0;
    const double zinit = e.zinit_fac * Frho;
    const double a_b = 1.0 / zinit;
    double t = a_b, dlin, HD_Ha;
    dlinear_ab(g, a_b, &dlin, &HD_Ha);
    const double Ha = ha_b_nr(a_b, e);
    ds.Ha = Ha;
    double y[6], dy[6], yout[6];
#pragma unroll
    for (int ax = 2; ax >= 0; --ax) y[ax] = a_b * (1.0 - dlin * ds.aLam[ax]);
#pragma unroll
    for (int ax = 2; ax >= 0; --ax) y[ax + 3] = Ha * (1.0 - (1.0 + HD_Ha) * dlin * ds.aLam[ax]);
    double zdynv[6], aturnv[3] = {0.0, 0.0, 0.0};
    int ldynv[6];
#pragma unroll
    for (int i = 0; i < 6; ++i) { zdynv[i] = -1.0; ldynv[i] = 0; }
    int istep = 0;
    // bounded: every round advances istep, and the loop ends at nstepmax
    for (;;) {
        ++istep;
        const double a_3 = y[2];
        const double dtstep = e.tfac * a_3 * sqrt(a_3) * ds.Ha;
        get_derivs(e, g, t, y, dy, ds);
        rk4_step(e, g, y, dy, t, dtstep, yout, ds);
#pragma unroll
        for (int i = 0; i < 6; ++i) y[i] = yout[i];
        t += dtstep;
#pragma unroll
        for (int ii = 0; ii < 3; ++ii) {
            if (ds.lvirv[ii] != ldynv[ii]) {
                zdynv[ii] = 1.0 / t;
                ldynv[ii] = 1;
            }
        }
#pragma unroll
        for (int ii = 3; ii < 6; ++ii) {
            if (ldynv[ii] != 1) {
                if (y[ii - 3] < aturnv[ii - 3]) {
                    zdynv[ii] = 1.0 / t;
                    ldynv[ii] = 1;
                } else {
                    aturnv[ii - 3] = y[ii - 3];
                }
            }
        }
        if (ds.lvirv[0] == 1 || istep >= e.nstepmax || t >= 2.0) break;
    }
    double z = -1.0;
#pragma unroll
    for (int i = 0; i < 6; ++i)
        if (i == idynax - 1) z = zdynv[i];
    double D = -1.0, fc = -1.0;
    if (z != -1.0) {
        D = dfnofa(g, 1.0 / z);
        fc = Frho * D;
    }
    zout[q] = z;
    if (Dout) Dout[q] = D;
    if (fcout) fcout[q] = fc;
    if (steps_out) steps_out[q] = istep;
}

// ---------------------------------- solver = :diffeq: adaptive Tsit5 (:333-485) ----
//
// The same integrator as the CPU restatement (oracle or_evolve_tsit5), operation for
// operation, so that both take the same steps: Tsitouras' 5(4) pair with OrdinaryDiffEq's
// controls (starting step of Hairer, Norsett & Wanner; RMS error norm with abstol 1e-8,
// reltol 1e-6; PI controller beta1 = 7/50, beta2 = 2/25, safety 9/10, step ratio in
// [1/10, 5]; at most 100,000 iterations), stopping after the first accepted step at which
// axis 1 has virialised.

// x^y for finite x > 0: 2^(y log2 x), log2 x from log_series and 2^f from its Taylor
// series (about 1e-15 relative); plain arithmetic, so the host restatement rounds alike.
__device__ double pow_pos(double x, double y) {
    double l2;
    log_series(x, &l2);
    const double v = y * l2;
    const double nn = floor(v + 0.5);
    const double f = (v - nn) * 0.6931471805599453;
    double p = 1.0;
    for (int k = 16; k >= 1; --k) p = 1.0 + f * p / (double)k;
    return ldexp(p, (int)nn);
}

// VirState (EllipsoidalCollapse.jl:327-333), with the growth-table lookup hint.
struct VirDev {
    int lvirv[3];
    int hint;
    double a_eq[3], zdynv[3];
};

// _diffeq_rhs! (EllipsoidalCollapse.jl:344-438): du at (t, u); freezes the virialised axes
// in u and advances the flags at every evaluation (accepted step or not), recording 1/a at
// the evaluation that sets each.  aLam[3] = Frho / 3; iforce_strat 2 keeps the velocities.
__device__ void diffeq_rhs(const EllDev& e, const GrowthDev& g, const double* aLam, double t,
                           double* u, double* du, VirDev& v) {
    const double a_b = t, a_b3 = a_b * a_b * a_b;
    const double Ha = ha_b_nr(a_b, e);
    const double Ha_inv = 1.0 / Ha;
    if (v.lvirv[2] == 0 && u[2] <= e.fcoll[2] * a_b) {
        v.lvirv[2] = 1;
        v.a_eq[2] = e.fcoll[2] * a_b;
        v.zdynv[2] = 1.0 / a_b;
    }
    double a_3eq2 = 0.0, a_3eq1 = 0.0;
    if (e.vs == 2 && v.lvirv[1] == 0) a_3eq2 = e.fcoll[1] * a_b;
    else if (e.vs == 1 && v.lvirv[2] == 1) a_3eq2 = v.a_eq[2] * 1.001;
    if (e.vs == 2 && v.lvirv[0] == 0) a_3eq1 = e.fcoll[0] * a_b;
    else if (e.vs == 1 && v.lvirv[2] == 1) a_3eq1 = v.a_eq[2] * 1.0003;
    if (v.lvirv[2] == 1 && v.lvirv[1] == 0 && u[1] <= a_3eq2) {
        v.lvirv[1] = 1;
        v.a_eq[1] = a_3eq2;
        v.zdynv[1] = 1.0 / a_b;
    }
    if (v.lvirv[2] == 1 && v.lvirv[0] == 0 && u[0] <= a_3eq1) {
        v.lvirv[0] = 1;
        v.a_eq[0] = a_3eq1;
        v.zdynv[0] = 1.0 / a_b;
    }
#pragma unroll
    for (int ax = 2; ax >= 0; --ax)
        if (v.lvirv[ax] == 1) { u[ax] = v.a_eq[ax]; u[ax + 3] = 0.0; }

    const double a1 = u[0], a2 = u[1], a3 = u[2];
    const double delta1_e = a_b3 / (a1 * a2 * a3);
    const double Frho_3 = aLam[3];
    double d0, d1_int, d1_ext = 0.0;
    if (e.fs == 0) {
        d0 = -e.Rvac * Ha_inv;
        d1_int = 1.5 * delta1_e / a_b3 * Ha_inv;
    } else {
        d0 = (0.5 / a_b3 - e.Rvac) * Ha_inv;
        d1_int = 1.5 * (delta1_e - 1.0) / a_b3 * Ha_inv;
        if (e.fs == 4 || e.fs == 5 || e.fs == 6) {
            double dlin, hd;
            dlinear_ab(g, a_b, &dlin, &hd, &v.hint);
            d1_ext = 1.5 / a_b3 * Ha_inv * dlin;
        } else if (e.fs == 3) {
            d1_ext = 1.5 * 2.5 / a_b3 * Ha_inv;
        }
    }
    double b[3] = {0.0, 0.0, 0.0};
    if (e.fs != 5 && e.fs != 6) get_b_2(a1, a2, a3, b);
    const double third = 1.0 / 3.0;
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
        if (v.lvirv[ax] == 1) { du[ax] = 0.0; du[ax + 3] = 0.0; continue; }
        du[ax] = u[ax + 3] * Ha_inv;
        double f = 0.0;
        if (e.fs == 0) f = -u[ax] * d1_int * b[ax];
        else if (e.fs == 1) f = -u[ax] * (d1_int * b[ax] + d0);
        else if (e.fs == 3) f = -u[ax] * (d1_int * b[ax] + d0 + d1_ext * (b[ax] - third));
        else if (e.fs == 4 || e.fs == 6)
            f = -u[ax] * (d1_int * b[ax] + d0 + d1_ext * (aLam[ax] - Frho_3));
        else if (e.fs == 5) f = -u[ax] * d0 - d1_ext * a_b * aLam[ax];
        du[ax + 3] = f;
    }
}

// Tsitouras' 5(4) pair (Comput. Math. Appl. 62 (2011) 770-775) in OrdinaryDiffEq's
// tabulation: nodes, stage weights (row 7 = the solution weights, first same as last) and
// the weights of the embedded error estimate.
__constant__ double kTsC[7] = {0.0, 0.161, 0.327, 0.9, 0.9800255409045097, 1.0, 1.0};
__constant__ double kTsA[7][6] = {
    {0, 0, 0, 0, 0, 0},
    {0.161, 0, 0, 0, 0, 0},
    {-0.008480655492356989, 0.335480655492357, 0, 0, 0, 0},
    {2.897153057105493, -6.359448489975075, 4.3622954328695815, 0, 0, 0},
    {5.325864828439257, -11.748883564062828, 7.4955393428898365, -0.09249506636175525, 0, 0},
    {5.86145544294642, -12.92096931784711, 8.159367898576159, -0.071584973281401,
     -0.028269050394068383, 0},
    {0.09646076681806523, 0.01, 0.4798896504144996, 1.379008574103742, -3.290069515436081,
     2.324710524099774}};
__constant__ double kTsE[7] = {-0.00178001105222577714, -0.0008164344596567469,
                               0.007880878010261995, -0.1447110071732629,
                               0.5823571654525552, -0.45808210592918697,
                               0.015151515151515152};

__device__ double rms6(const double* v) {
    double s = 0.0;
#pragma unroll
    for (int i = 0; i < 6; ++i) s += v[i] * v[i];
    return sqrt(s / 6.0);
}

// _evolve_diffeq (EllipsoidalCollapse.jl:440-485), one ellipsoid per thread: zvir = 1/a at
// axis idynax's virialisation (1-3), D(a) there and Frho D, all -1 without the event
// before a = 2.  steps_out: the iterations (accepted and rejected steps).
__global__ void __launch_bounds__(kEvolveThreads) evolve_tsit5_kernel(
    const EllDev e, const GrowthDev g, long long n, const double* __restrict__ Frho_in,
    const double* __restrict__ ev_in, const double* __restrict__ pv_in, int idynax,
    double* __restrict__ zout, double* __restrict__ Dout, double* __restrict__ fcout,
    int32_t* __restrict__ steps_out) {
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    const double Frho = Frho_in[q], e_v = ev_in[q], p_v = pv_in[q];
    const double abstol = 1e-8, reltol = 1e-6, tend = 2.0;
    const int maxiters = 100000;
    double aLam[4];
    aLam[2] = Frho / 3.0 * (1.0 + 3.0 * e_v + p_v);
    aLam[1] = Frho / 3.0 * (1.0 - 2.0 * p_v);
    aLam[0] = Frho / 3.0 * (1.0 - 3.0 * e_v + p_v);
    aLam[3] = Frho / 3.0;
    VirDev v;
    v.hint = 0;
#pragma unroll
    for (int i = 0; i < 3; ++i) { v.lvirv[i] = 0; v.a_eq[i] = 0.0; v.zdynv[i] = -1.0; }
    const double zinit = e.zinit_fac * Frho;
    const double a_b = 1.0 / zinit;
    double dlin, HD_Ha;
    dlinear_ab(g, a_b, &dlin, &HD_Ha, &v.hint);
    const double Ha = ha_b_nr(a_b, e);
    double u[6];
#pragma unroll
    for (int ax = 2; ax >= 0; --ax) u[ax] = a_b * (1.0 - dlin * aLam[ax]);
#pragma unroll
    for (int ax = 2; ax >= 0; --ax) u[ax + 3] = Ha * (1.0 - (1.0 + HD_Ha) * dlin * aLam[ax]);
    double t = a_b;

    double k[7][6], tmp[6], sc[6], u1[6];
    diffeq_rhs(e, g, aLam, t, u, k[0], v);
#pragma unroll
    for (int i = 0; i < 6; ++i) sc[i] = abstol + fabs(u[i]) * reltol;
#pragma unroll
    for (int i = 0; i < 6; ++i) tmp[i] = u[i] / sc[i];
    const double d0 = rms6(tmp);
#pragma unroll
    for (int i = 0; i < 6; ++i) tmp[i] = k[0][i] / sc[i];
    const double d1 = rms6(tmp);
    double dt0 = (d0 < 1e-5 || d1 < 1e-5) ? 1e-6 : 0.01 * (d0 / d1);
    if (dt0 > tend - t) dt0 = tend - t;
#pragma unroll
    for (int i = 0; i < 6; ++i) u1[i] = u[i] + dt0 * k[0][i];
    diffeq_rhs(e, g, aLam, t + dt0, u1, k[1], v);
#pragma unroll
    for (int i = 0; i < 6; ++i) tmp[i] = (k[1][i] - k[0][i]) / sc[i];
    const double d2 = rms6(tmp) / dt0;
    const double dmax = d1 > d2 ? d1 : d2;
    const double dt1 = dmax <= 1e-15 ? (1e-6 > dt0 * 1e-3 ? 1e-6 : dt0 * 1e-3)
                                     : pow_pos(0.01 / dmax, 0.2);
    double dt = 100.0 * dt0 < dt1 ? 100.0 * dt0 : dt1;
    if (dt > tend - t) dt = tend - t;
    diffeq_rhs(e, g, aLam, t, u, k[0], v);   // the first FSAL stage

    double qold = 1e-4;
    int iter = 0;
    // bounded: every round advances iter, and the loop ends at maxiters
    while (iter < maxiters && t < tend) {
        ++iter;
        if (dt > tend - t) dt = tend - t;
        if (!(dt > 1e-14 * t)) break;   // step size underflow: give up
        for (int st = 1; st < 7; ++st) {
#pragma unroll
            for (int i = 0; i < 6; ++i) {
                double acc = 0.0;
                for (int j = 0; j < st; ++j) acc += kTsA[st][j] * k[j][i];
                tmp[i] = u[i] + dt * acc;
            }
            diffeq_rhs(e, g, aLam, t + kTsC[st] * dt, tmp, k[st], v);
        }
        // tmp is the step's end, frozen by the last evaluation
        double r[6];
#pragma unroll
        for (int i = 0; i < 6; ++i) {
            double acc = 0.0;
#pragma unroll
            for (int j = 0; j < 7; ++j) acc += kTsE[j] * k[j][i];
            const double au = fabs(u[i]), an = fabs(tmp[i]);
            r[i] = (dt * acc) / (abstol + (au > an ? au : an) * reltol);
        }
        const double EEst = rms6(r);
        if (EEst <= 1.0) {
            double qq;
            if (EEst == 0.0) {
                qq = 0.1;
            } else {
                qq = pow_pos(EEst, 0.14) / pow_pos(qold, 0.08) / 0.9;
                qq = qq < 5.0 ? qq : 5.0;
                qq = qq > 0.1 ? qq : 0.1;
            }
            t = t + dt;
            if (tend - t <= 1e-13 * tend) t = tend;
#pragma unroll
            for (int i = 0; i < 6; ++i) { u[i] = tmp[i]; k[0][i] = k[6][i]; }
            qold = EEst > 1e-4 ? EEst : 1e-4;
            dt = dt / qq;
            if (v.lvirv[0] == 1) break;   // the terminating callback
        } else {
            const double q11 = EEst == EEst ? pow_pos(EEst, 0.14) / 0.9 : 5.0;
            dt = dt / (q11 < 5.0 ? q11 : 5.0);
        }
    }
    double z = -1.0;
#pragma unroll
    for (int i = 0; i < 3; ++i)
        if (i == idynax - 1) z = v.zdynv[i];
    double D = -1.0, fc = -1.0;
    if (z != -1.0) {
        D = dfnofa(g, 1.0 / z);
        fc = Frho * D;
    }
    zout[q] = z;
    if (Dout) Dout[q] = D;
    if (fcout) fcout[q] = fc;
    if (steps_out) steps_out[q] = iter;
}

}  // namespace

// ------------------------------------------------------------------- host side ----

namespace {

int check_inputs(const ht_ellipsoid* ep, const ht_growth* g, const char* who) {
    const std::string w(who);
    if (!ep || !g) return ht_fail(HT_ERR_INVALID, w + ": params or growth table is NULL");
    if (!(ep->Om > 0.0)) return ht_fail(HT_ERR_INVALID, w + ": Om must be positive");
    if (ep->iforce_strat < 0 || ep->iforce_strat > 6)
        return ht_fail(HT_ERR_INVALID, w + ": iforce_strat must be in 0..6");
    if (ep->ivir_strat != 1 && ep->ivir_strat != 2)
        return ht_fail(HT_ERR_INVALID, w + ": ivir_strat must be 1 or 2");
    if (ep->solver != HT_SOLVER_RK4 && ep->solver != HT_SOLVER_TSIT5)
        return ht_fail(HT_ERR_INVALID, w + ": solver must be HT_SOLVER_RK4 or HT_SOLVER_TSIT5");
    if (ep->nstepmax < 1 || ep->nstepmax > 100000000)
        return ht_fail(HT_ERR_INVALID, w + ": nstepmax must be in 1..10^8");
    if (!(ep->tfac > 0.0) || !(ep->zinit_fac > 0.0))
        return ht_fail(HT_ERR_INVALID, w + ": tfac and zinit_fac must be positive");
    if (g->ntab < 4 || !g->atab || !g->D_atab || !g->dlnD_dlnatab)
        return ht_fail(HT_ERR_INVALID, w + ": growth table needs ntab >= 4 host arrays");
    for (int i = 1; i < g->ntab; ++i)
        if (!(g->atab[i] > g->atab[i - 1]))
            return ht_fail(HT_ERR_INVALID, w + ": growth table atab must be increasing");
    return HT_OK;
}

EllDev ell_dev(const ht_ellipsoid* ep) {
    EllDev e;
    const double Omnr = ep->Om, Omvac = ep->OL, Omcurv = 1.0 - ep->Om - ep->OL;
    e.Rvac = Omvac / Omnr;
    e.Rcurv = Omcurv / Omnr;
    e.fs = ep->iforce_strat;
    e.vs = ep->ivir_strat;
    for (int i = 0; i < 3; ++i) e.fcoll[i] = ep->fcoll[i];
    e.tfac = ep->tfac;
    e.nstepmax = ep->nstepmax;
    e.zinit_fac = ep->zinit_fac;
    return e;
}

}  // namespace

extern "C" HT_API int ht_evolve_ellipses(int device, const ht_ellipsoid* ep,
                                         const ht_growth* growth, int64_t n,
                                         const double* d_Frho, const double* d_e_v,
                                         const double* d_p_v, int32_t idynax, double* d_zvir,
                                         double* d_D, double* d_fc, int32_t* d_steps,
                                         void* stream) {
    HT_RANGE("ht_evolve_ellipses");
    int rc = check_inputs(ep, growth, "ht_evolve_ellipses");
    if (rc != HT_OK) return rc;
    if (n < 0) return ht_fail(HT_ERR_INVALID, "ht_evolve_ellipses: n < 0");
    if (idynax < 1 || idynax > 6)
        return ht_fail(HT_ERR_INVALID, "ht_evolve_ellipses: idynax must be in 1..6");
    if (ep->solver == HT_SOLVER_TSIT5 && idynax > 3)
        return ht_fail(HT_ERR_INVALID,
                       "ht_evolve_ellipses: the Tsit5 path records axis virialisation only "
                       "(idynax 1..3)");
    if (n == 0) return HT_OK;
    if (!d_Frho || !d_e_v || !d_p_v || !d_zvir)
        return ht_fail(HT_ERR_INVALID, "ht_evolve_ellipses: NULL input or output array");
    HT_CUDA_TRY(cudaSetDevice(device), "ht_evolve_ellipses: cudaSetDevice");
    cudaStream_t st = (cudaStream_t)stream;
    const int nt = growth->ntab;
    const size_t tb = (size_t)nt * sizeof(double);
    double* buf = nullptr;
    HT_CUDA_TRY(cudaMallocAsync((void**)&buf, 3 * tb, st), "ht_evolve_ellipses: growth table");
    cudaError_t e = cudaMemcpyAsync(buf, growth->atab, tb, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(buf + nt, growth->D_atab, tb, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(buf + 2 * nt, growth->dlnD_dlnatab, tb, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        GrowthDev g{buf, buf + nt, buf + 2 * nt, nt, growth->amintab, growth->amaxtab,
                    growth->D_ainfty, growth->D_a0, growth->HD_Hainfty, growth->HD_Ha0};
        const long long blocks = (n + kEvolveThreads - 1) / kEvolveThreads;
        if (ep->solver == HT_SOLVER_TSIT5)
            evolve_tsit5_kernel<<<(unsigned)blocks, kEvolveThreads, 0, st>>>(
                ell_dev(ep), g, (long long)n, d_Frho, d_e_v, d_p_v, idynax, d_zvir, d_D, d_fc,
                d_steps);
        else
            evolve_kernel<<<(unsigned)blocks, kEvolveThreads, 0, st>>>(
                ell_dev(ep), g, (long long)n, d_Frho, d_e_v, d_p_v, idynax, d_zvir, d_D, d_fc,
                d_steps);
        e = cudaGetLastError();
    }
    // stream-ordered release: after the kernel that reads the table
    const cudaError_t ef = cudaFreeAsync(buf, st);
    if (e != cudaSuccess) return ht_cuda_fail(e, "ht_evolve_ellipses: launch");
    if (ef != cudaSuccess) return ht_cuda_fail(ef, "ht_evolve_ellipses: growth table release");
    return HT_OK;
}

extern "C" HT_API int ht_collapse_table(int device, const ht_ellipsoid* ep,
                                        const ht_growth* growth, int32_t nx, int32_t ny,
                                        int32_t nz, double X1, double X2, double Y1, double Y2,
                                        double Z1, double Z2, float* table) {
    HT_RANGE("ht_collapse_table");
    int rc = check_inputs(ep, growth, "ht_collapse_table");
    if (rc != HT_OK) return rc;
    if (nx < 2 || ny < 2 || nz < 2)
        return ht_fail(HT_ERR_INVALID, "ht_collapse_table: every axis needs >= 2 points");
    if (!table) return ht_fail(HT_ERR_INVALID, "ht_collapse_table: table is NULL");
    const long long n = (long long)nx * ny * nz;
    if (n > (1LL << 31)) return ht_fail(HT_ERR_INVALID, "ht_collapse_table: table too large");
    // the grid of CollapseTable.jl:29-50 on the host (10^x with the host's pow, as the
    // CPU restatement and Julia's 10.0^logF)
    const double dX = (X2 - X1) / (nx - 1), dY = (Y2 - Y1) / (ny - 1), dZ = (Z2 - Z1) / (nz - 1);
    std::vector<double> h(3 * (size_t)n);
    for (long long q = 0; q < n; ++q) {
        const int i = (int)(q % nx), j = (int)((q / nx) % ny), k = (int)(q / ((long long)nx * ny));
        const double x = X1 + i * dX, y = Y1 + j * dY, z = Z1 + k * dZ;
        h[q] = std::pow(10.0, x);
        h[n + q] = y;
        h[2 * n + q] = z * y;
    }
    HT_CUDA_TRY(cudaSetDevice(device), "ht_collapse_table: cudaSetDevice");
    double* d = nullptr;
    HT_CUDA_TRY(cudaMalloc((void**)&d, 4 * (size_t)n * sizeof(double)), "ht_collapse_table: buffers");
    cudaError_t e = cudaMemcpy(d, h.data(), 3 * (size_t)n * sizeof(double), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        cudaFree(d);
        return ht_cuda_fail(e, "ht_collapse_table: upload");
    }
    rc = ht_evolve_ellipses(device, ep, growth, n, d, d + n, d + 2 * n, 1, d + 3 * n, nullptr,
                            nullptr, nullptr, nullptr);
    if (rc == HT_OK) {
        e = cudaMemcpy(h.data(), d + 3 * n, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) rc = ht_cuda_fail(e, "ht_collapse_table: download");
    }
    cudaFree(d);
    if (rc != HT_OK) return rc;
    for (long long q = 0; q < n; ++q) table[q] = (float)h[q];
    return HT_OK;
}
