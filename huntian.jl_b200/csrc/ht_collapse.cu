// Collapse-table generation on the device: homogeneous-ellipsoid collapse with the
// reference's fixed-step "funny RK4" (EllipsoidalCollapse.jl:149-590 with solver = :rk4,
// the port of the Fortran HomogeneousEllipsoid.f90) for many (Frho, e_v, p_v) at once,
// and the zvir table of CollapseTable.jl:22-76 built from it.
//
// One thread integrates one ellipsoid in FP64; the entries are independent (20,000 for the
// 50 x 20 x 20 table).  The integration is a dependent chain of ~10^3 RK4 steps, each four
// right-hand sides with two Carlson RD evaluations (square-root chains): latency bound, so
// the launch uses small CTAs to spread the threads over every SM.  This file is compiled
// with -fmad=false: no product is fused into an addition, the operations run in the
// reference's order, and the results follow the CPU restatement to the last bit except
// where the library log of the oblate shape branch differs by an ulp.
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
                        (1.0 / one_ecc2 - log((1.0 + ecc) / one_ecc) * 0.5 / ecc));
        } else {
            const double ecc2 = 1.0 - r_3 * r_3, ecc = sqrt(ecc2);
            b3 = 0.5 * ((1.0 - ecc2) / ecc2 *
                        (1.0 / (1.0 - ecc2) - log((1.0 + ecc) / (1.0 - ecc)) * 0.5 / ecc));
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
