/*
 * CPU oracle for the halo-finding hot path.  TEST INFRASTRUCTURE ONLY (see ht_oracle.h):
 * a literal FP64 restatement of the reference Julia code, used by tests/ as the checker
 * and by bench.py as the timed CPU baseline.  The CUDA product never calls it.
 *
 * Reference files (guanyilun/Huntian.jl):
 *   src/HaloFinder/PeakFind.jl          find_peaks
 *   src/HaloFinder/RadialShell.jl       hRinteg, atab4, precompute_shells, fsc_of_z,
 *                                       kernel_strain, get_evals, analyse_peak
 *   src/ShellAnalysisGPU.jl             build_shell_tables, analyse_peak_gpu
 *   src/EllipsoidalCollapse/CollapseTable.jl   trilinear lookup with -1 outside
 *
 * Arithmetic follows Julia's promotion rules: fields are Float32, accumulators Float64,
 * and Float32*Int32 products (delta*offset, eta*offset) are rounded to Float32 before
 * being added to the Float64 accumulators, exactly as `Float32 * Int32 -> Float32` does.
 * Build with -ffp-contract=off so no product is fused into an add.
 */
#include "ht_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define PI_D 3.14159265358979323846
#define FOURPI (4.0 * PI_D)

/* ---------------------------------------------------------------- shells ---- */

/* RadialShell.jl:151-166.  Generation order dk, dj, di (di fastest); the counting sort
 * on r2 is stable, which reproduces Julia's stable sort!(cells; by = r2). */
int64_t or_precompute_shells(int rmax, or_cell* out, int64_t cap)
{
    const int r2max = rmax * rmax;
    int64_t* hist = (int64_t*)calloc((size_t)r2max + 2, sizeof(int64_t));
    int64_t total = 0;
    for (int dk = -rmax; dk <= rmax; ++dk)
        for (int dj = -rmax; dj <= rmax; ++dj)
            for (int di = -rmax; di <= rmax; ++di) {
                int r2 = di * di + dj * dj + dk * dk;
                if (r2 <= r2max) { hist[r2 + 1]++; total++; }
            }
    if (out != NULL) {
        for (int r = 1; r <= r2max + 1; ++r) hist[r] += hist[r - 1];
        for (int dk = -rmax; dk <= rmax; ++dk)
            for (int dj = -rmax; dj <= rmax; ++dj)
                for (int di = -rmax; di <= rmax; ++di) {
                    int r2 = di * di + dj * dj + dk * dk;
                    if (r2 <= r2max) {
                        int64_t pos = hist[r2]++;
                        if (pos < cap) {
                            out[pos].di = di; out[pos].dj = dj; out[pos].dk = dk;
                            out[pos].r2 = r2;
                        }
                    }
                }
    }
    free(hist);
    return total;
}

/* ShellAnalysisGPU.jl:44-71 (start is 0-based here). */
int or_build_shell_tables(const or_cell* cells, int64_t ncells,
                          int64_t* start, int32_t* count, int32_t* r2, int cap)
{
    int ns = 0;
    int64_t i = 0;
    while (i < ncells) {
        int32_t rr = cells[i].r2;
        int64_t s0 = i;
        while (i < ncells && cells[i].r2 == rr) ++i;
        if (ns < cap) { start[ns] = s0; count[ns] = (int32_t)(i - s0); r2[ns] = rr; }
        ++ns;
    }
    return ns;
}

/* ------------------------------------------------------------ SPH kernels ---- */

/* RadialShell.jl:95-121 */
double or_hRinteg(double u0, double u12)
{
    double x0 = fabs(u0);
    if (x0 >= 2.0) return 0.0;
    const double one7 = 1.0 / 7.0;
    double result = 1.6 * u12 - 6.4 * one7;
    double x02 = x0 * x0;
    double x04 = x02 * x02;
    if (x0 >= 1.0) {
        double h1 = x04 * (2.0 - x0 * (2.4 - x0 * (1.0 - x0 * one7)));
        double h2 = x02 * (4.0 - x0 * (4.0 - x0 * (1.5 - x0 * 0.2)));
        result = result - h2 * u12 + h1;
    } else {
        result = result - 0.2 * (u12 - one7);
        if (x0 > 0.0) {
            double h1 = x04 * (1.0 - x02 * (1.0 - 3.0 * x0 * one7));
            double h2 = x02 * (2.0 - x02 * (1.5 - 0.6 * x0));
            result = result - h2 * u12 + h1;
        }
    }
    return result;
}

/* RadialShell.jl:125-142 (out[0] is Julia's akk[1]). */
void or_atab4(double out[1101])
{
    const double ca = 3.0 / (2.0 * PI_D);
    const double cb = 1.0 / (4.0 * PI_D);
    for (int i = 1; i <= 1100; ++i) {
        double u = (i - 1) * 0.01;
        double ru = sqrt(u);
        double v;
        if (ru < 1.0) v = ca * (2.0 / 3.0 - u + 0.5 * u * ru);
        else if (ru <= 2.0) { double t = 2.0 - ru; v = cb * (t * t * t); }
        else v = 0.0;
        out[i - 1] = v;
    }
    out[1100] = 0.0;
}

/* --------------------------------------------------------- collapse table ---- */

/* CollapseTable.jl:126-138: Interpolations.jl BSpline(Linear()) on scaled regular axes,
 * extrapolate(.., -1): inside the closed box a trilinear blend, outside out_val. */
double or_interp(const or_ctab* ct, double x, double y, double z)
{
    if (!(x >= ct->x1 && x <= ct->x2 && y >= ct->y1 && y <= ct->y2 &&
          z >= ct->z1 && z <= ct->z2))
        return ct->out_val;
    double tx = (x - ct->x1) / ((ct->x2 - ct->x1) / (ct->nx - 1));
    double ty = (y - ct->y1) / ((ct->y2 - ct->y1) / (ct->ny - 1));
    double tz = (z - ct->z1) / ((ct->z2 - ct->z1) / (ct->nz - 1));
    int ix = (int)floor(tx), iy = (int)floor(ty), iz = (int)floor(tz);
    if (ix > ct->nx - 2) ix = ct->nx - 2;
    if (iy > ct->ny - 2) iy = ct->ny - 2;
    if (iz > ct->nz - 2) iz = ct->nz - 2;
    if (ix < 0) ix = 0;
    if (iy < 0) iy = 0;
    if (iz < 0) iz = 0;
    double fx = tx - ix, fy = ty - iy, fz = tz - iz;
    const int64_t sx = 1, sy = ct->nx, sz = (int64_t)ct->nx * ct->ny;
    const float* t = ct->table + ix * sx + iy * sy + iz * sz;
    double c000 = t[0], c100 = t[sx], c010 = t[sy], c110 = t[sx + sy];
    double c001 = t[sz], c101 = t[sx + sz], c011 = t[sy + sz], c111 = t[sx + sy + sz];
    double c00 = c000 * (1.0 - fx) + c100 * fx;
    double c10 = c010 * (1.0 - fx) + c110 * fx;
    double c01 = c001 * (1.0 - fx) + c101 * fx;
    double c11 = c011 * (1.0 - fx) + c111 * fx;
    double c0 = c00 * (1.0 - fy) + c10 * fy;
    double c1 = c01 * (1.0 - fy) + c11 * fy;
    return c0 * (1.0 - fz) + c1 * fz;
}

/* RadialShell.jl:181-195 */
double or_fsc_of_z(double z, const or_ctab* ct)
{
    double target = 1.0 + z;
    double lo = ct->x1, hi = ct->x2;
    for (int it = 0; it < 50; ++it) {
        double mid = 0.5 * (lo + hi);
        double zv = or_interp(ct, mid, 0.0, 0.0);
        if (zv > target) hi = mid; else lo = mid;
    }
    return pow(10.0, lo);
}

/* -------------------------------------------------------------- eigen 3x3 ---- */

/* Cyclic Jacobi (Golub & Van Loan, Alg. 8.4.3) on the upper triangle, as
 * Symmetric(mat) reads it (RadialShell.jl:215-220); eigenvalues sorted ascending. */
void or_eigvals_sym3(const double a_in[9], double lam[3])
{
    double a[3][3];
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) {
            int rr = r < c ? r : c, cc = r < c ? c : r;   /* upper triangle */
            a[r][c] = a_in[rr + 3 * cc];
        }
    for (int sweep = 0; sweep < 64; ++sweep) {
        double off = a[0][1] * a[0][1] + a[0][2] * a[0][2] + a[1][2] * a[1][2];
        double dia = a[0][0] * a[0][0] + a[1][1] * a[1][1] + a[2][2] * a[2][2];
        if (off == 0.0 || off <= 1e-40 * dia) break;
        for (int p = 0; p < 2; ++p)
            for (int q = p + 1; q < 3; ++q) {
                double apq = a[p][q];
                if (apq == 0.0) continue;
                double theta = (a[q][q] - a[p][p]) / (2.0 * apq);
                double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
                double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
                for (int k = 0; k < 3; ++k) {        /* A <- A J (columns p, q) */
                    double akp = a[k][p], akq = a[k][q];
                    a[k][p] = c * akp - s * akq;
                    a[k][q] = s * akp + c * akq;
                }
                for (int k = 0; k < 3; ++k) {        /* A <- J^T A (rows p, q) */
                    double apk = a[p][k], aqk = a[q][k];
                    a[p][k] = c * apk - s * aqk;
                    a[q][k] = s * apk + c * aqk;
                }
                a[p][q] = a[q][p] = 0.0;
            }
    }
    double e0 = a[0][0], e1 = a[1][1], e2 = a[2][2], t;
    if (e0 > e1) { t = e0; e0 = e1; e1 = t; }
    if (e1 > e2) { t = e1; e1 = e2; e2 = t; }
    if (e0 > e1) { t = e0; e0 = e1; e1 = t; }
    lam[0] = e0; lam[1] = e1; lam[2] = e2;
}

/* ------------------------------------------------------------- peak find ---- */

#define IDX(g, i, j, k) ((int64_t)((i) - 1) + (int64_t)(g##n1) * ((j) - 1) + \
                         (int64_t)(g##n1) * (g##n2) * ((k) - 1))

/* PeakFind.jl:15-78 */
int64_t or_find_peaks(const float* delta, int8_t* mask, int n1, int n2, int n3,
                      int nbuff, float fcrit, int64_t max_peaks,
                      int32_t* out_i, int32_t* out_j, int32_t* out_k, float* out_delta)
{
    int64_t np = 0;
    const int64_t s1 = n1, s2 = (int64_t)n1 * n2;
    for (int k = nbuff + 1; k <= n3 - nbuff; ++k)
        for (int j = nbuff + 1; j <= n2 - nbuff; ++j)
            for (int i = nbuff + 1; i <= n1 - nbuff; ++i) {
                int64_t c = (i - 1) + s1 * (j - 1) + s2 * (k - 1);
                if (mask[c] == 1) continue;
                float ff = delta[c];
                if (ff < fcrit) continue;
                int is_max = 1;
                for (int kk = -1; kk <= 1 && is_max; ++kk)
                    for (int jj = -1; jj <= 1 && is_max; ++jj)
                        for (int ii = -1; ii <= 1; ++ii)
                            if (ff < delta[c + ii + s1 * jj + s2 * kk]) { is_max = 0; break; }
                if (!is_max) continue;
                out_i[np] = i; out_j[np] = j; out_k[np] = k; out_delta[np] = ff;
                ++np;
                mask[c] = 1;
                if (np >= max_peaks) return np;
            }
    return np;
}

/* ------------------------------------------------------------ shell walk ---- */

typedef struct {   /* 1-based per-shell profile arrays, size maxm + 2 */
    int64_t maxm;
    double *rad, *Fbar;
    int64_t* nshell;
    double *S[3], *S2[3], *G[3], *Gf[3], *SR[3][3];
} prof_t;

static void prof_alloc(prof_t* p, int64_t maxm)
{
    p->maxm = maxm;
    size_t n = (size_t)maxm + 3;
    p->rad = (double*)calloc(n, sizeof(double));
    p->Fbar = (double*)calloc(n, sizeof(double));
    p->nshell = (int64_t*)calloc(n, sizeof(int64_t));
    for (int L = 0; L < 3; ++L) {
        p->S[L] = (double*)calloc(n, sizeof(double));
        p->S2[L] = (double*)calloc(n, sizeof(double));
        p->G[L] = (double*)calloc(n, sizeof(double));
        p->Gf[L] = (double*)calloc(n, sizeof(double));
        for (int K = 0; K < 3; ++K) p->SR[L][K] = (double*)calloc(n, sizeof(double));
    }
}

static void prof_free(prof_t* p)
{
    free(p->rad); free(p->Fbar); free(p->nshell);
    for (int L = 0; L < 3; ++L) {
        free(p->S[L]); free(p->S2[L]); free(p->G[L]); free(p->Gf[L]);
        for (int K = 0; K < 3; ++K) free(p->SR[L][K]);
    }
}

static double g_akk[1101];
static int g_akk_ready = 0;
static const double* akk_table(void)
{
    if (!g_akk_ready) {
#ifdef _OPENMP
#pragma omp critical(or_akk)
#endif
        {
            if (!g_akk_ready) { or_atab4(g_akk); g_akk_ready = 1; }
        }
    }
    return g_akk;
}

/* RadialShell.jl:225-274.  E is column-major 3x3. */
static void kernel_strain(const prof_t* P, int64_t mp, int64_t mlow, int64_t mupp,
                          double wRnor, double aRnor, double E[9], double grad[3],
                          double gradf[3])
{
    const double* akk = akk_table();
    const double hlatt_1 = 1.0, hlatt_2 = 1.0;
    for (int i = 0; i < 9; ++i) E[i] = 0.0;
    for (int i = 0; i < 3; ++i) { grad[i] = 0.0; gradf[i] = 0.0; }
    if (mp > 1) {
        for (int64_t m1 = mlow; m1 <= mupp; ++m1) {
            double u0 = hlatt_1 * (P->rad[mp] - P->rad[m1]);
            double u02 = u0 * u0;
            if (u02 < 4.0) {
                double u12 = hlatt_2 * (P->rad[mp] * P->rad[mp] + P->rad[m1] * P->rad[m1]);
                double den = u12 - u02;
                double wt = or_hRinteg(u0, u12) / (den * den);
                for (int L = 0; L < 3; ++L) {
                    grad[L] += wt * P->G[L][m1];
                    gradf[L] += wt * P->Gf[L][m1];
                    for (int K = 0; K < 3; ++K)
                        E[L + 3 * K] -= 0.5 * wt * (P->SR[L][K][m1] + P->SR[K][L][m1]);
                }
            }
        }
        double scale = wRnor / P->rad[mp];
        for (int i = 0; i < 9; ++i) E[i] *= scale;
        for (int i = 0; i < 3; ++i) { grad[i] *= scale; gradf[i] *= scale; }
    } else {
        for (int64_t m1 = mlow; m1 <= mupp; ++m1) {
            double u0 = hlatt_1 * P->rad[m1];
            double con = 100.0 * u0 * u0;
            int64_t icon = (int64_t)floor(con);
            double diff = con - (double)icon;
            int64_t i2c = icon + 1;                       /* 1-based akk index */
            double aww = akk[i2c - 1] + diff * (akk[i2c] - akk[i2c - 1]);
            double wt = 0.5 * aww / P->rad[m1];
            for (int L = 0; L < 3; ++L) {
                grad[L] += wt * P->G[L][m1];
                gradf[L] += wt * P->Gf[L][m1];
                for (int K = 0; K < 3; ++K)
                    E[L + 3 * K] -= 0.5 * wt * (P->SR[L][K][m1] + P->SR[K][L][m1]);
            }
        }
        for (int i = 0; i < 9; ++i) E[i] *= aRnor;
        for (int i = 0; i < 3; ++i) { grad[i] *= aRnor; gradf[i] *= aRnor; }
    }
}

static void ev_pv(const double E[9], double* Frho, double* e_v, double* p_v, double lam_out[3])
{
    double lam[3];
    or_eigvals_sym3(E, lam);
    double F = lam[0] + lam[1] + lam[2];
    *Frho = F;
    *e_v = 0.0; *p_v = 0.0;
    if (F > 0.0) {
        *e_v = 0.5 * (lam[2] - lam[0]) / F;
        *p_v = 0.5 * (lam[2] + lam[0] - 2.0 * lam[1]) / F;
    }
    if (lam_out) { lam_out[0] = lam[0]; lam_out[1] = lam[1]; lam_out[2] = lam[2]; }
}

/* Product of a Float32 field value and an integer offset as the reference forms it:
 * Float32 * Int32 is Float32 in Julia, so every cell product is rounded to Float32 before
 * it enters the Float64 shell sum (RadialShell.jl:437-443, ShellAnalysisGPU.jl:205-215).
 * With exact products on (or_set_exact_products) the product is formed in Float64, where
 * it is exact: the "full-FP64" variant of the oracle, whose difference from the default
 * is the reference's own rounding noise. */
static int g_exact_products = 0;

void or_set_exact_products(int on) { g_exact_products = on != 0; }

static inline double cell_product(float v, int32_t d)
{
    return g_exact_products ? (double)v * (double)d : (double)(float)(v * (float)d);
}

static void set_no_collapse(or_result* r)
{
    memset(r, 0, sizeof(*r));
    r->RTHL = -1.0;
    r->zvir_half = -1.0;
    r->margin = INFINITY;
}

/* Smallest |value - threshold| over the collapse-deciding comparisons of one peak (the
 * Fbar-vs-fcrit tests of the crossing search and the zvir-vs-ZZon tests of the inward
 * walk): a diagnostic for collapse flips against another implementation, not a
 * reference output. */
static void note_margin(double* margin, double diff)
{
    const double d = fabs(diff);
    if (d < *margin) *margin = d;
}

/* Shared tail of analyse_peak / analyse_peak_gpu once the profiles exist:
 * RadialShell.jl:449-859 (ShellAnalysisGPU.jl:233-535).  m = last finalised shell.
 * gpu_conv selects the analyse_peak_gpu differences (mrf lag, Frhoh guard, d2F / mask
 * over the shell table); zvir selects whether zvir_half is computed. */
typedef struct {
    const or_grid* g; int ipk[3]; const or_cell* shells; int64_t npart;
    const int64_t* st_start; const int32_t* st_count; const int32_t* st_r2; int nshells;
    int64_t nshells_max;
} walk_ctx;

static int tail(const walk_ctx* W, prof_t* P, int64_t m, int64_t m0, int64_t mupp,
                int64_t mrf, double alatt, double ZZon, double fcrit, const or_ctab* ct,
                int nbuff, int gpu_conv, int zvir, or_result* out)
{
    const double aRnor = 3.0 / alatt;
    const double wRnor = 3.0 * (1.0 / FOURPI) / alatt;
    double E[9], g1[3], gf1[3];

    /* gradient at the filter scale (RadialShell.jl:466-482) */
    double rlow_rf = fmax(P->rad[mrf] - 2.0, 0.0);
    int64_t mlow_rf = mrf;
    if (mrf > 1)
        for (int64_t m1 = mrf - 1; m1 >= 1; --m1) if (P->rad[m1] > rlow_rf) mlow_rf = m1;
    double rupp_rf = P->rad[mrf] + 2.0;
    int64_t mupp_rf = mrf;
    for (int64_t m1 = mrf + 1; m1 <= m; ++m1) if (P->rad[m1] < rupp_rf) mupp_rf = m1;
    double gradpkrf[3];
    kernel_strain(P, mrf, mlow_rf, mupp_rf, wRnor, aRnor, E, gradpkrf, gf1);

    /* crossing (RadialShell.jl:485-526) */
    double margin = INFINITY;
    note_margin(&margin, P->Fbar[m0] - fcrit);
    if (P->Fbar[m0] >= fcrit) {
        int found = 0;
        for (int64_t mm = m0; mm <= m; ++mm) {
            note_margin(&margin, P->Fbar[mm] - fcrit);
            if (P->Fbar[mm] < fcrit) { m0 = mm; found = 1; break; }
        }
        if (!found) mupp = m;
        if (found) {
            double rupp_m0 = P->rad[m0] + 2.0;
            mupp = m0;
            for (int64_t mm = m0 + 1; mm <= m; ++mm) if (P->rad[mm] < rupp_m0) mupp = mm;
        }
    } else {
        int64_t mstart = m0 - 1 > 1 ? m0 - 1 : 1;
        int found = 0;
        for (int64_t mp = mstart; mp >= 1; --mp) {
            note_margin(&margin, P->Fbar[mp] - fcrit);
            if (P->Fbar[mp] >= fcrit) { found = 1; break; }
            m0 = mp;
        }
        if (!found) { set_no_collapse(out); out->margin = margin; return 2; }
        double rupp_m0 = P->rad[m0] + 2.0;
        int64_t mupp_new = m0;
        for (int64_t mm = m0 + 1; mm <= m; ++mm) if (P->rad[mm] < rupp_m0) mupp_new = mm;
        mupp = mupp_new;
    }

    /* inward walk (RadialShell.jl:530-686) */
    double rlow = fmax(P->rad[m0] - 2.0, 0.0);
    int64_t mlow = m0;
    if (m0 > 1)
        for (int64_t m1 = m0 - 1; m1 >= 1; --m1) if (P->rad[m1] > rlow) mlow = m1;

    double Ebar_m0[9], gp_m0[3], gpf_m0[3];
    kernel_strain(P, m0, mlow, mupp, wRnor, aRnor, Ebar_m0, gp_m0, gpf_m0);
    double Frho_m0, e_v_m0, p_v_m0;
    ev_pv(Ebar_m0, &Frho_m0, &e_v_m0, &p_v_m0, NULL);
    double Frhoh_m0 = Frho_m0;
    Frho_m0 = P->Fbar[m0];
    const double zvir1p_m0 = -1.0;   /* RadialShell.jl:566-567 */

    double zvir1 = -1.0, zvir1p = -1.0;
    double Ebar_last[9], strain_mat[9], gp_last[3], gpf_last[3], gp_prev[3], gpf_prev[3];
    double Frhoh, Frho, e_v, p_v, Frhpk, Fnupk, Fevpk, Fpvpk;
    int collapsed = 0;
    memcpy(Ebar_last, Ebar_m0, sizeof E); memcpy(strain_mat, Ebar_m0, sizeof E);
    memcpy(gp_last, gp_m0, sizeof g1); memcpy(gpf_last, gpf_m0, sizeof g1);
    memcpy(gp_prev, gp_m0, sizeof g1); memcpy(gpf_prev, gpf_m0, sizeof g1);
    Frhoh = Frhoh_m0; Frho = Frho_m0; e_v = e_v_m0; p_v = p_v_m0;
    Frhpk = Frhoh_m0; Fnupk = Frho_m0; Fevpk = e_v_m0; Fpvpk = p_v_m0;

    if (zvir1p_m0 >= ZZon) {
        zvir1 = -1.0; zvir1p = zvir1p_m0; collapsed = 1;
    } else {
        zvir1 = zvir1p_m0;
        if (m0 == 1) { set_no_collapse(out); out->margin = margin; return 3; }
        for (int64_t mp = m0 - 1; mp >= 1; --mp) {
            double rupp_mp = P->rad[mp] + 2.0;
            double rlow_mp = fmax(P->rad[mp] - 2.0, 0.0);
            if (P->rad[mupp] > rupp_mp) {
                int64_t mupp_new = mp;
                for (int64_t m1 = mp + 1; m1 <= mupp; ++m1) if (P->rad[m1] < rupp_mp) mupp_new = m1;
                mupp = mupp_new;
            }
            if (mlow > 1 && P->rad[mlow - 1] > rlow_mp) {
                int64_t mlownew = mlow;
                for (int64_t m1 = mlow - 1; m1 >= 1; --m1) if (P->rad[m1] > rlow_mp) mlownew = m1;
                mlow = mlownew;
            }
            double Eb[9], gp[3], gpf[3];
            kernel_strain(P, mp, mlow, mupp, wRnor, aRnor, Eb, gp, gpf);
            double Frho_mp, e_v_mp, p_v_mp;
            ev_pv(Eb, &Frho_mp, &e_v_mp, &p_v_mp, NULL);
            double Frhoh_mp = Frho_mp;
            Frho_mp = P->Fbar[mp];
            double zvir1p_mp = -1.0;
            if (Frho_mp > 0.0) {
                double poe = e_v_mp < 1e-5 ? 0.0 : p_v_mp / e_v_mp;
                zvir1p_mp = or_interp(ct, log10(Frho_mp), e_v_mp, poe);
                note_margin(&margin, zvir1p_mp - ZZon);
            }
            if (zvir1p_mp >= ZZon) {
                m0 = mp + 1;
                zvir1p = zvir1p_mp;
                memcpy(Ebar_last, Eb, sizeof E);
                memcpy(gp_last, gp, sizeof g1); memcpy(gpf_last, gpf, sizeof g1);
                Frhoh = Frhoh_mp; Frho = Frho_mp; e_v = e_v_mp; p_v = p_v_mp;
                collapsed = 1;
                break;
            }
            zvir1 = zvir1p_mp;
            Frhpk = Frhoh_mp; Fnupk = Frho_mp; Fevpk = e_v_mp; Fpvpk = p_v_mp;
            memcpy(gp_prev, gp, sizeof g1); memcpy(gpf_prev, gpf, sizeof g1);
            memcpy(strain_mat, Eb, sizeof E);
            Frhoh = Frhoh_mp; Frho = Frho_mp; e_v = e_v_mp; p_v = p_v_mp;
            memcpy(Ebar_last, Eb, sizeof E);
            memcpy(gp_last, gp, sizeof g1); memcpy(gpf_last, gpf, sizeof g1);
        }
    }
    /* Frhpk..Fpvpk, Frho, e_v, p_v are carried as in the reference but unused there */
    (void)Frhpk; (void)Fnupk; (void)Fevpk; (void)Fpvpk; (void)Frho; (void)e_v; (void)p_v;
    if (!collapsed) { set_no_collapse(out); out->margin = margin; return 4; }

    /* RTHL (RadialShell.jl:689-700) */
    double dZvir = zvir1p - zvir1, RTHL;
    double rp = P->rad[m0 - 1], rm = P->rad[m0];
    if (zvir1 > 0.0 && dZvir != 0.0) {
        double RTHL3 = rp * rp * rp + (rm * rm * rm - rp * rp * rp) * (zvir1p - ZZon) / dZvir;
        RTHL = pow(RTHL3, 1.0 / 3.0);
    } else {
        RTHL = rp;
    }
    if (!(RTHL > 0.0)) { set_no_collapse(out); out->margin = margin; return 5; }

    double RTHL3 = RTHL * RTHL * RTHL;
    double RTHL5 = RTHL3 * RTHL * RTHL;
    double rad3p = rp * rp * rp, rad3 = rm * rm * rm, drad3 = rad3 - rad3p;
    double dFbar = P->Fbar[m0] - P->Fbar[m0 - 1];
    double Fbarx, smat[9], gpk[3], gpkf[3];
    if (zvir1 > 0.0 && drad3 != 0.0) {
        double frac = (RTHL3 - rad3p) / drad3;
        Fbarx = P->Fbar[m0 - 1] + frac * dFbar;
        for (int i = 0; i < 9; ++i) smat[i] = Ebar_last[i] + frac * (strain_mat[i] - Ebar_last[i]);
        for (int i = 0; i < 3; ++i) {
            gpk[i] = gp_last[i] + frac * (gp_prev[i] - gp_last[i]);
            gpkf[i] = gpf_last[i] + frac * (gpf_prev[i] - gpf_last[i]);
        }
    } else {
        Fbarx = P->Fbar[m0 - 1];
        memcpy(smat, Ebar_last, sizeof E);
        memcpy(gpk, gp_prev, sizeof g1); memcpy(gpkf, gpf_prev, sizeof g1);
    }

    /* normalize_strain + eigen (RadialShell.jl:730-734) */
    double tr = smat[0] + smat[4] + smat[8];
    if (tr != 0.0) for (int i = 0; i < 9; ++i) smat[i] *= Fbarx / tr;
    double Frhoc, e_v_f, p_v_f, lamf[3];
    ev_pv(smat, &Frhoc, &e_v_f, &p_v_f, lamf);

    /* strain_mat = Ebar_last * (Fbarx / Frhoh)  (RadialShell.jl:736; the GPU variant
     * guards Frhoh == 0, ShellAnalysisGPU.jl:459) */
    double strain_final[9];
    if (gpu_conv && Frhoh == 0.0) memcpy(strain_final, Ebar_last, sizeof E);
    else for (int i = 0; i < 9; ++i) strain_final[i] = Ebar_last[i] * (Fbarx / Frhoh);

    /* Sbar (RadialShell.jl:739-754) */
    double Sb[3] = {0, 0, 0}, Sb2[3] = {0, 0, 0};
    int64_t nSbar = 0;
    for (int64_t m1 = 1; m1 <= m0 - 1; ++m1)
        if (P->nshell[m1] > 0) {
            for (int L = 0; L < 3; ++L) { Sb[L] += P->S[L][m1]; Sb2[L] += P->S2[L][m1]; }
            nSbar += P->nshell[m1];
        }
    if (nSbar > 0) for (int L = 0; L < 3; ++L) { Sb[L] /= (double)nSbar; Sb2[L] /= (double)nSbar; }

    /* Srb (RadialShell.jl:757-771) */
    double Srb = 0.0, rad5p = 0.0;
    if (m0 > 2)
        for (int64_t mp = 2; mp <= m0 - 1; ++mp) {
            double r = P->rad[mp];
            double rad5 = r * r * r * r * r;
            Srb += 0.5 * (P->Fbar[mp - 1] + P->Fbar[mp]) * (rad5 - rad5p);
            rad5p = rad5;
        }
    if (zvir1 > 0.0 && dZvir != 0.0) Srb += 0.5 * (P->Fbar[m0 - 1] + Fbarx) * (RTHL5 - rad5p);
    if (Fbarx * RTHL5 > 0.0) Srb /= (Fbarx * RTHL5);

    const or_grid* g = W->g;
    const int n1 = g->n1, n2 = g->n2, n3 = g->n3;
    const int64_t s1 = n1, s2 = (int64_t)n1 * n2;
    const int* ipk = W->ipk;
    double d2F = 0.0;
    if (!gpu_conv) {
        /* mask (RadialShell.jl:773-782) */
        if (g->mask)
            for (int64_t jp = 1; jp <= W->npart; ++jp) {
                const or_cell* c = &W->shells[jp - 1];
                if (sqrt((double)c->r2) > RTHL) continue;
                int iv1 = ipk[0] + c->di, iv2 = ipk[1] + c->dj, iv3 = ipk[2] + c->dk;
                if (iv1 < nbuff + 1 || iv1 > n1 - nbuff || iv2 < nbuff + 1 || iv2 > n2 - nbuff ||
                    iv3 < nbuff + 1 || iv3 > n3 - nbuff) continue;
                g->mask[(iv1 - 1) + s1 * (iv2 - 1) + s2 * (iv3 - 1)] = 1;
            }
        /* d2F (RadialShell.jl:785-799): centre excluded, stops at the first
         * out-of-tile cell in shell order */
        if (g->lapd) {
            int64_t navg = 0;
            for (int64_t jp = 2; jp <= W->npart; ++jp) {
                const or_cell* c = &W->shells[jp - 1];
                if (sqrt((double)c->r2) > RTHL) continue;
                int iv1 = ipk[0] + c->di, iv2 = ipk[1] + c->dj, iv3 = ipk[2] + c->dk;
                if (iv1 < 1 || iv1 > n1 || iv2 < 1 || iv2 > n2 || iv3 < 1 || iv3 > n3) break;
                navg += 1;
                d2F += (double)g->lapd[(iv1 - 1) + s1 * (iv2 - 1) + s2 * (iv3 - 1)];
            }
            if (navg > 0) d2F /= (double)navg;
        }
    } else {
        /* d2F and mask over the shell table (ShellAnalysisGPU.jl:496-528) */
        if (g->lapd) {
            int64_t nd2 = 0;
            for (int s = 0; s < W->nshells; ++s) {
                if (sqrt((double)W->st_r2[s]) > RTHL) break;
                for (int32_t c = 0; c < W->st_count[s]; ++c) {
                    const or_cell* cc = &W->shells[W->st_start[s] + c];
                    int iv1 = ipk[0] + cc->di, iv2 = ipk[1] + cc->dj, iv3 = ipk[2] + cc->dk;
                    if (iv1 < 1 || iv1 > n1 || iv2 < 1 || iv2 > n2 || iv3 < 1 || iv3 > n3) continue;
                    d2F += (double)g->lapd[(iv1 - 1) + s1 * (iv2 - 1) + s2 * (iv3 - 1)];
                    nd2 += 1;
                }
            }
            if (nd2 > 0) d2F /= (double)nd2;
        }
        if (g->mask)
            for (int s = 0; s < W->nshells; ++s) {
                if (sqrt((double)W->st_r2[s]) > RTHL) break;
                for (int32_t c = 0; c < W->st_count[s]; ++c) {
                    const or_cell* cc = &W->shells[W->st_start[s] + c];
                    int iv1 = ipk[0] + cc->di, iv2 = ipk[1] + cc->dj, iv3 = ipk[2] + cc->dk;
                    if (iv1 < 1 || iv1 > n1 || iv2 < 1 || iv2 > n2 || iv3 < 1 || iv3 > n3) continue;
                    if (iv1 > nbuff && iv1 <= n1 - nbuff && iv2 > nbuff && iv2 <= n2 - nbuff &&
                        iv3 > nbuff && iv3 <= n3 - nbuff)
                        g->mask[(iv1 - 1) + s1 * (iv2 - 1) + s2 * (iv3 - 1)] = 1;
                }
            }
    }

    /* zvir_half (RadialShell.jl:801-859) */
    double zvir_half = gpu_conv && !zvir ? 0.0 : -1.0;
    if (zvir && RTHL >= 3.0) {
        for (int jj = 1; jj <= 10; ++jj) {
            double rcur = RTHL * pow((jj - 1) / 9.0 * 0.5 + 0.5, 1.0 / 3.0);
            double rupp_rc = rcur + 2.0;
            int64_t mupp_rc = 1;
            for (int64_t m1 = 2; m1 <= m - 1; ++m1) {
                if (P->rad[m1] > rupp_rc) { mupp_rc = m1; break; }
                else if (P->rad[m1] == 0.0) { mupp_rc = m1 - 1; break; }
                mupp_rc = m1;
            }
            double rlow_rc = fmax(rcur - 2.0, 0.0);
            int64_t mlow_rc = 1;
            for (int64_t m1 = 1; m1 <= m - 1; ++m1) if (P->rad[m1] > rlow_rc) { mlow_rc = m1; break; }
            int64_t m0_rc = 1;
            for (int64_t m1 = 1; m1 <= m - 1; ++m1) {
                if (P->rad[m1] > rcur) { m0_rc = m1; break; }
                m0_rc = m1;
            }
            double Eb[9], gp[3], gpf[3];
            kernel_strain(P, m0_rc, mlow_rc, mupp_rc, wRnor, aRnor, Eb, gp, gpf);
            double Frho_rc, e_v_rc, p_v_rc;
            ev_pv(Eb, &Frho_rc, &e_v_rc, &p_v_rc, NULL);
            double Frhoc_rc = P->Fbar[m0_rc];
            double poe_rc = e_v_rc < 1e-5 ? 0.0 : p_v_rc / e_v_rc;
            double zvir_rc = -1.0;
            if (Frhoc_rc > 0.0) zvir_rc = or_interp(ct, log10(Frhoc_rc), e_v_rc, poe_rc);
            if (zvir_rc - 1.0 > zvir_half) zvir_half = zvir_rc - 1.0;
        }
    }

    out->RTHL = RTHL; out->Srb = Srb; out->Fbarx = Fbarx; out->e_v = e_v_f; out->p_v = p_v_f;
    out->zvir_half = zvir_half; out->d2F = d2F;
    for (int i = 0; i < 3; ++i) {
        out->Sbar[i] = Sb[i]; out->Sbar2[i] = Sb2[i]; out->gradpk[i] = gpk[i];
        out->gradpkf[i] = gpkf[i]; out->gradpkrf[i] = gradpkrf[i]; out->eigs[i] = lamf[i];
    }
    memcpy(out->strain, strain_final, sizeof strain_final);
    out->margin = margin;
    return 0;
}

/* RadialShell.jl:281-865 */
int or_analyse_peak(const or_grid* g, int64_t ipp, double alatt, int ir2min, double ZZon,
                    double Rfclvi, const or_ctab* ct, const or_cell* shells, int64_t nshellcells,
                    int nbuff, double rmax2rs, double fcrit_in, or_result* out)
{
    int64_t npartmax = nshellcells, npart;
    if (rmax2rs > 0.0) {
        double x = rmax2rs * Rfclvi / alatt;
        int64_t v = (int64_t)floor(4.0 / 3.0 * PI_D * (x * x * x));
        npart = v < npartmax ? v : npartmax;
    } else {
        npart = npartmax;
    }
    const int n1 = g->n1, n2 = g->n2, n3 = g->n3;
    const int64_t s1 = n1, s2 = (int64_t)n1 * n2;
    int ipk[3];
    ipk[2] = (int)((ipp - 1) / s2 + 1);
    ipk[1] = (int)(((ipp - 1) % s2) / n1 + 1);
    ipk[0] = (int)((ipp - 1) % n1 + 1);
    const int64_t cpk = (ipk[0] - 1) + s1 * (ipk[1] - 1) + s2 * (ipk[2] - 1);

    if (rmax2rs > 0.0 && g->mask) {
        if ((int64_t)g->mask[cpk] > (int64_t)floor(Rfclvi / alatt * rmax2rs)) {
            set_no_collapse(out); return 1;
        }
    }
    double fcrit = fcrit_in >= 0.0 ? fcrit_in : or_fsc_of_z(ZZon - 1.0, ct);
    if (npart < 2) { set_no_collapse(out); return 4; }

    /* The reference sizes its profile arrays npart + 2 (RadialShell.jl:318); m never
     * exceeds the number of distinct r^2 among the first npart cells, so that bound is
     * used here (same values, smaller allocation). */
    int64_t nsh_part = 1;
    for (int64_t jp = 1; jp < npart; ++jp)
        if (shells[jp].r2 != shells[jp - 1].r2) ++nsh_part;
    int64_t maxm = nsh_part + 2;
    prof_t P;
    prof_alloc(&P, maxm);
    int64_t m = 1, m0 = 1;
    P.rad[1] = 0.0;
    P.Fbar[1] = (double)g->delta[cpk];
    P.nshell[1] = 1;
    const int ilpt2 = g->eta2x != NULL;
    P.S[0][1] = g->etax[cpk]; P.S[1][1] = g->etay[cpk]; P.S[2][1] = g->etaz[cpk];
    if (ilpt2) { P.S2[0][1] = g->eta2x[cpk]; P.S2[1][1] = g->eta2y[cpk]; P.S2[2][1] = g->eta2z[cpk]; }
    /* slots 2 are already zero (calloc), as RadialShell.jl:347-360 sets them */

    double Fshell = 0.0;
    int64_t nsh = 0;
    int32_t ir2p = shells[1].r2;
    double dFbarp = P.Fbar[1];
    double rupp_init = sqrt((double)ir2min) + 2.0;
    int ifcrit = 1;
    int64_t mupp = 1;

    for (int64_t jp = 2; jp <= npart; ++jp) {
        const or_cell* c = &shells[jp - 1];
        int32_t ir2 = c->r2;
        if (ir2 != ir2p) {
            m += 1;
            P.rad[m] = sqrt((double)ir2p);
            P.nshell[m] = nsh;
            double dFbar = nsh > 0 ? Fshell / (double)nsh : 0.0;
            double rad3p = P.rad[m - 1] * P.rad[m - 1] * P.rad[m - 1];
            double rad3 = P.rad[m] * P.rad[m] * P.rad[m];
            P.Fbar[m] = (rad3p * P.Fbar[m - 1] + 0.5 * (dFbarp + dFbar) * (rad3 - rad3p)) / rad3;
            dFbarp = dFbar;
            if (ifcrit == 1) {
                m0 = m;
                if (ir2p > ir2min) {
                    rupp_init = P.rad[m0] + 2.0;
                    ifcrit = 0;
                    mupp = m;
                }
            } else {
                if (P.rad[m] < rupp_init) mupp = m;
            }
            ir2p = ir2;
            Fshell = 0.0;
            nsh = 0;
            for (int L = 0; L < 3; ++L) {
                P.S[L][m + 1] = 0.0; P.S2[L][m + 1] = 0.0;
                P.G[L][m] /= P.rad[m]; P.Gf[L][m] /= P.rad[m];
                P.G[L][m + 1] = 0.0; P.Gf[L][m + 1] = 0.0;
                for (int K = 0; K < 3; ++K) { P.SR[L][K][m] /= P.rad[m]; P.SR[L][K][m + 1] = 0.0; }
            }
        }
        int iv1 = ipk[0] + c->di, iv2 = ipk[1] + c->dj, iv3 = ipk[2] + c->dk;
        if (iv1 < 1 || iv1 > n1 || iv2 < 1 || iv2 > n2 || iv3 < 1 || iv3 > n3) continue;
        nsh += 1;
        int64_t cv = (iv1 - 1) + s1 * (iv2 - 1) + s2 * (iv3 - 1);
        float dv = g->delta[cv];
        Fshell += (double)dv;
        float ev[3] = {g->etax[cv], g->etay[cv], g->etaz[cv]};
        float e2[3] = {0.f, 0.f, 0.f};
        if (ilpt2) { e2[0] = g->eta2x[cv]; e2[1] = g->eta2y[cv]; e2[2] = g->eta2z[cv]; }
        float dT = g->delta[(iv3 - 1) + s1 * (iv1 - 1) + s2 * (iv2 - 1)];
        const int32_t ix[3] = {c->di, c->dj, c->dk};
        for (int L = 0; L < 3; ++L) {
            P.S[L][m + 1] += (double)ev[L];
            P.S2[L][m + 1] += (double)e2[L];
            P.G[L][m + 1] += cell_product(dv, ix[L]);
            P.Gf[L][m + 1] += cell_product(dT, ix[L]);
            for (int K = 0; K < 3; ++K) P.SR[L][K][m + 1] += cell_product(ev[L], ix[K]);
        }
    }

    /* mrf (RadialShell.jl:449-464), per cell with the lagging counter */
    double rmrf = 10.0;
    int64_t mrf = 1;
    int32_t ir2p_rf = shells[1].r2;
    int64_t mrfi = 1;
    const double R2 = (Rfclvi / alatt) * (Rfclvi / alatt);
    for (int64_t jp = 2; jp <= npart; ++jp) {
        int32_t ir2 = shells[jp - 1].r2;
        double d = fabs((double)ir2 - R2);
        if (d < rmrf) { mrf = mrfi; rmrf = fmin(rmrf, d); }
        if (ir2 != ir2p_rf) { mrfi += 1; ir2p_rf = ir2; }
    }

    walk_ctx W;
    memset(&W, 0, sizeof W);
    W.g = g; W.ipk[0] = ipk[0]; W.ipk[1] = ipk[1]; W.ipk[2] = ipk[2];
    W.shells = shells; W.npart = npart;
    int code = tail(&W, &P, m, m0, mupp, mrf, alatt, ZZon, fcrit, ct, nbuff, 0, 1, out);
    prof_free(&P);
    return code;
}

/* ShellAnalysisGPU.jl:81-535 (conv 0) / reference CUDA kernels (conv 1), with the shell
 * tables already grouped. */
static int analyse_gpu_impl(const or_grid* g, int64_t ipp, double alatt, int ir2min,
                            double ZZon, double Rfclvi, const or_ctab* ct,
                            const or_cell* shells, int64_t nshellcells,
                            const int64_t* st_start, const int32_t* st_count,
                            const int32_t* st_r2, int nshells, int nbuff, double rmax2rs,
                            double fcrit_in, int conv, or_result* out)
{
    int64_t nshells_max = nshells - 1;
    if (rmax2rs > 0.0) {
        double lim = rmax2rs * Rfclvi / alatt;
        double r2_limit = lim * lim;
        nshells_max = 0;
        for (int s = 1; s <= nshells - 1; ++s) {
            if (!((double)st_r2[s - 1] <= r2_limit)) break;
            nshells_max = s;
        }
    }
    int code = 0;
    if (nshells_max < 2) { set_no_collapse(out); return 4; }

    {
        const int n1 = g->n1, n2 = g->n2, n3 = g->n3;
        const int64_t s1 = n1, s2 = (int64_t)n1 * n2;
        int ipk[3];
        ipk[2] = (int)((ipp - 1) / s2 + 1);
        ipk[1] = (int)(((ipp - 1) % s2) / n1 + 1);
        ipk[0] = (int)((ipp - 1) % n1 + 1);
        const int64_t cpk = (ipk[0] - 1) + s1 * (ipk[1] - 1) + s2 * (ipk[2] - 1);
        if (conv == 0 && rmax2rs > 0.0 && g->mask) {
            if ((int64_t)g->mask[cpk] > (int64_t)floor(Rfclvi / alatt * rmax2rs)) {
                set_no_collapse(out); return 1;
            }
        }
        double fcrit = fcrit_in >= 0.0 ? fcrit_in : or_fsc_of_z(ZZon - 1.0, ct);
        const int ilpt2 = g->eta2x != NULL;
        prof_t P;
        prof_alloc(&P, nshells_max + 2);
        int64_t m = 1;
        P.rad[1] = 0.0;
        P.Fbar[1] = (double)g->delta[cpk];
        P.nshell[1] = 1;
        P.S[0][1] = g->etax[cpk]; P.S[1][1] = g->etay[cpk]; P.S[2][1] = g->etaz[cpk];
        if (ilpt2) { P.S2[0][1] = g->eta2x[cpk]; P.S2[1][1] = g->eta2y[cpk]; P.S2[2][1] = g->eta2z[cpk]; }
        double dFbarp = P.Fbar[1];
        int64_t m0 = 1, mupp = 1;
        int ifcrit = 1;
        double rupp_init = sqrt((double)ir2min) + 2.0;
        int first_shell = st_r2[0] == 0 ? 2 : 1;
        for (int64_t s = first_shell; s <= nshells_max; ++s) {
            int32_t r2 = st_r2[s - 1];
            double Fshell = 0.0, lS[3] = {0, 0, 0}, lS2[3] = {0, 0, 0}, lG[3] = {0, 0, 0},
                   lGf[3] = {0, 0, 0}, lSR[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
            int64_t nsh = 0;
            for (int32_t c = 0; c < st_count[s - 1]; ++c) {
                const or_cell* cc = &shells[st_start[s - 1] + c];
                int iv1 = ipk[0] + cc->di, iv2 = ipk[1] + cc->dj, iv3 = ipk[2] + cc->dk;
                if (iv1 < 1 || iv1 > n1 || iv2 < 1 || iv2 > n2 || iv3 < 1 || iv3 > n3) continue;
                nsh += 1;
                int64_t cv = (iv1 - 1) + s1 * (iv2 - 1) + s2 * (iv3 - 1);
                float dv = g->delta[cv];
                Fshell += (double)dv;
                float ev[3] = {g->etax[cv], g->etay[cv], g->etaz[cv]};
                float dT = g->delta[(iv3 - 1) + s1 * (iv1 - 1) + s2 * (iv2 - 1)];
                const int32_t ix[3] = {cc->di, cc->dj, cc->dk};
                for (int L = 0; L < 3; ++L) {
                    lS[L] += (double)ev[L];
                    if (ilpt2) {
                        float e2 = L == 0 ? g->eta2x[cv] : L == 1 ? g->eta2y[cv] : g->eta2z[cv];
                        lS2[L] += (double)e2;
                    }
                    lG[L] += cell_product(dv, ix[L]);
                    lGf[L] += cell_product(dT, ix[L]);
                    for (int K = 0; K < 3; ++K) lSR[L][K] += cell_product(ev[L], ix[K]);
                }
            }
            m += 1;
            P.rad[m] = sqrt((double)r2);
            P.nshell[m] = nsh;
            double dFbar = nsh > 0 ? Fshell / (double)nsh : 0.0;
            double rad3p = P.rad[m - 1] * P.rad[m - 1] * P.rad[m - 1];
            double rad3 = P.rad[m] * P.rad[m] * P.rad[m];
            P.Fbar[m] = (rad3p * P.Fbar[m - 1] + 0.5 * (dFbarp + dFbar) * (rad3 - rad3p)) / rad3;
            dFbarp = dFbar;
            if (ifcrit == 1) {
                m0 = m;
                if (r2 > ir2min) { rupp_init = P.rad[m0] + 2.0; ifcrit = 0; mupp = m; }
            } else {
                if (P.rad[m] < rupp_init) mupp = m;
            }
            for (int L = 0; L < 3; ++L) {
                P.S[L][m] = lS[L]; P.S2[L][m] = lS2[L];
                P.G[L][m] = lG[L] / P.rad[m]; P.Gf[L][m] = lGf[L] / P.rad[m];
                for (int K = 0; K < 3; ++K) P.SR[L][K][m] = lSR[L][K] / P.rad[m];
            }
        }
        /* mrf (ShellAnalysisGPU.jl:234-254): the counter lags the shell index by one */
        double rmrf = 10.0;
        int64_t mrf = 1, mrfi = 1;
        const double R2 = (Rfclvi / alatt) * (Rfclvi / alatt);
        int64_t send = nshells_max < nshells ? nshells_max : nshells;
        for (int64_t s = (st_r2[0] == 0 ? 2 : 1); s <= send; ++s) {
            int32_t r2 = st_r2[s - 1];
            for (int32_t c = 0; c < st_count[s - 1]; ++c) {
                double d = fabs((double)r2 - R2);
                if (d < rmrf) { mrf = mrfi; rmrf = d; }
            }
            if (s < send && st_r2[s] != r2) mrfi += 1;
        }
        walk_ctx W;
        memset(&W, 0, sizeof W);
        W.g = g; W.ipk[0] = ipk[0]; W.ipk[1] = ipk[1]; W.ipk[2] = ipk[2];
        W.shells = shells; W.npart = nshellcells;
        W.st_start = st_start; W.st_count = st_count; W.st_r2 = st_r2; W.nshells = nshells;
        W.nshells_max = nshells_max;
        code = tail(&W, &P, m, m0, mupp, mrf, alatt, ZZon, fcrit, ct, nbuff, 1, conv == 1, out);
        prof_free(&P);
    }
    return code;
}

static int count_shells(const or_cell* shells, int64_t nshellcells)
{
    int cap = 0;
    int64_t i = 0;
    while (i < nshellcells) {
        int32_t rr = shells[i].r2;
        while (i < nshellcells && shells[i].r2 == rr) ++i;
        ++cap;
    }
    return cap;
}

int or_analyse_peak_gpu(const or_grid* g, int64_t ipp, double alatt, int ir2min, double ZZon,
                        double Rfclvi, const or_ctab* ct, const or_cell* shells,
                        int64_t nshellcells, int nbuff, double rmax2rs, double fcrit_in,
                        int conv, or_result* out)
{
    int cap = count_shells(shells, nshellcells);
    int64_t* st_start = (int64_t*)malloc(sizeof(int64_t) * (size_t)cap);
    int32_t* st_count = (int32_t*)malloc(sizeof(int32_t) * (size_t)cap);
    int32_t* st_r2 = (int32_t*)malloc(sizeof(int32_t) * (size_t)cap);
    int nshells = or_build_shell_tables(shells, nshellcells, st_start, st_count, st_r2, cap);
    int code = analyse_gpu_impl(g, ipp, alatt, ir2min, ZZon, Rfclvi, ct, shells, nshellcells,
                                st_start, st_count, st_r2, nshells, nbuff, rmax2rs, fcrit_in,
                                conv, out);
    free(st_start); free(st_count); free(st_r2);
    return code;
}

void or_analyse_batch(const or_grid* g, int64_t npeaks, const int32_t* pi, const int32_t* pj,
                      const int32_t* pk, const int32_t* ir2min, const double* Rf,
                      const double* ZZon, const double* fcrit, double alatt,
                      const or_ctab* ct, const or_cell* shells, int64_t nshellcells,
                      int nbuff, double rmax2rs, int kind, or_result* out, int32_t* codes,
                      int nthreads)
{
    (void)akk_table();
    const int64_t n1 = g->n1, n2 = g->n2;
    int cap = count_shells(shells, nshellcells);
    int64_t* st_start = (int64_t*)malloc(sizeof(int64_t) * (size_t)cap);
    int32_t* st_count = (int32_t*)malloc(sizeof(int32_t) * (size_t)cap);
    int32_t* st_r2 = (int32_t*)malloc(sizeof(int32_t) * (size_t)cap);
    int nshells = or_build_shell_tables(shells, nshellcells, st_start, st_count, st_r2, cap);
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
#endif
    for (int64_t p = 0; p < npeaks; ++p) {
        int64_t ipp = (int64_t)pi[p] + (int64_t)(pj[p] - 1) * n1 + (int64_t)(pk[p] - 1) * n1 * n2;
        int c;
        if (kind == 0)
            c = or_analyse_peak(g, ipp, alatt, ir2min[p], ZZon[p], Rf[p], ct, shells, nshellcells,
                                nbuff, rmax2rs, fcrit[p], &out[p]);
        else
            c = analyse_gpu_impl(g, ipp, alatt, ir2min[p], ZZon[p], Rf[p], ct, shells,
                                 nshellcells, st_start, st_count, st_r2, nshells, nbuff,
                                 rmax2rs, fcrit[p], kind == 2 ? 1 : 0, &out[p]);
        if (codes) codes[p] = c;
    }
    free(st_start); free(st_count); free(st_r2);
}

int or_max_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
