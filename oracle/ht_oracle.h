/*
 * CPU oracle for the halo-finding hot path (peak finding + radial-shell collapse).
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C, FP64 restatement of the reference
 * algorithm (guanyilun/Huntian.jl) used as the checker for the CUDA library and as the
 * timed CPU baseline.  Nothing in the product library links or calls it.
 *
 * Every function cites the reference file:line it restates.  Arrays are 1-based in the
 * comments (Julia convention); the C code uses 0-based storage with explicit offsets.
 * Fields are column-major (i fastest), FP32, as in the reference.
 */
#ifndef HT_ORACLE_H
#define HT_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* One lattice offset of the shell list (RadialShell.jl:34-39). */
typedef struct { int32_t di, dj, dk, r2; } or_cell;

/* All offsets with r2 <= rmax^2, generated dk-outer/dj/di-inner and stable-sorted by r2
 * (RadialShell.jl:151-166).  Returns the count; writes at most `cap` cells. */
int64_t or_precompute_shells(int rmax, or_cell* out, int64_t cap);

/* Group sorted cells into shells (ShellAnalysisGPU.jl:44-71).  start is 0-based. */
int or_build_shell_tables(const or_cell* cells, int64_t ncells,
                          int64_t* start, int32_t* count, int32_t* r2, int cap);

double or_hRinteg(double u0, double u12);               /* RadialShell.jl:95-121 */
void   or_atab4(double out[1101]);                      /* RadialShell.jl:125-142 */

/* Collapse table (CollapseTable.jl:96-138): Float32 (nx,ny,nz) column-major on regular
 * axes; trilinear inside the closed box, out_val outside. */
typedef struct {
    const float* table; int nx, ny, nz;
    double x1, x2, y1, y2, z1, z2;
    double out_val;
} or_ctab;
double or_interp(const or_ctab* ct, double x, double y, double z);
double or_fsc_of_z(double z, const or_ctab* ct);         /* RadialShell.jl:181-195 */

/* Ascending eigenvalues of a symmetric 3x3 matrix (column-major a[9]); cyclic Jacobi in
 * FP64, standing in for LAPACK eigvals(Symmetric) (RadialShell.jl:215-220). */
void or_eigvals_sym3(const double a[9], double lam[3]);

/* PeakFind.find_peaks (PeakFind.jl:15-78).  Appends up to max_peaks peaks in k/j/i scan
 * order, sets mask=1 at each.  Outputs are 1-based i,j,k and the flat 1-based ipp.
 * Returns the number of peaks written. */
int64_t or_find_peaks(const float* delta, int8_t* mask, int n1, int n2, int n3,
                      int nbuff, float fcrit, int64_t max_peaks,
                      int32_t* out_i, int32_t* out_j, int32_t* out_k, float* out_delta);

/* Fields of one tile (RadialShell.jl:41-52).  eta2*, mask, lapd may be NULL. */
typedef struct {
    const float *delta, *etax, *etay, *etaz, *eta2x, *eta2y, *eta2z;
    int8_t* mask;
    const float* lapd;
    int n1, n2, n3;
} or_grid;

/* PeakResult (RadialShell.jl:54-90) plus the eigenvalues the GPU entry returns
 * (ext/CUDAExt.jl:1904-1906).  strain is column-major 3x3. */
typedef struct {
    double RTHL, Srb, Sbar[3], Sbar2[3], strain[9], gradpk[3], gradpkrf[3];
    double Fbarx, e_v, p_v, zvir_half, gradpkf[3], d2F, eigs[3];
    /* diagnostic, not a reference output: the smallest |Fbar - fcrit| or |zvir - ZZon|
     * over the comparisons that decided the collapse (infinity when none did) */
    double margin;
} or_result;

/* RadialShell.analyse_peak (RadialShell.jl:281-865), literal: per-cell shell walk, FP64.
 * fcrit < 0 means "use fsc_of_z(ZZon-1)".  Returns a reject code (0 = collapsed,
 * 1 premask, 2 no fcrit crossing, 3 m0==1, 4 no collapse, 5 RTHL<=0). */
int or_analyse_peak(const or_grid* g, int64_t ipp, double alatt, int ir2min, double ZZon,
                    double Rfclvi, const or_ctab* ct, const or_cell* shells, int64_t nshellcells,
                    int nbuff, double rmax2rs, double fcrit, or_result* out);

/* ShellAnalysisGPU.analyse_peak_gpu (ShellAnalysisGPU.jl:81-535): per-shell gather.
 * conv = 0: literal (zvir_half = 0).
 * conv = 1: semantics of the reference CUDA post-process kernel
 *           (ext/CUDAExt.jl:1213-1912): zvir_half computed as RadialShell.jl:801-859,
 *           eigs output, no premask. */
int or_analyse_peak_gpu(const or_grid* g, int64_t ipp, double alatt, int ir2min, double ZZon,
                        double Rfclvi, const or_ctab* ct, const or_cell* shells,
                        int64_t nshellcells, int nbuff, double rmax2rs, double fcrit,
                        int conv, or_result* out);

/* Many peaks at once on all host threads (OpenMP).  kind: 0 = or_analyse_peak,
 * 1 = or_analyse_peak_gpu(conv 0), 2 = or_analyse_peak_gpu(conv 1).  Per-peak
 * ir2min/Rf/ZZon/fcrit arrays.  Mask writes are idempotent (value 1). */
void or_analyse_batch(const or_grid* g, int64_t npeaks, const int32_t* pi, const int32_t* pj,
                      const int32_t* pk, const int32_t* ir2min, const double* Rf,
                      const double* ZZon, const double* fcrit, double alatt,
                      const or_ctab* ct, const or_cell* shells, int64_t nshellcells,
                      int nbuff, double rmax2rs, int kind, or_result* out, int32_t* codes,
                      int nthreads);

int or_max_threads(void);

/* 0 (default): cell products rounded to Float32 as the reference forms them; 1: products
 * formed exactly in Float64 (the full-FP64 oracle).  Process-wide; set it between calls. */
void or_set_exact_products(int on);

/* ---- collapse-table generation (or_collapse.c) ---- */

/* DlinearTables (Cosmology.jl:68-78): D(a)/a and dlnD/dlna on an ascending table of a. */
typedef struct {
    const double* atab; const double* D_atab; const double* dlnD; int ntab;
    double amintab, amaxtab, D_ainfty, D_a0, HD_Hainfty, HD_Ha0;
} or_growth;

/* EllipsoidParams (EllipsoidalCollapse.jl:10-45) with its cosmology (Om, OL). */
typedef struct {
    double Om, OL;
    int iforce_strat, ivir_strat;
    double fcoll[3];          /* fcoll_1, fcoll_2, fcoll_3 */
    double tfac;
    int nstepmax;
    double zinit_fac;
    or_growth growth;
    int solver;               /* 0: the fixed-step RK4 (:rk4); 1: adaptive Tsit5 (:diffeq) */
} or_ellipsoid;

void   or_dlinear_ab(const or_growth* g, double ai, double* dlin, double* hd_ha);
double or_dfnofa(const or_growth* g, double ai);
double or_elliptic_rd(double x, double y, double z);
void   or_get_b_2(double a1, double a2, double a3, double b[3]);
int    or_evolve_ellipse(const or_ellipsoid* ep, double Frho, double e_v, double p_v,
                         int idynax, double out[3]);
double or_pow_pos(double x, double y);
void   or_make_table(const or_ellipsoid* ep, int nx, int ny, int nz, double X1, double X2,
                     double Y1, double Y2, double Z1, double Z2, float* table);

#ifdef __cplusplus
}
#endif
#endif
