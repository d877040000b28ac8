// Radial-shell collapse on sm_100a.
//
// A peak is handled by a group of G = 8 lanes of one warp (four peaks share a warp; on
// the benchmark tiles this beat 32 lanes per peak for the long walks as well as for the
// short ones).  For each peak the group walks the shells of the r^2-sorted offset table
// outward (the per-shell gather of ShellAnalysisGPU.jl:153-229 / ext/CUDAExt.jl:752-924):
// each lane accumulates 13 sums per shell in FP64 from the FP32 cell values (delta,
// delta*d, delta^T*d, and the symmetrised strain psi_L d_K + psi_K d_L, every product
// exact in FP64); the lanes' partial sums are combined in FP64 in a fixed order through
// shared memory, and the shell's profile (Fbar, gradients, strain) goes to a per-group
// scratch slot in FP64.  The walk stops as
// soon as every shell the post-processing reads has been gathered.  The same group then
// runs the post-processing of RadialShell.jl:449-859 / ext/CUDAExt.jl:1213-1912 in FP64:
// fcrit crossing, the inward strain/eigen/barrier walk (G steps evaluated at once, one per
// lane), RTHL interpolation, Sbar and the mask update (one second pass over the cells within
// the collapsed radius), Srb, d2F and zvir_half.  The SPH window weights of
// kernel_strain depend only on the two shell radii, so they come from a table built once
// per context.
//
// Two execution modes give identical results:
//   PLAIN   reads the eight reference fields separately, static item->warp schedule;
//   BATCHED reads 32-byte interleaved cell records (one sector per cell) built by
//           pack_kernel, persistent grid with a dynamic work queue.
#include <math.h>
#include <string.h>

#include <mutex>
#include <string>

#include <cub/device/device_radix_sort.cuh>

#include "ht_internal.cuh"

namespace {

constexpr int kWarpsPerBlock = 8;
constexpr int kThreads = kWarpsPerBlock * 32;
constexpr int kRec = 16;          // doubles per shell in the scratch profile
constexpr int kSmallG = 8;        // lanes per peak
constexpr int kPeaksPerItem = 32 / kSmallG;  // peaks per work item (one per group)

// Scratch profile record, one per shell m (1-based); rows are 128-byte aligned, and the
// twelve values the SPH window sums read (G, Gf, SR) fill the last 96 bytes, so that they
// come in three 256-bit loads:
enum : int {
    P_FBAR = 0,
    P_CSRB = 1,   // running Srb numerator, RadialShell.jl:760-764
    P_G = 4,      // 3: Gshell / rad
    P_GF = 7,     // 3: Gshellf / rad
    P_SR = 10,    // 6: (SR_LK + SR_KL) / rad for 11, 22, 33, 12, 13, 23
};
static_assert(P_GF == P_G + 3 && P_SR == P_G + 6 && P_SR + 6 == kRec && P_G % 4 == 0,
              "G, Gf, SR: twelve contiguous doubles on a 32-byte boundary at the row's end");

// Per-cell sums gathered for every shell.
enum : int { V_F = 0, V_N = 1, V_G = 2, V_GF = 5, V_SR = 8, V_ROWS = 14 };

// Shared-memory staging per group: [V_ROWS][G + 1] doubles for the shell sums (the last
// column holds the totals), or [G + 1][kStepW] doubles for inward-walk steps.
constexpr int kStepW = 14;
__host__ __device__ constexpr int group_smem_doubles(int G) {
    return V_ROWS * (G + 1) > (G + 1) * kStepW ? V_ROWS * (G + 1) : (G + 1) * kStepW;
}
constexpr int kWarpSmemDoubles = kPeaksPerItem * group_smem_doubles(kSmallG);

struct WalkArgs {
    const float4* rec;
    const float* delta;
    const float* ex;
    const float* ey;
    const float* ez;
    const float* e2x;
    const float* e2y;
    const float* e2z;
    const float* lapd;
    int n1, n2, n3;
    long long s2;

    const char4* off;
    const int2* cell;       // nullable: (linear offset n1-n2-n3 of the bound tile, char4 bits)
    int nhunt;              // largest |d| of any table offset
    const int32_t* start;
    const int32_t* count;
    const int32_t* r2;
    const double* rad;
    const double* irad;     // 1 / rad (0 for the centre shell)
    const double* irad3;    // 1 / rad^3
    int nshells;
    const int32_t* wrow;   // SPH weight table: row mp = entries [wrow[mp], wrow[mp+1])
    const double2* wpk;    // entry: (weight, m1)

    const float* ct;
    int nx, ny, nz;
    double X1, X2, Y1, Y2, Z1, Z2, out_val;
    const double* akk;

    const int32_t* pi;
    const int32_t* pj;
    const int32_t* pk;
    const double* Rf;
    const int32_t* ir2min;
    const float* ZZon;
    const float* fcrit;
    long long npeaks;
    const int32_t* order;   // nullable processing order
    const int4* bounds;     // nullable per-peak Bounds (m, m0_init, mrf, need_rf)

    double alatt, wRnor, aRnor, rmax2rs;
    double zh_frac[10];     // cbrt(0.5 + 0.5 jj / 9), jj = 0..9 (zvir_half radii)
    int nbuff;
    int conv;
    int block_bits;         // LEARNED order: Morton block of 2^block_bits cells
    int8_t* mask;
    ht_results out;

    double* scratch;        // one slot of scratch_stride doubles per group
    long long scratch_stride;
    int32_t* queue;
    int dynamic;
    unsigned long long* stats;
    unsigned long long* reject;   // nullable: the context's HT_REJECT_* counters
    int32_t* status;              // the context's status word (HT_CHECKED index checks)
    long long ntile;              // n1 n2 n3: cells of the bound tile
    long long ncells;             // entries of the offset and cell tables
};

// ------------------------------------------------------------ small helpers ----

// Per-lane FP64 accumulator.  The gathered values are FP32 and the offsets small
// integers, so every product below is exact in FP64 and each step rounds once; the gather
// is latency bound, so the FP64 pipe has room for it (FP32 Kahan sums were measured to
// leave up to 4e-6 relative error on ill-conditioned strain traces, which FP64 removes).
struct Acc {
    double s;
    __device__ __forceinline__ void zero() { s = 0.0; }
    __device__ __forceinline__ void add(float x) { s += (double)x; }
    __device__ __forceinline__ void add_prod(float x, float y) {
        s = fma((double)x, (double)y, s);
    }
    __device__ __forceinline__ double value() const { return s; }
};

// Largest m in [lo, hi] with rad[m] < x, or lo - 1 if none (rad ascending).
__device__ __forceinline__ int last_below(const double* rad, int lo, int hi, double x) {
    int a = lo, b = hi, ans = lo - 1;
    while (a <= b) {
        int mid = (a + b) >> 1;
        if (rad[mid] < x) { ans = mid; a = mid + 1; } else { b = mid - 1; }
    }
    return ans;
}

// Largest m in [lo, hi] with rad[m] <= x, or lo - 1 if none.
__device__ __forceinline__ int last_le(const double* rad, int lo, int hi, double x) {
    int a = lo, b = hi, ans = lo - 1;
    while (a <= b) {
        int mid = (a + b) >> 1;
        if (rad[mid] <= x) { ans = mid; a = mid + 1; } else { b = mid - 1; }
    }
    return ans;
}

// Smallest m in [lo, hi] with rad[m] > x, or hi + 1 if none.
__device__ __forceinline__ int first_above(const double* rad, int lo, int hi, double x) {
    int a = lo, b = hi, ans = hi + 1;
    while (a <= b) {
        int mid = (a + b) >> 1;
        if (rad[mid] > x) { ans = mid; b = mid - 1; } else { a = mid + 1; }
    }
    return ans;
}

// G lanes of one warp working on one peak.
struct Group {
    int G, t, q;
    unsigned mask;
    __device__ __forceinline__ unsigned ballot(bool p) const {
        const unsigned b = __ballot_sync(mask, p) >> (q * G);
        return G == 32 ? b : (b & ((1u << G) - 1u));
    }
    __device__ __forceinline__ void sync() const { __syncwarp(mask); }
    __device__ __forceinline__ double sum(double x) const {
        for (int o = G >> 1; o >= 1; o >>= 1) x += __shfl_xor_sync(mask, x, o, G);
        return x;
    }
};

struct Strain {
    double E[6];   // 11, 22, 33, 12, 13, 23
    double g[3];
    double gf[3];
};

// kernel_strain (RadialShell.jl:225-274) centred on shell mp over the shells m1 of its
// weight-table row with lo <= m1 <= hi, in FP64.  The row of mp > 1 lists the shells
// with (rad[mp] - rad[m1])^2 < 4 and hRinteg(u0, u12) / (u12 - u0^2)^2 as weight; the
// row of mp = 1 lists shells 2..U(1) with the atab4 weight 0.5 * W / rad[m1].  The
// weighted sums are scaled by wRnor / rad[mp] (mp > 1) or aRnor (mp = 1) at the end, in
// the reference's order.
// The twelve window values (G, Gf, SR) of a profile row in three 256-bit loads.  The rows
// were written by the group's lanes before the post-processing began (the group synced
// since), and this is the only access to them in the caller's loop.
__device__ __forceinline__ void load_row12(const double* q, double (&r)[12]) {
    const double* b = q + P_G;
    asm volatile("ld.global.v4.f64 {%0,%1,%2,%3}, [%4];"
                 : "=d"(r[0]), "=d"(r[1]), "=d"(r[2]), "=d"(r[3]) : "l"(b));
    asm volatile("ld.global.v4.f64 {%0,%1,%2,%3}, [%4];"
                 : "=d"(r[4]), "=d"(r[5]), "=d"(r[6]), "=d"(r[7]) : "l"(b + 4));
    asm volatile("ld.global.v4.f64 {%0,%1,%2,%3}, [%4];"
                 : "=d"(r[8]), "=d"(r[9]), "=d"(r[10]), "=d"(r[11]) : "l"(b + 8));
}

__device__ __noinline__ Strain kernel_strain(const int32_t* __restrict__ wrow,
                                             const double2* __restrict__ wpk,
                                             const double* __restrict__ rad, double wRnor,
                                             double aRnor, const double* __restrict__ P,
                                             int mp, int lo, int hi) {
    Strain s;
#pragma unroll
    for (int i = 0; i < 6; ++i) s.E[i] = 0.0;
#pragma unroll
    for (int i = 0; i < 3; ++i) { s.g[i] = 0.0; s.gf[i] = 0.0; }
    const int e0 = __ldg(wrow + mp), e1 = __ldg(wrow + mp + 1);
    for (int e = e0; e < e1; ++e) {
        const double2 we = __ldg(wpk + e);
        const int m1 = (int)we.y;
        if (m1 > hi) break;
        if (m1 < lo) continue;
        const double wt = we.x;
        const double hw = 0.5 * wt;
        double r[12];
        load_row12(P + (size_t)m1 * kRec, r);
#pragma unroll
        for (int L = 0; L < 3; ++L) {
            s.g[L] += wt * r[L];
            s.gf[L] += wt * r[3 + L];
        }
#pragma unroll
        for (int i = 0; i < 6; ++i) s.E[i] -= hw * r[6 + i];
    }
    const double scale = mp > 1 ? wRnor / rad[mp] : aRnor;
#pragma unroll
    for (int i = 0; i < 6; ++i) s.E[i] *= scale;
#pragma unroll
    for (int i = 0; i < 3; ++i) { s.g[i] *= scale; s.gf[i] *= scale; }
    return s;
}

// kernel_strain's central branch over shells lo..hi computed directly (used for the
// gradient at the filter scale when mrf = 1, whose window starts at the centre shell:
// its weight 0.5 * W(0) / 0 is infinite and the reference's gradient is NaN).
__device__ __noinline__ Strain kernel_strain_central(const double* __restrict__ rad,
                                                     const double* __restrict__ akk,
                                                     double aRnor,
                                                     const double* __restrict__ P, int lo,
                                                     int hi) {
    Strain s;
#pragma unroll
    for (int i = 0; i < 6; ++i) s.E[i] = 0.0;
#pragma unroll
    for (int i = 0; i < 3; ++i) { s.g[i] = 0.0; s.gf[i] = 0.0; }
    for (int m1 = lo; m1 <= hi; ++m1) {
        const double r1 = rad[m1];
        const double con = 100.0 * r1 * r1;
        const double fl = floor(con);
        const int icon = (int)fl;
        const double diff = con - fl;
        double aww = 0.0;
        if (icon >= 0 && icon < 1100) aww = akk[icon] + diff * (akk[icon + 1] - akk[icon]);
        const double wt = 0.5 * aww / r1;
        const double hw = 0.5 * wt;
        double r[12];
        load_row12(P + (size_t)m1 * kRec, r);
#pragma unroll
        for (int L = 0; L < 3; ++L) {
            s.g[L] += wt * r[L];
            s.gf[L] += wt * r[3 + L];
        }
#pragma unroll
        for (int i = 0; i < 6; ++i) s.E[i] -= hw * r[6 + i];
    }
#pragma unroll
    for (int i = 0; i < 6; ++i) s.E[i] *= aRnor;
#pragma unroll
    for (int i = 0; i < 3; ++i) { s.g[i] *= aRnor; s.gf[i] *= aRnor; }
    return s;
}

// The walk's arguments stay in the kernel's parameter space (constant bank): functions
// that read them are inlined, and the out-of-line ones above receive the fields they use.
// (A reference to the parameter block passed out of line makes every thread copy it to
// local memory and read its fields from there.)
__device__ __forceinline__ Strain strain_at(const WalkArgs& a, const double* P, int mp,
                                            int lo, int hi) {
    return kernel_strain(a.wrow, a.wpk, a.rad, a.wRnor, a.aRnor, P, mp, lo, hi);
}
__device__ __forceinline__ Strain strain_central(const WalkArgs& a, const double* P, int lo,
                                                 int hi) {
    return kernel_strain_central(a.rad, a.akk, a.aRnor, P, lo, hi);
}

// Ascending eigenvalues of a symmetric 3x3 matrix by cyclic Jacobi rotations in FP64
// (Rutishauser's formulation: t = sgn(theta) / (|theta| + sqrt(theta^2 + 1))): backward
// stable, so every eigenvalue is accurate to a few ulps of the matrix norm even when two
// of them coincide.  Six sweeps converge a 3x3 matrix to machine precision (quadratic
// convergence); a rotation whose off-diagonal entry is already zero is skipped.
__device__ __noinline__ void eig3_jacobi(const double* E, double* lam) {
    double a00 = E[0], a11 = E[1], a22 = E[2], a01 = E[3], a02 = E[4], a12 = E[5];
    for (int sweep = 0; sweep < 6; ++sweep) {
        if (a01 == 0.0 && a02 == 0.0 && a12 == 0.0) break;
        // (p, q) = (0, 1)
        if (a01 != 0.0) {
            const double th = (a11 - a00) / (2.0 * a01);
            const double t = (th >= 0.0 ? 1.0 : -1.0) / (fabs(th) + sqrt(th * th + 1.0));
            const double c = 1.0 / sqrt(t * t + 1.0), sn = t * c;
            a00 -= t * a01; a11 += t * a01; a01 = 0.0;
            const double r0 = a02, r1 = a12;
            a02 = c * r0 - sn * r1; a12 = sn * r0 + c * r1;
        }
        // (p, q) = (0, 2)
        if (a02 != 0.0) {
            const double th = (a22 - a00) / (2.0 * a02);
            const double t = (th >= 0.0 ? 1.0 : -1.0) / (fabs(th) + sqrt(th * th + 1.0));
            const double c = 1.0 / sqrt(t * t + 1.0), sn = t * c;
            a00 -= t * a02; a22 += t * a02; a02 = 0.0;
            const double r0 = a01, r1 = a12;
            a01 = c * r0 - sn * r1; a12 = sn * r0 + c * r1;
        }
        // (p, q) = (1, 2)
        if (a12 != 0.0) {
            const double th = (a22 - a11) / (2.0 * a12);
            const double t = (th >= 0.0 ? 1.0 : -1.0) / (fabs(th) + sqrt(th * th + 1.0));
            const double c = 1.0 / sqrt(t * t + 1.0), sn = t * c;
            a11 -= t * a12; a22 += t * a12; a12 = 0.0;
            const double r0 = a01, r1 = a02;
            a01 = c * r0 - sn * r1; a02 = sn * r0 + c * r1;
        }
    }
    double e0 = a00, e1 = a11, e2 = a22, t;
    if (e0 > e1) { t = e0; e0 = e1; e1 = t; }
    if (e1 > e2) { t = e1; e1 = e2; e2 = t; }
    if (e0 > e1) { t = e0; e0 = e1; e1 = t; }
    lam[0] = e0; lam[1] = e1; lam[2] = e2;
}

// Ascending eigenvalues of a symmetric 3x3 matrix in FP64, replacing LAPACK
// eigvals(Symmetric) (RadialShell.jl:215-220).  E = (11, 22, 33, 12, 13, 23).  The
// trigonometric solution of the characteristic cubic (O. K. Smith, Comm. ACM 4(4):168,
// 1961) is used where its angle is well conditioned; near a double eigenvalue (|r| close
// to 1, where acos amplifies the rounding of r by 1 / sqrt(1 - r^2)) the Jacobi solver
// above takes over, so the eigenvalue differences behind e_v and p_v keep full FP64
// accuracy.
__device__ __noinline__ void eig3(const double* E, double* lam) {
    const double a11 = E[0], a22 = E[1], a33 = E[2], a12 = E[3], a13 = E[4], a23 = E[5];
    const double q = (a11 + a22 + a33) / 3.0;
    const double b11 = a11 - q, b22 = a22 - q, b33 = a33 - q;
    const double off = a12 * a12 + a13 * a13 + a23 * a23;
    const double p2 = (b11 * b11 + b22 * b22 + b33 * b33 + 2.0 * off) / 6.0;
    if (!(p2 > 0.0)) { lam[0] = lam[1] = lam[2] = q; return; }
    const double pp = sqrt(p2);
    const double ip = 1.0 / pp;
    const double c11 = b11 * ip, c22 = b22 * ip, c33 = b33 * ip;
    const double c12 = a12 * ip, c13 = a13 * ip, c23 = a23 * ip;
    double r = 0.5 * (c11 * (c22 * c33 - c23 * c23) - c12 * (c12 * c33 - c23 * c13) +
                      c13 * (c12 * c23 - c22 * c13));
    if (fabs(r) > 1.0 - 1e-4) { eig3_jacobi(E, lam); return; }
    const double phi = acos(r) / 3.0;
    double e2 = q + 2.0 * pp * cos(phi);
    double e0 = q + 2.0 * pp * cos(phi + 2.0943951023931957);
    double e1 = 3.0 * q - e0 - e2;
    double t;
    if (e0 > e1) { t = e0; e0 = e1; e1 = t; }
    if (e1 > e2) { t = e1; e1 = e2; e2 = t; }
    if (e0 > e1) { t = e0; e0 = e1; e1 = t; }
    lam[0] = e0; lam[1] = e1; lam[2] = e2;
}

// Trilinear collapse-table lookup, -1 (out_val) outside the closed box
// (CollapseTable.jl:126-138), in FP64 over the Float32 table.
__device__ __forceinline__ double interp3(const WalkArgs& a, double x, double y, double z) {
    if (!(x >= a.X1 && x <= a.X2 && y >= a.Y1 && y <= a.Y2 && z >= a.Z1 && z <= a.Z2))
        return a.out_val;
    double tx = (x - a.X1) / ((a.X2 - a.X1) / (a.nx - 1));
    double ty = (y - a.Y1) / ((a.Y2 - a.Y1) / (a.ny - 1));
    double tz = (z - a.Z1) / ((a.Z2 - a.Z1) / (a.nz - 1));
    int ix = (int)floor(tx), iy = (int)floor(ty), iz = (int)floor(tz);
    ix = min(max(ix, 0), a.nx - 2);
    iy = min(max(iy, 0), a.ny - 2);
    iz = min(max(iz, 0), a.nz - 2);
    double fx = tx - ix, fy = ty - iy, fz = tz - iz;
    const long long sy = a.nx, sz = (long long)a.nx * a.ny;
    const float* t = a.ct + ix + iy * sy + iz * sz;
    double c000 = __ldg(t), c100 = __ldg(t + 1), c010 = __ldg(t + sy), c110 = __ldg(t + 1 + sy);
    double c001 = __ldg(t + sz), c101 = __ldg(t + 1 + sz), c011 = __ldg(t + sy + sz),
           c111 = __ldg(t + 1 + sy + sz);
    double c00 = c000 * (1.0 - fx) + c100 * fx;
    double c10 = c010 * (1.0 - fx) + c110 * fx;
    double c01 = c001 * (1.0 - fx) + c101 * fx;
    double c11 = c011 * (1.0 - fx) + c111 * fx;
    double c0 = c00 * (1.0 - fy) + c10 * fy;
    double c1 = c01 * (1.0 - fy) + c11 * fy;
    return c0 * (1.0 - fz) + c1 * fz;
}

// e_v, p_v and the eigen trace of a strain matrix (RadialShell.jl:633-639).
struct Shape { double trace, e_v, p_v, lam[3]; };
__device__ __forceinline__ Shape shape_of(const double E[6]) {
    Shape s;
    eig3(E, s.lam);
    s.trace = s.lam[0] + s.lam[1] + s.lam[2];
    s.e_v = 0.0; s.p_v = 0.0;
    if (s.trace > 0.0) {
        s.e_v = 0.5 * (s.lam[2] - s.lam[0]) / s.trace;
        s.p_v = 0.5 * (s.lam[2] + s.lam[0] - 2.0 * s.lam[1]) / s.trace;
    }
    return s;
}

// zvir of one inward-walk step (RadialShell.jl:629-648): the step's strain, its
// eigen trace (Frhoh) and zvir at shell mp.
struct Step {
    Strain k;
    double trace;
    double zvir;
};

__device__ __forceinline__ Step eval_step(const WalkArgs& a, const double* P, int mp, int m,
                                          bool force_minus_one) {
    Step st;
    st.k = strain_at(a, P, mp, 1, m);
    const Shape sh = shape_of(st.k.E);
    st.trace = sh.trace;
    st.zvir = -1.0;
    if (!force_minus_one) {
        const double Frho = P[(size_t)mp * kRec + P_FBAR];
        if (Frho > 0.0) {
            const double poe = sh.e_v < 1e-5 ? 0.0 : sh.p_v / sh.e_v;
            st.zvir = interp3(a, log10(Frho), sh.e_v, poe);
        }
    }
    return st;
}

__device__ __forceinline__ void write_no_collapse(const WalkArgs& a, long long p,
                                                  const Group& g) {
    const ht_results& o = a.out;
    for (int i = g.t; i < 9; i += g.G) o.strain[9 * p + i] = 0.f;
    if (g.t < 3) {
        o.eigs[3 * p + g.t] = 0.f; o.Sbar[3 * p + g.t] = 0.f; o.Sbar2[3 * p + g.t] = 0.f;
        o.gradpk[3 * p + g.t] = 0.f; o.gradpkf[3 * p + g.t] = 0.f;
        o.gradpkrf[3 * p + g.t] = 0.f;
    }
    if (g.t == 0) {
        o.RTHL[p] = -1.0f; o.Fbarx[p] = 0.f; o.e_v[p] = 0.f; o.p_v[p] = 0.f;
        o.Srb[p] = 0.f; o.d2F[p] = 0.f; o.zvir_half[p] = -1.0f;
        if (o.collapse_shell) o.collapse_shell[p] = 0;
    }
}

__device__ __forceinline__ void write_walk_shells(const WalkArgs& a, long long p,
                                                  const Group& g, int shells) {
    if (g.t == 0 && a.out.walk_shells) a.out.walk_shells[p] = shells;
}

template <bool PACKED>
struct CellLoader;

template <>
struct CellLoader<true> {
    // the cell's 32-byte record in one 256-bit load (records are 32-byte aligned): one
    // L1 request per cell instead of two
    __device__ __forceinline__ static void load(const WalkArgs& a, long long idx, int, int,
                                                int, float (&v)[8]) {
        if (!HT_INDEX_OK(a.status, idx, a.ntile)) {
            for (int i = 0; i < 8; ++i) v[i] = __int_as_float(0x7fc00000);
            return;
        }
        asm("ld.global.nc.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
            : "=f"(v[0]), "=f"(v[1]), "=f"(v[2]), "=f"(v[3]), "=f"(v[4]), "=f"(v[5]),
              "=f"(v[6]), "=f"(v[7])
            : "l"(a.rec + 2 * idx));
    }
};

template <>
struct CellLoader<false> {
    __device__ __forceinline__ static void load(const WalkArgs& a, long long idx, int iv1,
                                                int iv2, int iv3, float (&v)[8]) {
        // transposed read delta[iv3, iv1, iv2] (ext/CUDAExt.jl:819-820), cubic tile
        const long long idt = (long long)(iv3 - 1) + (long long)a.n1 * (iv1 - 1) +
                              a.s2 * (iv2 - 1);
        if (!HT_INDEX_OK(a.status, idx, a.ntile) || !HT_INDEX_OK(a.status, idt, a.ntile)) {
            for (int i = 0; i < 8; ++i) v[i] = __int_as_float(0x7fc00000);
            return;
        }
        v[0] = __ldg(a.delta + idx);
        v[1] = __ldg(a.delta + idt);
        v[2] = __ldg(a.ex + idx);
        v[3] = __ldg(a.ey + idx);
        v[4] = __ldg(a.ez + idx);
        if (a.e2x) {
            v[5] = __ldg(a.e2x + idx); v[6] = __ldg(a.e2y + idx); v[7] = __ldg(a.e2z + idx);
        } else {
            v[5] = 0.f; v[6] = 0.f; v[7] = 0.f;
        }
    }
};

// Gather cells [c_begin, c_end) of the r^2-sorted offset list around (ci, cj, ck): lane t
// of the group takes cells c_begin + t + u G in order and calls f(v, offset, idx, c) for
// the in-tile ones (idx: the cell's linear index in the tile, c: its place in the list).
// Out-of-tile cells are skipped (the reference never wraps).
template <bool PACKED, class F>
__device__ __forceinline__ void gather(const WalkArgs& a, int ci, int cj, int ck, int c_begin,
                                       int c_end, const Group& g, bool interior, F&& f) {
    if (c_end > c_begin && !HT_INDEX_OK(a.status, c_end - 1, a.ncells)) return;
    if (interior) {
        // every offset of the table stays inside the tile: no bounds test, and the cell's
        // linear offset comes precomputed with its (di, dj, dk)
        const long long cidx = (long long)(ci - 1) + (long long)a.n1 * (cj - 1) +
                               a.s2 * (ck - 1);
        // two of the lane's cells are requested before either is summed (same summation
        // order), so their record loads overlap: 473 against 498 ms on the 1152 tile's
        // walk; four at a time spilled and was no faster
        int c = c_begin + g.t;
        for (; c + g.G < c_end; c += 2 * g.G) {
            const int2 e0 = __ldg(a.cell + c), e1 = __ldg(a.cell + c + g.G);
            char4 o0, o1;
            memcpy(&o0, &e0.y, 4);
            memcpy(&o1, &e1.y, 4);
            float v0[8], v1[8];
            CellLoader<PACKED>::load(a, cidx + e0.x, ci + o0.x, cj + o0.y, ck + o0.z, v0);
            CellLoader<PACKED>::load(a, cidx + e1.x, ci + o1.x, cj + o1.y, ck + o1.z, v1);
            f(v0, o0, cidx + e0.x, c);
            f(v1, o1, cidx + e1.x, c + g.G);
        }
        if (c < c_end) {
            const int2 e = __ldg(a.cell + c);
            char4 o;
            memcpy(&o, &e.y, 4);
            float v[8];
            CellLoader<PACKED>::load(a, cidx + e.x, ci + o.x, cj + o.y, ck + o.z, v);
            f(v, o, cidx + e.x, c);
        }
        return;
    }
    for (int c = c_begin + g.t; c < c_end; c += g.G) {
        const char4 o = __ldg(a.off + c);
        const int iv1 = ci + o.x, iv2 = cj + o.y, iv3 = ck + o.z;
        if (iv1 < 1 || iv1 > a.n1 || iv2 < 1 || iv2 > a.n2 || iv3 < 1 || iv3 > a.n3) continue;
        const long long idx = (long long)(iv1 - 1) + (long long)a.n1 * (iv2 - 1) +
                              a.s2 * (iv3 - 1);
        float v[8];
        CellLoader<PACKED>::load(a, idx, iv1, iv2, iv3, v);
        f(v, o, idx, c);
    }
}

// mrf, the shell whose gradient is reported as gradpkrf (RadialShell.jl:449-464 for the
// CPU convention, ShellAnalysisGPU.jl:234-254 for the GPU one): the first shell s >= 2
// minimising |r2[s] - (Rf/alatt)^2| below 10, minus the lag of the reference counters.
__device__ __forceinline__ int find_mrf(const WalkArgs& a, double R2, int smax, int conv) {
    int lo = 2, hi = smax, first_ge = smax + 1;
    while (lo <= hi) {
        int mid = (lo + hi) >> 1;
        if ((double)a.r2[mid] >= R2) { first_ge = mid; hi = mid - 1; } else { lo = mid + 1; }
    }
    int best = -1;
    double bestd = 10.0;
    for (int s = max(2, first_ge - 1); s <= min(smax, first_ge); ++s) {
        double d = fabs((double)a.r2[s] - R2);
        if (d < bestd) { bestd = d; best = s; }
    }
    if (best < 0) return 1;
    if (conv == HT_CONV_GPU) return best - 1;
    return best >= 3 ? best - 2 : 1;
}

// Data-independent walk bounds of a peak: the last finalised shell m, the first shell
// past ir2min (m0_init), mrf and the last shell of mrf's window (need_rf).
struct Bounds { int m, m0_init, mrf, need_rf; };

__device__ __forceinline__ Bounds peak_bounds(const WalkArgs& a, double Rf, int ir2min) {
    Bounds b;
    const int nshells = a.nshells;
    // nshells - 1: the reference's per-cell loop never closes the last shell; rmax2rs
    // limits the shells further (ext/CUDAExt.jl:2192-2200)
    b.m = nshells - 1;
    if (a.rmax2rs > 0.0) {
        const double lim = a.rmax2rs * Rf / a.alatt;
        const double r2lim = lim * lim;
        int lo = 1, hi = nshells - 1, cnt = 0;
        while (lo <= hi) {
            int mid = (lo + hi) >> 1;
            if ((double)a.r2[mid] <= r2lim) { cnt = mid; lo = mid + 1; } else { hi = mid - 1; }
        }
        b.m = cnt;
    }
    b.m0_init = b.m;
    {
        int lo = 2, hi = b.m;
        while (lo <= hi) {
            int mid = (lo + hi) >> 1;
            if (a.r2[mid] > ir2min) { b.m0_init = mid; hi = mid - 1; } else { lo = mid + 1; }
        }
    }
    const double RR = Rf / a.alatt;
    b.mrf = b.m >= 2 ? find_mrf(a, RR * RR, a.conv == HT_CONV_GPU ? b.m : nshells, a.conv) : 1;
    b.need_rf = b.m >= 2 ? max(b.mrf, last_below(a.rad, 1, b.m, a.rad[b.mrf] + 2.0)) : 1;
    return b;
}

__device__ __forceinline__ Bounds bounds_of(const WalkArgs& a, long long p) {
    if (a.bounds) {
        const int4 v = __ldg(a.bounds + p);
        return Bounds{v.x, v.y, v.z, v.w};
    }
    return peak_bounds(a, a.Rf[p], a.ir2min[p]);
}

// One count of reject reason r in the block's shared counters (lane 0 of the group).
__device__ __forceinline__ void count_reject(unsigned* rej, const Group& g, int r) {
    if (g.t == 0) atomicAdd(rej + r, 1u);
}

template <bool PACKED>
__device__ __forceinline__ void process_peak(const WalkArgs& a, long long p, double* __restrict__ P,
                             double* __restrict__ R, const Group& g, unsigned* rej) {
    const double* rad = a.rad;
    const int G = g.G, t = g.t, RP = G + 1;
    const int ci = a.pi[p], cj = a.pj[p], ck = a.pk[p];
    const double ZZon = (double)a.ZZon[p];
    const double fcrit = (double)a.fcrit[p];
    if (ci < 1 || ci > a.n1 || cj < 1 || cj > a.n2 || ck < 1 || ck > a.n3) {
        // a centre outside the tile has no cells to walk (the reference would fault)
        write_walk_shells(a, p, g, 0);
        write_no_collapse(a, p, g);
        count_reject(rej, g, HT_REJECT_OUTSIDE);
        return;
    }
    const Bounds bd = bounds_of(a, p);
    const int m = bd.m;
    if (m < 2) {
        write_walk_shells(a, p, g, 1);
        write_no_collapse(a, p, g);
        count_reject(rej, g, HT_REJECT_NO_COLLAPSE);
        return;
    }

    // ---------------------------------------------------------------- walk ----
    float cv[8];
    const long long cidx = (long long)(ci - 1) + (long long)a.n1 * (cj - 1) + a.s2 * (ck - 1);
    const bool interior = a.cell && ci - 1 >= a.nhunt && ci + a.nhunt <= a.n1 &&
                          cj - 1 >= a.nhunt && cj + a.nhunt <= a.n2 && ck - 1 >= a.nhunt &&
                          ck + a.nhunt <= a.n3;
    CellLoader<PACKED>::load(a, cidx, ci, cj, ck, cv);
    const double Fbar1 = (double)cv[0];
    for (int i = t; i < kRec; i += G) P[kRec + i] = i == P_FBAR ? Fbar1 : 0.0;
    double Fbarp = Fbar1, dFbarp = Fbar1, radp = 0.0, rad5p = 0.0, csrb = 0.0;
    int m_c = 0;          // first shell >= m0_init with Fbar < fcrit (0: none yet)
    int stop_at = m + 1;  // the walk ends after this shell
    int s_end = 1;
    double cells_in = 1.0;

    for (int s = 2; s <= m; ++s) {
        const int st = __ldg(a.start + s);
        const int cnt = __ldg(a.count + s);
        Acc acc[13];
#pragma unroll
        for (int i = 0; i < 13; ++i) acc[i].zero();
        int nin = 0;
        gather<PACKED>(a, ci, cj, ck, st, st + cnt, g, interior,
                       [&](const float (&v)[8], char4 o, long long, int) {
            const float d0 = (float)o.x, d1 = (float)o.y, d2 = (float)o.z;
            ++nin;
            acc[0].add(v[0]);
            acc[1].add_prod(v[0], d0); acc[2].add_prod(v[0], d1); acc[3].add_prod(v[0], d2);
            acc[4].add_prod(v[1], d0); acc[5].add_prod(v[1], d1); acc[6].add_prod(v[1], d2);
            const float e0 = v[2], e1 = v[3], e2 = v[4];
            // the diagonal strain sums psi_L d_L are doubled when the shell is finalised
            // (doubling commutes with the rounding of every product and sum)
            acc[7].add_prod(e0, d0);
            acc[8].add_prod(e1, d1);
            acc[9].add_prod(e2, d2);
            acc[10].add_prod(e0, d1); acc[10].add_prod(e1, d0);
            acc[11].add_prod(e0, d2); acc[11].add_prod(e2, d0);
            acc[12].add_prod(e1, d2); acc[12].add_prod(e2, d1);
        });
        // combine the lanes in FP64, lanes 0..G-1 in order (deterministic)
        R[V_F * RP + t] = acc[0].value();
        R[V_N * RP + t] = (double)nin;
#pragma unroll
        for (int i = 0; i < 12; ++i) R[(V_G + i) * RP + t] = acc[1 + i].value();
        g.sync();
        for (int v = t; v < V_ROWS; v += G) {
            double sum = 0.0;
            for (int u = 0; u < G; ++u) sum += R[v * RP + u];
            R[v * RP + G] = sum;
        }
        g.sync();
        // finalise shell s (ShellAnalysisGPU.jl:197-228)
        const double Fs = R[V_F * RP + G];
        const double ns = R[V_N * RP + G];
        const double rs = rad[s];
        const double dF = ns > 0.0 ? Fs / ns : 0.0;
        const double r3p = radp * radp * radp, r3 = rs * rs * rs;
        const double Fbar_s = (r3p * Fbarp + 0.5 * (dFbarp + dF) * (r3 - r3p)) * a.irad3[s];
        const double r5 = rs * rs * rs * rs * rs;
        csrb += 0.5 * (Fbarp + Fbar_s) * (r5 - rad5p);
        double* q = P + (size_t)s * kRec;
        if (!HT_INDEX_OK(a.status, s, a.nshells + 2)) break;
        for (int i = t; i < kRec; i += G) {
            double v;
            if (i == P_FBAR) v = Fbar_s;
            else if (i == P_CSRB) v = csrb;
            else if (i < P_G) continue;   // unused
            else if (i >= P_SR && i < P_SR + 3) v = (2.0 * R[(V_G + i - P_G) * RP + G]) * a.irad[s];
            else v = R[(V_G + i - P_G) * RP + G] * a.irad[s];   // G, Gf, SR rows in order
            q[i] = v;
        }
        g.sync();
        cells_in += ns;
        Fbarp = Fbar_s; dFbarp = dF; radp = rs; rad5p = r5;
        s_end = s;
        // early exit: stop once every shell the post-processing reads is present --
        // Fbar up to the crossing m_c, gradients/strain of shells within r < rad[m0]+2
        // plus the first shell beyond it (zvir_half windows), and the mrf window.
        if (m_c == 0 && s >= bd.m0_init && Fbar_s < fcrit) {
            m_c = s;
            stop_at = max(first_above(rad, s + 1, m, rs + 2.0), bd.need_rf);
        }
        if (s >= stop_at) break;
    }
    if (t == 0 && a.stats) {
        atomicAdd(a.stats, (unsigned long long)cells_in);
        atomicAdd(a.stats + 1, (unsigned long long)s_end);
    }
    write_walk_shells(a, p, g, s_end);

    // ------------------------------------------------------ post-processing ----
    // gradient at the filter scale (RadialShell.jl:466-482); when mrf = 1 the window
    // starts at the centre shell
    double gradpkrf[3];
    {
        const Strain k = bd.mrf > 1 ? strain_at(a, P, bd.mrf, 1, bd.need_rf)
                                    : strain_central(a, P, 1, bd.need_rf);
        gradpkrf[0] = k.g[0]; gradpkrf[1] = k.g[1]; gradpkrf[2] = k.g[2];
    }

    // crossing (RadialShell.jl:485-526)
    int m0 = bd.m0_init;
    if (P[(size_t)m0 * kRec + P_FBAR] >= fcrit) {
        if (m_c != 0) m0 = m_c;   // else: no crossing, m0 stays, windows reach m
    } else {
        // inward: first shell below m0_init (from the top) with Fbar >= fcrit
        bool found = false;
        for (int base = bd.m0_init - 1; base >= 1 && !found; base -= G) {
            const int mp = base - t;
            const bool ge = mp >= 1 && P[(size_t)mp * kRec + P_FBAR] >= fcrit;
            const unsigned bal = g.ballot(ge);
            if (bal) {
                m0 = base - (__ffs(bal) - 1) + 1;
                found = true;
            }
        }
        if (!found) {   // RadialShell.jl:516-518
            write_no_collapse(a, p, g);
            count_reject(rej, g, HT_REJECT_NO_FCRIT);
            return;
        }
    }

    // inward walk (RadialShell.jl:529-686): step u evaluates shell m0 - u; step 0 is m0
    // itself with zvir forced to -1 (RadialShell.jl:566-567).  The G lanes evaluate G
    // consecutive steps at once; the first step with zvir >= ZZon collapses.  Step
    // results are staged in R (row = lane, row G = last step of the previous round).
    int tstar = -1, lrow = 0, prow = 0;
    for (int base = 0; base < m0; base += G) {
        const int u = base + t;
        double* row = R + t * kStepW;
        bool hit = false;
        if (u < m0) {
            const Step st = eval_step(a, P, m0 - u, m, u == 0);
#pragma unroll
            for (int i = 0; i < 6; ++i) row[i] = st.k.E[i];
#pragma unroll
            for (int i = 0; i < 3; ++i) { row[6 + i] = st.k.g[i]; row[9 + i] = st.k.gf[i]; }
            row[12] = st.trace;
            row[13] = st.zvir;
            hit = st.zvir >= ZZon;
        }
        const unsigned bal = g.ballot(hit);
        g.sync();
        if (bal) {
            const int l = __ffs(bal) - 1;
            tstar = base + l;
            lrow = l;
            prow = l > 0 ? l - 1 : G;
            break;
        }
        for (int i = t; i < 14; i += G) R[G * kStepW + i] = R[(G - 1) * kStepW + i];
        g.sync();
    }
    if (tstar < 0 || (tstar == 0 && m0 == 1)) {
        // m0 = 1 without a collapse at the centre: RadialShell.jl:603-605; no collapse:
        // :683-685; a collapse at the centre shell has no inner radius (RTHL <= 0)
        write_no_collapse(a, p, g);
        count_reject(rej, g, tstar == 0 ? HT_REJECT_RTHL_NEG
                             : m0 == 1 ? HT_REJECT_M0_ONE : HT_REJECT_NO_COLLAPSE);
        return;
    }
    if (tstar == 0) prow = lrow;
    const double* Lr = R + lrow * kStepW;   // collapse step ("last")
    const double* Pr = R + prow * kStepW;   // the step before it ("prev")

    const int m0f = m0 - tstar + 1;   // collapse at shell mp* = m0f - 1
    const double zvir1p = Lr[13];
    const double zvir1 = tstar == 0 ? -1.0 : Pr[13];
    const double dZ = zvir1p - zvir1;
    const double rp = rad[m0f - 1], rm = rad[m0f];
    double RTHL;
    if (zvir1 > 0.0 && dZ != 0.0) {
        const double R3 = rp * rp * rp + (rm * rm * rm - rp * rp * rp) * (zvir1p - ZZon) / dZ;
        RTHL = pow(R3, 1.0 / 3.0);
    } else {
        RTHL = rp;
    }
    if (RTHL <= 0.0) {   // RadialShell.jl:697-699
        write_no_collapse(a, p, g);
        count_reject(rej, g, HT_REJECT_RTHL_NEG);
        return;
    }

    const double RTHL3 = RTHL * RTHL * RTHL, RTHL5 = RTHL3 * RTHL * RTHL;
    const double rad3p = rp * rp * rp, rad3 = rm * rm * rm, drad3 = rad3 - rad3p;
    const double Fb_m = P[(size_t)m0f * kRec + P_FBAR];
    const double Fb_p = P[(size_t)(m0f - 1) * kRec + P_FBAR];
    double Fbarx, smat[6], gpk[3], gpkf[3];
    if (zvir1 > 0.0 && drad3 != 0.0) {
        const double frac = (RTHL3 - rad3p) / drad3;
        Fbarx = Fb_p + frac * (Fb_m - Fb_p);
#pragma unroll
        for (int i = 0; i < 6; ++i) smat[i] = Lr[i] + frac * (Pr[i] - Lr[i]);
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            gpk[i] = Lr[6 + i] + frac * (Pr[6 + i] - Lr[6 + i]);
            gpkf[i] = Lr[9 + i] + frac * (Pr[9 + i] - Lr[9 + i]);
        }
    } else {
        Fbarx = Fb_p;
#pragma unroll
        for (int i = 0; i < 6; ++i) smat[i] = Lr[i];
#pragma unroll
        for (int i = 0; i < 3; ++i) { gpk[i] = Pr[6 + i]; gpkf[i] = Pr[9 + i]; }
    }
    // normalize_strain + eigen (RadialShell.jl:730-734)
    const double tr = smat[0] + smat[1] + smat[2];
    if (tr != 0.0) {
        const double sc = Fbarx / tr;
#pragma unroll
        for (int i = 0; i < 6; ++i) smat[i] *= sc;
    }
    const Shape fin = shape_of(smat);
    // strain_final (RadialShell.jl:736, guarded as ShellAnalysisGPU.jl:459)
    double sfin[6];
    const double Frhoh = Lr[12];
    if (a.conv == HT_CONV_GPU && Frhoh == 0.0) {
#pragma unroll
        for (int i = 0; i < 6; ++i) sfin[i] = Lr[i];
    } else {
#pragma unroll
        for (int i = 0; i < 6; ++i) sfin[i] = Lr[i] * (Fbarx / Frhoh);
    }
    // Srb (RadialShell.jl:757-771) from the running numerator at shell m0f - 1
    double Srb = P[(size_t)(m0f - 1) * kRec + P_CSRB];
    const double r5p = m0f - 1 >= 2 ? rp * rp * rp * rp * rp : 0.0;
    if (zvir1 > 0.0 && dZ != 0.0) Srb += 0.5 * (Fb_p + Fbarx) * (RTHL5 - r5p);
    if (Fbarx * RTHL5 > 0.0) Srb /= (Fbarx * RTHL5);
    g.sync();   // R is reused below

    // cells with r <= RTHL: shells 1..s_in form a contiguous prefix of the cell list
    const int s_in = last_le(rad, 1, a.nshells, RTHL);
    const int ncell_in = s_in >= 1 ? __ldg(a.start + s_in) + __ldg(a.count + s_in) : 0;

    // Sbar, Sbar2 (RadialShell.jl:739-754): mean psi over the in-tile cells of shells
    // 1..m0f-1; and the mask: the core cells within RTHL (ShellAnalysisGPU.jl:513-528,
    // RadialShell.jl:773-782).  Both are prefixes of the cell list that differ by at most
    // shell m0f (RTHL lies between rad[m0f - 1] and rad[m0f]), so one pass over the longer
    // prefix serves both (a separate mask pass cost 3 % of the walk on the 1152 tile).
    double Sb[3], Sb2[3];
    {
        const int ncell = __ldg(a.start + m0f);
        const int nmask = a.mask ? ncell_in : 0;
        Acc ks[6];
#pragma unroll
        for (int i = 0; i < 6; ++i) ks[i].zero();
        int nloc = 0;
        gather<PACKED>(a, ci, cj, ck, 0, max(ncell, nmask), g, interior,
                       [&](const float (&v)[8], char4 o, long long idx, int c) {
            if (c < ncell) {
#pragma unroll
                for (int i = 0; i < 6; ++i) ks[i].add(v[2 + i]);
                ++nloc;
            }
            if (c < nmask) {
                const int iv1 = ci + o.x, iv2 = cj + o.y, iv3 = ck + o.z;
                if (iv1 > a.nbuff && iv1 <= a.n1 - a.nbuff && iv2 > a.nbuff &&
                    iv2 <= a.n2 - a.nbuff && iv3 > a.nbuff && iv3 <= a.n3 - a.nbuff &&
                    HT_INDEX_OK(a.status, idx, a.ntile))
                    a.mask[idx] = 1;
            }
        });
        const double nS = g.sum((double)nloc);
#pragma unroll
        for (int L = 0; L < 3; ++L) {
            const double s1 = g.sum(ks[L].value()), s2v = g.sum(ks[3 + L].value());
            Sb[L] = nS > 0.0 ? s1 / nS : 0.0;
            Sb2[L] = nS > 0.0 ? s2v / nS : 0.0;
        }
    }

    // d2F
    double d2F = 0.0;
    if (a.lapd) {
        Acc ks; ks.zero();
        int nloc = 0;
        if (a.conv == HT_CONV_GPU) {
            // all in-tile cells of shells with r <= RTHL, centre included
            // (ShellAnalysisGPU.jl:496-511)
            for (int c = t; c < ncell_in; c += G) {
                const char4 o = __ldg(a.off + c);
                const int iv1 = ci + o.x, iv2 = cj + o.y, iv3 = ck + o.z;
                if (iv1 < 1 || iv1 > a.n1 || iv2 < 1 || iv2 > a.n2 || iv3 < 1 || iv3 > a.n3) continue;
                const long long idx = (long long)(iv1 - 1) + (long long)a.n1 * (iv2 - 1) +
                                      a.s2 * (iv3 - 1);
                ks.add(__ldg(a.lapd + idx));
                ++nloc;
            }
        } else {
            // cells 2.. in shell order, stopping at the first out-of-tile cell
            // (RadialShell.jl:785-799)
            for (int base = 1; base < ncell_in; base += G) {
                const int c = base + t;
                bool oob = false;
                int iv1 = 0, iv2 = 0, iv3 = 0;
                if (c < ncell_in) {
                    const char4 o = __ldg(a.off + c);
                    iv1 = ci + o.x; iv2 = cj + o.y; iv3 = ck + o.z;
                    oob = iv1 < 1 || iv1 > a.n1 || iv2 < 1 || iv2 > a.n2 || iv3 < 1 || iv3 > a.n3;
                }
                const unsigned bal = g.ballot(oob);
                const int lim = bal ? __ffs(bal) - 1 : G;
                if (c < ncell_in && t < lim) {
                    const long long idx = (long long)(iv1 - 1) + (long long)a.n1 * (iv2 - 1) +
                                          a.s2 * (iv3 - 1);
                    ks.add(__ldg(a.lapd + idx));
                    ++nloc;
                }
                if (bal) break;
            }
        }
        const double tot = g.sum(ks.value());
        const double nt = g.sum((double)nloc);
        if (nt > 0.0) d2F = tot / nt;
    }

    // zvir_half (RadialShell.jl:801-859): radius jj is handled by lane (jj - 1) % G
    double zvir_half = -1.0;
    if (RTHL >= 3.0) {
        double mx = -1.0;
        bool nan = false;
        for (int jj0 = 0; jj0 < 10; jj0 += G) {
            const int jj = jj0 + t;   // 0-based radius index
            if (jj >= 10) continue;
            double zf = a.zh_frac[0];   // constant indices: the table stays in the parameters
#pragma unroll
            for (int q = 1; q < 10; ++q)
                if (jj == q) zf = a.zh_frac[q];
            const double rcur = RTHL * zf;
            const int mm1 = m - 1;
            int mupp_rc = 1;
            if (mm1 >= 2) {
                const int f = first_above(rad, 2, mm1, rcur + 2.0);
                mupp_rc = f <= mm1 ? f : mm1;
            }
            int mlow_rc = 1;
            {
                const int f = first_above(rad, 1, mm1, fmax(rcur - 2.0, 0.0));
                if (f <= mm1) mlow_rc = f;
            }
            int m0_rc = 1;
            if (mm1 >= 1) {
                const int f = first_above(rad, 1, mm1, rcur);
                m0_rc = f <= mm1 ? f : mm1;
            }
            const Strain k = m0_rc > 1 ? strain_at(a, P, m0_rc, mlow_rc, mupp_rc)
                                       : strain_central(a, P, mlow_rc, mupp_rc);
            const Shape sh = shape_of(k.E);
            const double Fc = P[(size_t)m0_rc * kRec + P_FBAR];
            const double poe = sh.e_v < 1e-5 ? 0.0 : sh.p_v / sh.e_v;
            double z = -1.0;
            if (Fc > 0.0) z = interp3(a, log10(Fc), sh.e_v, poe);
            const double zl = z - 1.0;
            if (isnan(zl)) nan = true;
            else mx = fmax(mx, zl);
        }
        // Julia's max propagates NaN
        const bool anynan = g.ballot(nan) != 0u;
        for (int o = G >> 1; o >= 1; o >>= 1) mx = fmax(mx, __shfl_xor_sync(g.mask, mx, o, G));
        zvir_half = anynan ? __longlong_as_double(0x7ff8000000000000ULL) : mx;
    }

    // outputs
    const ht_results& o = a.out;
    if (t == 0) {
        o.RTHL[p] = (float)RTHL;
        o.Fbarx[p] = (float)Fbarx;
        o.e_v[p] = (float)fin.e_v;
        o.p_v[p] = (float)fin.p_v;
        o.Srb[p] = (float)Srb;
        o.d2F[p] = (float)d2F;
        o.zvir_half[p] = (float)zvir_half;
        if (o.collapse_shell) o.collapse_shell[p] = m0f - 1;
    }
    for (int i = t; i < 9; i += G) {
        const int L = i % 3, K = i / 3;   // column-major (L, K)
        int idx6;
        if (L == K) idx6 = L;
        else if (L + K == 1) idx6 = 3;
        else if (L + K == 2) idx6 = 4;
        else idx6 = 5;
        o.strain[9 * p + i] = (float)sfin[idx6];
    }
    if (t < 3) {
        o.Sbar[3 * p + t] = (float)Sb[t];
        o.Sbar2[3 * p + t] = (float)Sb2[t];
        o.gradpk[3 * p + t] = (float)gpk[t];
        o.gradpkf[3 * p + t] = (float)gpkf[t];
        o.gradpkrf[3 * p + t] = (float)gradpkrf[t];
        o.eigs[3 * p + t] = (float)fin.lam[t];
    }
}

// One work item: kPeaksPerItem consecutive entries of the processing order, one per
// group of kSmallG lanes; group q of warp w owns scratch slot kPeaksPerItem w + q.
template <bool PACKED>
__device__ __forceinline__ void process_item(const WalkArgs& a, long long item, double* P0,
                                             double* W, int lane, unsigned* rej) {
    const int q = lane / kSmallG;
    const long long e = item * kPeaksPerItem + q;
    long long p = -1;
    if (e < a.npeaks) {
        p = a.order ? (long long)__ldg(a.order + e) : e;
        if (p < 0 || p >= a.npeaks) p = -1;   // not a peak index: skipped
    }
    const Group g{kSmallG, lane % kSmallG, q, ((1u << kSmallG) - 1u) << (q * kSmallG)};
    if (p >= 0)
        process_peak<PACKED>(a, p, P0 + q * a.scratch_stride,
                             W + q * group_smem_doubles(kSmallG), g, rej);
    __syncwarp();
}

// 3 blocks per SM: 80 registers; the few spills cost less than the lost occupancy.
template <bool PACKED>
__global__ void __launch_bounds__(kThreads, 3) walk_kernel(const WalkArgs a) {
    extern __shared__ double smem[];
    __shared__ unsigned rej[HT_REJECT_COUNT];   // the block's reject counts
    if (threadIdx.x < HT_REJECT_COUNT) rej[threadIdx.x] = 0u;
    __syncthreads();
    const int lane = threadIdx.x & 31;
    double* W = smem + (threadIdx.x >> 5) * kWarpSmemDoubles;
    const long long gw = (long long)blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5);
    const long long nw = (long long)gridDim.x * kWarpsPerBlock;
    double* P0 = a.scratch + gw * (32 / kSmallG) * a.scratch_stride;
    const long long nitems = (a.npeaks + kPeaksPerItem - 1) / kPeaksPerItem;
    long long item;
    if (a.dynamic) {
        int q = 0;
        if (lane == 0) q = atomicAdd(a.queue, 1);
        item = __shfl_sync(0xffffffffu, q, 0);
    } else {
        item = gw;
    }
    while (item < nitems) {
        process_item<PACKED>(a, item, P0, W, lane, rej);
        if (a.dynamic) {
            int q = 0;
            if (lane == 0) q = atomicAdd(a.queue, 1);
            item = __shfl_sync(0xffffffffu, q, 0);
        } else {
            item += nw;
        }
    }
    __syncthreads();
    if (threadIdx.x < HT_REJECT_COUNT && a.reject && rej[threadIdx.x])
        atomicAdd(a.reject + threadIdx.x, (unsigned long long)rej[threadIdx.x]);
}
// Processing order for BATCHED mode: key = Morton code of the 0-based (i, j, k), 20 bits
// per axis; in LEARNED mode coarse spatial blocks of 2^block_bits cells (a Morton prefix)
// and, inside a block, the predicted walk cost (descending).  Peaks consecutive in this
// order sit close together in the tile, so the warps walking them at the same time
// gather largely the same cell records, which then come from L2; in LEARNED mode the four
// peaks of a warp also walk similar distances.  The order changes no result (outputs are
// indexed by peak).
__device__ __forceinline__ unsigned long long spread3(unsigned v) {
    unsigned long long x = v & 0xfffffu;
    x = (x | x << 32) & 0x1f00000000ffffULL;
    x = (x | x << 16) & 0x1f0000ff0000ffULL;
    x = (x | x << 8) & 0x100f00f00f00f00fULL;
    x = (x | x << 4) & 0x10c30c30c30c30c3ULL;
    x = (x | x << 2) & 0x1249249249249249ULL;
    return x;
}

__global__ void __launch_bounds__(256) order_key_kernel(const WalkArgs a,
                                                        unsigned long long* __restrict__ keys,
                                                        int32_t* __restrict__ idx,
                                                        int4* __restrict__ bounds,
                                                        const float* __restrict__ cost) {
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= a.npeaks) return;
    const Bounds b = peak_bounds(a, a.Rf[p], a.ir2min[p]);
    bounds[p] = make_int4(b.m, b.m0_init, b.mrf, b.need_rf);
    if (!keys) return;
    const unsigned i = (unsigned)max(a.pi[p] - 1, 0), j = (unsigned)max(a.pj[p] - 1, 0),
                   k = (unsigned)max(a.pk[p] - 1, 0);
    const unsigned long long mort = spread3(i) | (spread3(j) << 1) | (spread3(k) << 2);
    if (cost) {
        // learned order: coarse spatial blocks of 2^block_bits cells (Morton prefix, keeps
        // the L2 locality), then descending predicted cost (1/16-cell steps, 24 bits)
        float c = cost[p];
        c = c == c ? fminf(fmaxf(c, 0.f), 1.0e6f) : 0.f;
        const unsigned long long q = min((unsigned long long)(c * 16.f), 0xFFFFFFull);
        const unsigned long long blk = (mort >> a.block_bits) & ((1ull << 38) - 1);
        keys[p] = (blk << 24) | (0xFFFFFFull - q);
    } else {
        keys[p] = mort;
    }
    idx[p] = (int32_t)p;
}

// Cell table of the bound tile: the linear offset di + n1 dj + n1 n2 dk of every table
// offset next to its (di, dj, dk), so that interior peaks gather with one 8-byte load and
// no bounds test per cell.
__global__ void __launch_bounds__(256) cell_table_kernel(const char4* __restrict__ off,
                                                         int2* __restrict__ cell,
                                                         long long ncells, int n1,
                                                         long long s2) {
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncells) return;
    const char4 o = off[c];
    int bits;
    memcpy(&bits, &o, 4);
    cell[c] = make_int2((int)(o.x + (long long)n1 * o.y + s2 * o.z), bits);
}

// Interleaved cell records: rec[2c] = (delta, delta[k,i,j], eta x, eta y),
// rec[2c+1] = (eta z, eta2 x, eta2 y, eta2 z).  A 32x32 (i, k) tile of the transposed
// read is staged through shared memory so both the reads and the record writes are
// coalesced along i.  Grid: (ceil(n/32), ceil(n/32), n) over (i-tile, k-tile, j).
__global__ void __launch_bounds__(256) pack_kernel(const float* __restrict__ delta,
                                                   const float* __restrict__ ex,
                                                   const float* __restrict__ ey,
                                                   const float* __restrict__ ez,
                                                   const float* __restrict__ e2x,
                                                   const float* __restrict__ e2y,
                                                   const float* __restrict__ e2z, int n,
                                                   float4* __restrict__ rec) {
    __shared__ float tile[32][33];
    const int i0 = blockIdx.x * 32, k0 = blockIdx.y * 32, j = blockIdx.z;
    const long long nn = (long long)n * n;
    // tile[ii][kk] = delta[(k0+kk) + n*(i0+ii) + n^2*j]   (coalesced along kk)
    for (int r = threadIdx.y; r < 32; r += 8) {
        const int ii = r, kk = threadIdx.x;
        const int i = i0 + ii, k = k0 + kk;
        float v = 0.f;
        if (i < n && k < n) v = delta[(long long)k + (long long)n * i + nn * j];
        tile[ii][kk] = v;
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += 8) {
        const int kk = r, ii = threadIdx.x;
        const int i = i0 + ii, k = k0 + kk;
        if (i < n && k < n) {
            const long long c = (long long)i + (long long)n * j + nn * k;
            float4 x, y;
            x.x = delta[c];
            x.y = tile[ii][kk];
            x.z = ex[c];
            x.w = ey[c];
            y.x = ez[c];
            if (e2x) { y.y = e2x[c]; y.z = e2y[c]; y.w = e2z[c]; }
            else { y.y = 0.f; y.z = 0.f; y.w = 0.f; }
            rec[2 * c] = x;
            rec[2 * c + 1] = y;
        }
    }
}

}  // namespace

int ht_launch_pack(ht_ctx* ctx, cudaStream_t st) {
    const ht_fields& f = ctx->fields;
    const int n = f.n1;
    dim3 grid((n + 31) / 32, (n + 31) / 32, n), block(32, 8);
    pack_kernel<<<grid, block, 0, st>>>(f.delta, f.etax, f.etay, f.etaz, f.eta2x, f.eta2y,
                                         f.eta2z, n, ctx->d_rec);
    HT_CUDA_TRY(cudaGetLastError(), "pack_kernel launch");
    ctx->last_kernels = 1;
    return HT_OK;
}

// Fill the kernel arguments common to both entry points.
static void fill_args(WalkArgs& a, const ht_ctx* ctx, const ht_fields& f, const ht_peak_batch* b,
                      double alatt, double rmax2rs, int32_t nbuff, int8_t* d_mask, int32_t conv,
                      const ht_results* out) {
    a.rec = ctx->d_rec;
    a.delta = f.delta; a.ex = f.etax; a.ey = f.etay; a.ez = f.etaz;
    a.e2x = f.eta2x; a.e2y = f.eta2y; a.e2z = f.eta2z; a.lapd = f.lapd;
    a.n1 = f.n1; a.n2 = f.n2; a.n3 = f.n3;
    a.s2 = (long long)f.n1 * f.n2;
    a.off = ctx->d_off; a.start = ctx->d_start; a.count = ctx->d_count; a.r2 = ctx->d_r2;
    a.rad = ctx->d_rad; a.nshells = ctx->nshells;
    a.irad = ctx->d_irad; a.irad3 = ctx->d_irad3;
    a.cell = nullptr; a.nhunt = ctx->nhunt;
    for (int jj = 0; jj < 10; ++jj) a.zh_frac[jj] = cbrt(jj / 9.0 * 0.5 + 0.5);
    a.wrow = ctx->d_wrow; a.wpk = ctx->d_wpk;
    a.ct = ctx->d_ct; a.nx = ctx->nx; a.ny = ctx->ny; a.nz = ctx->nz;
    a.X1 = ctx->X1; a.X2 = ctx->X2; a.Y1 = ctx->Y1; a.Y2 = ctx->Y2; a.Z1 = ctx->Z1;
    a.Z2 = ctx->Z2; a.out_val = ctx->out_val; a.akk = ctx->d_akk;
    a.pi = b->pi; a.pj = b->pj; a.pk = b->pk; a.Rf = b->Rf; a.ir2min = b->ir2min;
    a.ZZon = b->ZZon; a.fcrit = b->fcrit; a.npeaks = b->npeaks; a.order = b->order;
    a.bounds = nullptr;
    a.alatt = alatt;
    const double pi = 3.14159265358979323846;
    a.aRnor = 3.0 / alatt;                   // RadialShell.jl:296-300 with hlatt = 1
    a.wRnor = 3.0 * (1.0 / (4.0 * pi)) / alatt;
    a.rmax2rs = rmax2rs; a.nbuff = nbuff; a.conv = conv; a.mask = d_mask; a.out = *out;
    a.block_bits = ctx->tune_block_bits;
    a.queue = nullptr; a.dynamic = 0; a.stats = nullptr; a.reject = ctx->d_stats + 16;
    a.status = (int32_t*)(ctx->d_stats + 8);
    a.ntile = (long long)f.n1 * f.n2 * f.n3; a.ncells = ctx->ncells;
}

static size_t walk_smem_bytes() {
    return (size_t)kWarpsPerBlock * kWarpSmemDoubles * sizeof(double);
}

template <bool PACKED>
static int walk_blocks_per_sm(int* bpsm) {
    const size_t smem = walk_smem_bytes();
    cudaError_t e = cudaFuncSetAttribute(walk_kernel<PACKED>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess)
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(bpsm, walk_kernel<PACKED>, kThreads,
                                                          smem);
    if (e != cudaSuccess) return ht_cuda_fail(e, "walk_kernel occupancy query");
    if (*bpsm < 1) *bpsm = 1;
    return HT_OK;
}

int ht_launch_walk(ht_ctx* ctx, const ht_peak_batch* b, double alatt, double rmax2rs,
                   int32_t nbuff, int8_t* d_mask, int32_t conv, int32_t mode,
                   const ht_results* out, cudaStream_t st) {
    const bool packed = mode != HT_MODE_PLAIN;   // BATCHED and LEARNED
    int bpsm = 0;
    int rc = packed ? walk_blocks_per_sm<true>(&bpsm) : walk_blocks_per_sm<false>(&bpsm);
    if (rc != HT_OK) return rc;
    if (ctx->tune_walk_bpsm > 0 && ctx->tune_walk_bpsm < bpsm) bpsm = ctx->tune_walk_bpsm;
    long long blocks = (long long)ctx->num_sms * bpsm;
    const long long items = (b->npeaks + kPeaksPerItem - 1) / kPeaksPerItem;
    const long long need = (items + kWarpsPerBlock - 1) / kWarpsPerBlock;
    if (blocks > need) blocks = need;
    if (blocks < 1) blocks = 1;
    const long long stride = (long long)(ctx->nshells + 2) * kRec;
    const size_t slots = (size_t)blocks * kWarpsPerBlock * (32 / kSmallG);
    rc = ht_grow((void**)&ctx->d_scratch, &ctx->scratch_bytes, slots * stride * sizeof(double),
                 "shell-walk scratch");
    if (rc != HT_OK) return rc;

    WalkArgs a;
    fill_args(a, ctx, ctx->fields, b, alatt, rmax2rs, nbuff, d_mask, conv, out);
    a.scratch = ctx->d_scratch; a.scratch_stride = stride;
    a.queue = ctx->d_queue; a.dynamic = packed ? 1 : 0;
    // interior gather table for this tile's dims (skipped if an offset could overflow int)
    const long long n1 = ctx->fields.n1, s2 = (long long)ctx->fields.n1 * ctx->fields.n2;
    if ((long long)ctx->nhunt * (1 + n1 + s2) < 0x7fffffffLL) {
        if (ctx->cell_n1 != (int)n1 || ctx->cell_n2 != ctx->fields.n2 || !ctx->d_cell) {
            if (!ctx->d_cell) {
                rc = ht_alloc((void**)&ctx->d_cell, (size_t)ctx->ncells * sizeof(int2),
                              "interior cell table");
                if (rc != HT_OK) return rc;
            }
            cell_table_kernel<<<(unsigned)((ctx->ncells + 255) / 256), 256, 0, st>>>(
                ctx->d_off, ctx->d_cell, ctx->ncells, (int)n1, s2);
            HT_CUDA_TRY(cudaGetLastError(), "cell_table_kernel launch");
            ctx->cell_n1 = (int)n1;
            ctx->cell_n2 = ctx->fields.n2;
        }
        a.cell = ctx->d_cell;
    }
    a.stats = ctx->d_stats;
    int nk = 0;
    if (packed && b->npeaks > 0) {
        // per-peak walk bounds (one thread per peak, instead of binary searches inside the
        // walk), and without a caller order the spatial processing order
        if (b->npeaks > 0x7fffffffLL)
            return ht_fail(HT_ERR_CAPACITY, "ht_shell_analyse: more than 2^31-1 peaks in one batch");
        const int np = (int)b->npeaks;
        const bool sort = !b->order && np > 1;
        size_t temp = 0;
        if (sort)
            HT_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, temp,
                                                        (unsigned long long*)nullptr,
                                                        (unsigned long long*)nullptr,
                                                        (int32_t*)nullptr, (int32_t*)nullptr, np,
                                                        0, 63, st),
                        "radix sort size query");
        const size_t bb = ((size_t)np * 16 + 255) / 256 * 256;
        const size_t kb = sort ? ((size_t)np * 8 + 255) / 256 * 256 : 0;
        const size_t ib = sort ? ((size_t)np * 4 + 255) / 256 * 256 : 0;
        rc = ht_grow(&ctx->d_order_ws, &ctx->order_ws_bytes, bb + 2 * kb + 2 * ib + temp,
                     "peak-order workspace");
        if (rc != HT_OK) return rc;
        char* w = (char*)ctx->d_order_ws;
        int4* bounds = (int4*)w;
        unsigned long long* k_in = sort ? (unsigned long long*)(w + bb) : nullptr;
        unsigned long long* k_out = sort ? (unsigned long long*)(w + bb + kb) : nullptr;
        int32_t* v_in = sort ? (int32_t*)(w + bb + 2 * kb) : nullptr;
        int32_t* v_out = sort ? (int32_t*)(w + bb + 2 * kb + ib) : nullptr;
        void* tmp = w + bb + 2 * kb + 2 * ib;
        const float* cost = mode == HT_MODE_LEARNED ? b->cost : nullptr;
        order_key_kernel<<<(unsigned)((np + 255) / 256), 256, 0, st>>>(a, k_in, v_in, bounds,
                                                                        cost);
        HT_CUDA_TRY(cudaGetLastError(), "order_key_kernel launch");
        nk = 1;
        if (sort) {
            HT_CUDA_TRY(cub::DeviceRadixSort::SortPairs(tmp, temp, k_in, k_out, v_in, v_out,
                                                        np, 0, 63, st),
                        "radix sort of the peak order");
            a.order = v_out;
            nk += 3;   // the radix sort's passes (approximate count)
        }
        a.bounds = bounds;
    }
    HT_CUDA_TRY(cudaMemsetAsync(ctx->d_queue, 0, sizeof(int32_t), st), "queue reset");
    HT_CUDA_TRY(cudaMemsetAsync(ctx->d_stats, 0, 2 * sizeof(unsigned long long), st),
                "stats reset");
    const size_t smem = walk_smem_bytes();
    if (packed) walk_kernel<true><<<(unsigned)blocks, kThreads, smem, st>>>(a);
    else walk_kernel<false><<<(unsigned)blocks, kThreads, smem, st>>>(a);
    HT_CUDA_TRY(cudaGetLastError(), "walk_kernel launch");
    ctx->last_kernels = 1 + nk;
    return HT_OK;
}
// ------------------------------------------------- allocation-free entry point ----
//
// ht_shell_analyse_static: the shell collapse for callers that must not allocate device
// memory during the call -- code running while a stream is being captured into a CUDA
// graph, or hosts whose device memory is owned by a pool that only they may carve.  The
// walk's per-warp profile scratch, which ht_shell_analyse sizes and allocates with
// cudaMalloc, lives here in one file-scope __device__ array of kStaticScratchBytes
// instead.  Every GPU that loads the library holds that array until the process exits.

namespace {

constexpr size_t kStaticScratchBytes = 32u << 20;   // 32 MiB
__device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

// Device address of g_static_scratch per device, resolved once per device with that
// device current (a host-side name of a __device__ array is not a device address).  The
// address belongs to the device's primary context: after a cudaDeviceReset it is stale,
// so the library must not be used across a reset of a device it has run on.
constexpr int kMaxDevices = 64;
void* g_static_addr[kMaxDevices] = {};
std::mutex g_static_mu;

int static_scratch_address(int device, void** out) {
    if (device < 0 || device >= kMaxDevices)
        return ht_fail(HT_ERR_INVALID, "ht_shell_analyse_static: device id out of range");
    std::lock_guard<std::mutex> lk(g_static_mu);
    if (!g_static_addr[device]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
        if (e != cudaSuccess) return ht_cuda_fail(e, "cudaGetSymbolAddress(g_static_scratch)");
        g_static_addr[device] = p;
    }
    *out = g_static_addr[device];
    return HT_OK;
}

}  // namespace

extern "C" HT_API int ht_shell_analyse_static(ht_ctx* ctx, const ht_fields* f,
                                              const ht_peak_batch* b, double alatt,
                                              double rmax2rs, int32_t nbuff, int8_t* d_mask,
                                              int32_t conv, const ht_results* out,
                                              void* stream) {
    HT_RANGE("ht_shell_analyse_static");
    if (!ctx || !f || !b || !out)
        return ht_fail(HT_ERR_INVALID, "ht_shell_analyse_static: NULL argument");
    if (!f->delta || !f->etax || !f->etay || !f->etaz)
        return ht_fail(HT_ERR_INVALID, "ht_shell_analyse_static: delta and eta x/y/z are required");
    if ((f->eta2x || f->eta2y || f->eta2z) && !(f->eta2x && f->eta2y && f->eta2z))
        return ht_fail(HT_ERR_INVALID, "ht_shell_analyse_static: give all of eta2x/y/z or none");
    if (f->n1 < 1 || f->n1 != f->n2 || f->n1 != f->n3)
        return ht_fail(HT_ERR_INVALID, "ht_shell_analyse_static: the tile must be cubic");
    if (b->npeaks < 0) return ht_fail(HT_ERR_INVALID, "ht_shell_analyse_static: npeaks < 0");
    if (b->npeaks > 0 && (!b->pi || !b->pj || !b->pk || !b->Rf || !b->ir2min || !b->ZZon ||
                          !b->fcrit || !out->RTHL || !out->Fbarx || !out->e_v || !out->p_v ||
                          !out->strain || !out->eigs || !out->Srb || !out->Sbar ||
                          !out->Sbar2 || !out->gradpk || !out->gradpkf || !out->gradpkrf ||
                          !out->d2F || !out->zvir_half))
        return ht_fail(HT_ERR_INVALID, "ht_shell_analyse_static: NULL peak or result array");
    if (!(alatt > 0.0)) return ht_fail(HT_ERR_INVALID, "ht_shell_analyse_static: alatt must be > 0");
    if (conv != HT_CONV_GPU && conv != HT_CONV_CPU)
        return ht_fail(HT_ERR_INVALID, "ht_shell_analyse_static: unknown conv");
    if (conv == HT_CONV_CPU && rmax2rs > 0.0)
        return ht_fail(HT_ERR_INVALID, "ht_shell_analyse_static: HT_CONV_CPU supports rmax2rs == 0 only");
    if (nbuff < 0) return ht_fail(HT_ERR_INVALID, "ht_shell_analyse_static: nbuff < 0");
    if (ctx->nshells < 3)
        return ht_fail(HT_ERR_INVALID, "ht_shell_analyse_static: hunt radius too small");
    // one block (8 warps x 4 group slots) must fit the static scratch
    const long long stride = (long long)(ctx->nshells + 2) * kRec;
    const size_t per_block =
        (size_t)kWarpsPerBlock * (32 / kSmallG) * stride * sizeof(double);
    if (per_block > kStaticScratchBytes)
        return ht_fail(HT_ERR_CAPACITY,
                       "ht_shell_analyse_static: the hunt radius needs " +
                           std::to_string(per_block) + " bytes of scratch per block, more than "
                           "the static maximum of " + std::to_string(kStaticScratchBytes));
    ctx->last_kernels = 0;
    if (b->npeaks == 0) return HT_OK;
    HT_CUDA_TRY(cudaSetDevice(ctx->device), "cudaSetDevice");
    void* scratch = nullptr;
    int rc = static_scratch_address(ctx->device, &scratch);
    if (rc != HT_OK) return rc;
    int bpsm = 0;
    rc = walk_blocks_per_sm<false>(&bpsm);
    if (rc != HT_OK) return rc;
    if (ctx->tune_walk_bpsm > 0 && ctx->tune_walk_bpsm < bpsm) bpsm = ctx->tune_walk_bpsm;
    long long blocks = (long long)ctx->num_sms * bpsm;
    const long long fit = (long long)(kStaticScratchBytes / per_block);
    const long long items = (b->npeaks + kPeaksPerItem - 1) / kPeaksPerItem;
    const long long need = (items + kWarpsPerBlock - 1) / kWarpsPerBlock;
    if (blocks > fit) blocks = fit;
    if (blocks > need) blocks = need;

    WalkArgs a;
    fill_args(a, ctx, *f, b, alatt, rmax2rs, nbuff, d_mask, conv, out);
    a.rec = nullptr;
    a.scratch = (double*)scratch; a.scratch_stride = stride;
    a.queue = nullptr; a.dynamic = 0;   // static item-to-warp schedule: no counter to clear
    a.stats = nullptr;
    const size_t smem = walk_smem_bytes();
    walk_kernel<false><<<(unsigned)blocks, kThreads, smem, (cudaStream_t)stream>>>(a);
    HT_CUDA_TRY(cudaGetLastError(), "walk_kernel launch (static scratch)");
    ctx->last_kernels = 1;
    return HT_OK;
}

// ------------------------------------------------------------ measurement aid ----
//
// Scattered 32-byte record gathers with the walk's own load, one per index, and nothing
// else: with random indices this is the gather rate of a walk that found none of its
// cells in a cache.

namespace {

__global__ void __launch_bounds__(256) record_gather_kernel(const float4* __restrict__ rec,
                                                            long long ncells,
                                                            const int64_t* __restrict__ idx,
                                                            long long n,
                                                            float* __restrict__ out) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const long long c = __ldg(idx + i);
        if (c < 0 || c >= ncells) {
            out[i] = __int_as_float(0x7fc00000);
            continue;
        }
        float v[8];
        asm("ld.global.nc.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
            : "=f"(v[0]), "=f"(v[1]), "=f"(v[2]), "=f"(v[3]), "=f"(v[4]), "=f"(v[5]),
              "=f"(v[6]), "=f"(v[7])
            : "l"(rec + 2 * c));
        out[i] = ((v[0] + v[1]) + (v[2] + v[3])) + ((v[4] + v[5]) + (v[6] + v[7]));
    }
}

}  // namespace

extern "C" HT_API int ht_record_gather_probe(ht_ctx* ctx, const int64_t* d_idx, int64_t n_idx,
                                             float* d_out, void* stream) {
    HT_RANGE("ht_record_gather_probe");
    if (!ctx || (n_idx > 0 && (!d_idx || !d_out)))
        return ht_fail(HT_ERR_INVALID, "ht_record_gather_probe: NULL argument");
    if (n_idx < 0) return ht_fail(HT_ERR_INVALID, "ht_record_gather_probe: n_idx < 0");
    if (!ctx->bound || !ctx->d_rec)
        return ht_fail(HT_ERR_STATE, "ht_record_gather_probe: no packed tile (ht_fields_pack)");
    ctx->last_kernels = 0;
    if (n_idx == 0) return HT_OK;
    HT_CUDA_TRY(cudaSetDevice(ctx->device), "cudaSetDevice");
    long long blocks = (n_idx + 255) / 256;
    const long long cap = (long long)ctx->num_sms * 8;
    if (blocks > cap) blocks = cap;
    const long long ncells = (long long)ctx->fields.n1 * ctx->fields.n2 * ctx->fields.n3;
    record_gather_kernel<<<(unsigned)blocks, 256, 0, (cudaStream_t)stream>>>(
        ctx->d_rec, ncells, d_idx, n_idx, d_out);
    HT_CUDA_TRY(cudaGetLastError(), "record_gather_kernel launch");
    ctx->last_kernels = 1;
    return HT_OK;
}
