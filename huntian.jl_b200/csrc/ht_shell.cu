// Radial-shell collapse on sm_100a: one warp per peak.
//
// For every peak the warp walks the shells of the r^2-sorted offset table outward
// (the per-shell gather of ShellAnalysisGPU.jl:153-229 / ext/CUDAExt.jl:752-924),
// accumulating 22 FP32 sums per shell with Kahan compensation in each lane and
// combining the lanes in FP64.  The per-shell profile (Fbar, gradients, symmetrised
// strain sums and running means) goes to a per-warp scratch slot in FP64.  The walk
// stops as soon as every shell the post-processing can read has been gathered.  The
// same warp then runs the post-processing of RadialShell.jl:449-859 /
// ext/CUDAExt.jl:1213-1912 in FP64: fcrit crossing, the inward strain/eigen/barrier
// walk (32 steps evaluated at once, one per lane), RTHL interpolation, Sbar, Srb, d2F,
// zvir_half and the mask update.
//
// Two execution modes give identical results:
//   PLAIN   reads the eight reference fields separately, static peak->warp schedule;
//   BATCHED reads 32-byte interleaved cell records (one sector per cell) built by
//           ht_pack_kernel, persistent grid with a dynamic work queue.
#include <math.h>

#include <mutex>
#include <string>

#include "ht_internal.cuh"

namespace {

constexpr int kWarpsPerBlock = 8;
constexpr int kThreads = kWarpsPerBlock * 32;
constexpr int kRec = 24;   // doubles per shell in the scratch profile

// Scratch profile record, one per shell m (1-based):
enum : int {
    P_FBAR = 0,
    P_G = 1,      // 3: Gshell / rad
    P_GF = 4,     // 3: Gshellf / rad
    P_SR = 7,     // 6: (SR_LK + SR_KL) / rad for 11, 22, 33, 12, 13, 23
    P_CS = 13,    // 3: running sum of Sshell over shells 1..m
    P_CS2 = 16,   // 3: running sum of S2shell
    P_CN = 19,    // running count of in-tile cells
    P_CSRB = 20,  // running Srb numerator, RadialShell.jl:760-764
};

// Values held by the lanes after the transposed reduction of one shell.
enum : int {
    V_F = 0, V_N = 1, V_S = 2, V_S2 = 5, V_G = 8, V_GF = 11, V_SR = 14, V_COUNT = 23
};

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
    const int32_t* start;
    const int32_t* count;
    const int32_t* r2;
    const double* rad;
    int nshells;

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

    double alatt, wRnor, aRnor, rmax2rs;
    int nbuff;
    int conv;
    int8_t* mask;
    ht_results out;

    double* scratch;
    long long scratch_stride;
    int32_t* queue;
    int dynamic;
    unsigned long long* stats;
};

// ------------------------------------------------------------ small helpers ----

struct Kahan {
    float s, c;
    __device__ __forceinline__ void zero() { s = 0.f; c = 0.f; }
    __device__ __forceinline__ void add(float x) {
        float y = x - c;
        float t = s + y;
        c = (t - s) - y;
        s = t;
    }
    __device__ __forceinline__ double value() const { return (double)s - (double)c; }
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

// RadialShell.jl:95-121 (Fortran hRinteg).
__device__ __forceinline__ double hRinteg(double u0, double u12) {
    double x0 = fabs(u0);
    if (x0 >= 2.0) return 0.0;
    const double one7 = 1.0 / 7.0;
    double result = 1.6 * u12 - 6.4 * one7;
    double x02 = x0 * x0, x04 = x02 * x02;
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

struct Strain {
    double E[6];   // 11, 22, 33, 12, 13, 23
    double g[3];
    double gf[3];
};

// kernel_strain (RadialShell.jl:225-274) over shells lo..hi of the profile `P`,
// centred on shell mp, in FP64.  Shells at |rad[mp] - rad[m1]| >= 2 carry no weight.
__device__ Strain kernel_strain(const double* __restrict__ P, const double* __restrict__ rad,
                                const double* __restrict__ akk, int mp, int lo, int hi,
                                double wRnor, double aRnor) {
    Strain s;
#pragma unroll
    for (int i = 0; i < 6; ++i) s.E[i] = 0.0;
#pragma unroll
    for (int i = 0; i < 3; ++i) { s.g[i] = 0.0; s.gf[i] = 0.0; }
    double scale;
    if (mp > 1) {
        const double rmp = rad[mp];
        for (int m1 = lo; m1 <= hi; ++m1) {
            const double r1 = rad[m1];
            const double u0 = rmp - r1;
            const double u02 = u0 * u0;
            if (u02 < 4.0) {
                const double u12 = rmp * rmp + r1 * r1;
                const double den = u12 - u02;
                const double wt = hRinteg(u0, u12) / (den * den);
                const double* q = P + (size_t)m1 * kRec;
                const double hw = 0.5 * wt;
#pragma unroll
                for (int L = 0; L < 3; ++L) {
                    s.g[L] += wt * q[P_G + L];
                    s.gf[L] += wt * q[P_GF + L];
                }
#pragma unroll
                for (int i = 0; i < 6; ++i) s.E[i] -= hw * q[P_SR + i];
            }
        }
        scale = wRnor / rmp;
    } else {
        for (int m1 = lo; m1 <= hi; ++m1) {
            const double r1 = rad[m1];
            const double con = 100.0 * r1 * r1;
            const double fl = floor(con);
            const int icon = (int)fl;
            const double diff = con - fl;
            double aww = 0.0;
            if (icon >= 0 && icon < 1100) aww = akk[icon] + diff * (akk[icon + 1] - akk[icon]);
            const double wt = 0.5 * aww / r1;
            const double* q = P + (size_t)m1 * kRec;
            const double hw = 0.5 * wt;
#pragma unroll
            for (int L = 0; L < 3; ++L) {
                s.g[L] += wt * q[P_G + L];
                s.gf[L] += wt * q[P_GF + L];
            }
#pragma unroll
            for (int i = 0; i < 6; ++i) s.E[i] -= hw * q[P_SR + i];
        }
        scale = aRnor;
    }
#pragma unroll
    for (int i = 0; i < 6; ++i) s.E[i] *= scale;
#pragma unroll
    for (int i = 0; i < 3; ++i) { s.g[i] *= scale; s.gf[i] *= scale; }
    return s;
}

// Ascending eigenvalues of a symmetric 3x3 matrix by cyclic Jacobi rotations in FP64
// (Golub & Van Loan, Alg. 8.4.3), replacing LAPACK eigvals(Symmetric)
// (RadialShell.jl:215-220).  E = (11, 22, 33, 12, 13, 23).
__device__ void eig3(const double E[6], double lam[3]) {
    double a[3][3];
    a[0][0] = E[0]; a[1][1] = E[1]; a[2][2] = E[2];
    a[0][1] = a[1][0] = E[3];
    a[0][2] = a[2][0] = E[4];
    a[1][2] = a[2][1] = E[5];
    for (int sweep = 0; sweep < 64; ++sweep) {
        double off = a[0][1] * a[0][1] + a[0][2] * a[0][2] + a[1][2] * a[1][2];
        double dia = a[0][0] * a[0][0] + a[1][1] * a[1][1] + a[2][2] * a[2][2];
        if (off == 0.0 || off <= 1e-40 * dia) break;
#pragma unroll
        for (int pq = 0; pq < 3; ++pq) {
            const int p = pq == 2 ? 1 : 0;
            const int q = pq == 0 ? 1 : 2;
            double apq = a[p][q];
            if (apq == 0.0) continue;
            double theta = (a[q][q] - a[p][p]) / (2.0 * apq);
            double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
            double c = 1.0 / sqrt(t * t + 1.0), sn = t * c;
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                double akp = a[k][p], akq = a[k][q];
                a[k][p] = c * akp - sn * akq;
                a[k][q] = sn * akp + c * akq;
            }
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                double apk = a[p][k], aqk = a[q][k];
                a[p][k] = c * apk - sn * aqk;
                a[q][k] = sn * apk + c * aqk;
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

// Trilinear collapse-table lookup, -1 (out_val) outside the closed box
// (CollapseTable.jl:126-138), in FP64 over the Float32 table.
__device__ double interp3(const WalkArgs& a, double x, double y, double z) {
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

// Per-warp shared-memory staging: the 23 per-lane shell sums during the walk, and the
// results of 32 inward-walk steps (+ one carried step) during the post-processing.
constexpr int kRedRows = 23, kRedPitch = 33;          // [value][lane], padded pitch
constexpr int kStepW = 16, kStepRows = 33;            // [lane or carry][field]
constexpr int kWarpSmemDoubles =
    kRedRows * kRedPitch > kStepRows * kStepW ? kRedRows * kRedPitch : kStepRows * kStepW;

// Lane v (< 23) returns the warp total of value v, summed over lanes 0..31 in order
// (deterministic).  `R` is the warp's staging area.
__device__ __forceinline__ double warp_column_sum(double* R, int lane) {
    __syncwarp();
    double s = 0.0;
    if (lane < kRedRows) {
        const double* r = R + lane * kRedPitch;
#pragma unroll 8
        for (int t = 0; t < 32; ++t) s += r[t];
    }
    __syncwarp();
    return s;
}

__device__ __forceinline__ double warp_sum(double x) {
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    return x;
}

__device__ void write_no_collapse(const WalkArgs& a, long long p, int lane) {
    const ht_results& o = a.out;
    if (lane == 0) {
        o.RTHL[p] = -1.0f; o.Fbarx[p] = 0.f; o.e_v[p] = 0.f; o.p_v[p] = 0.f;
        o.Srb[p] = 0.f; o.d2F[p] = 0.f; o.zvir_half[p] = -1.0f;
    }
    if (lane < 9) o.strain[9 * p + lane] = 0.f;
    if (lane < 3) {
        o.eigs[3 * p + lane] = 0.f; o.Sbar[3 * p + lane] = 0.f; o.Sbar2[3 * p + lane] = 0.f;
        o.gradpk[3 * p + lane] = 0.f; o.gradpkf[3 * p + lane] = 0.f;
        o.gradpkrf[3 * p + lane] = 0.f;
    }
}

// One step of the inward walk evaluated by one lane.
struct Step {
    Strain k;
    double trace;   // Frhoh
    double zvir;
};

__device__ __forceinline__ Step eval_step(const WalkArgs& a, const double* P, int mp, int m,
                                          bool force_minus_one) {
    const double* rad = a.rad;
    int lo, hi;
    if (mp > 1) {
        lo = first_above(rad, 2, mp, fmax(rad[mp] - 2.0, 0.0));
        hi = last_below(rad, mp, m, rad[mp] + 2.0);
        if (hi < mp) hi = mp;
    } else {
        lo = 2;
        hi = last_below(rad, 2, m, 2.0);
    }
    Step st;
    st.k = kernel_strain(P, rad, a.akk, mp, lo, hi, a.wRnor, a.aRnor);
    Shape sh = shape_of(st.k.E);
    st.trace = sh.trace;
    st.zvir = -1.0;
    if (!force_minus_one) {
        const double Frho = P[(size_t)mp * kRec + P_FBAR];
        if (Frho > 0.0) {
            double poe = sh.e_v < 1e-5 ? 0.0 : sh.p_v / sh.e_v;
            st.zvir = interp3(a, log10(Frho), sh.e_v, poe);
        }
    }
    return st;
}

template <bool PACKED>
struct CellLoader;

template <>
struct CellLoader<true> {
    __device__ __forceinline__ static void load(const WalkArgs& a, int iv1, int iv2, int iv3,
                                                float (&v)[8]) {
        const long long idx = (long long)(iv1 - 1) + (long long)a.n1 * (iv2 - 1) +
                              a.s2 * (iv3 - 1);
        const float4 x = __ldg(a.rec + 2 * idx);
        const float4 y = __ldg(a.rec + 2 * idx + 1);
        v[0] = x.x; v[1] = x.y; v[2] = x.z; v[3] = x.w;
        v[4] = y.x; v[5] = y.y; v[6] = y.z; v[7] = y.w;
    }
};

template <>
struct CellLoader<false> {
    __device__ __forceinline__ static void load(const WalkArgs& a, int iv1, int iv2, int iv3,
                                                float (&v)[8]) {
        const long long idx = (long long)(iv1 - 1) + (long long)a.n1 * (iv2 - 1) +
                              a.s2 * (iv3 - 1);
        // transposed read delta[iv3, iv1, iv2] (ext/CUDAExt.jl:819-820), cubic tile
        const long long idt = (long long)(iv3 - 1) + (long long)a.n1 * (iv1 - 1) +
                              a.s2 * (iv2 - 1);
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

// mrf, the shell whose gradient is reported as gradpkrf (RadialShell.jl:449-464 for the
// CPU convention, ShellAnalysisGPU.jl:234-254 for the GPU one): the first shell s >= 2
// minimising |r2[s] - (Rf/alatt)^2| below 10, minus the lag of the reference counters.
__device__ int find_mrf(const WalkArgs& a, double R2, int smax, int conv) {
    // first s in [2, smax] with r2 >= R2
    int lo = 2, hi = smax, first_ge = smax + 1;
    while (lo <= hi) {
        int mid = (lo + hi) >> 1;
        if ((double)a.r2[mid] >= R2) { first_ge = mid; hi = mid - 1; } else { lo = mid + 1; }
    }
    int best = -1;
    double bestd = 10.0;
    // candidates in ascending order: first_ge - 1, first_ge (strict < keeps the first)
    for (int s = max(2, first_ge - 1); s <= min(smax, first_ge); ++s) {
        double d = fabs((double)a.r2[s] - R2);
        if (d < bestd) { bestd = d; best = s; }
    }
    if (best < 0) return 1;
    if (conv == HT_CONV_GPU) return best - 1;
    return best >= 3 ? best - 2 : 1;
}

template <bool PACKED>
__device__ void process_peak(const WalkArgs& a, long long p, double* __restrict__ P,
                             double* __restrict__ R, int lane) {
    const double* rad = a.rad;
    const int ci = a.pi[p], cj = a.pj[p], ck = a.pk[p];
    const double Rf = a.Rf[p];
    const int ir2min = a.ir2min[p];
    const double ZZon = (double)a.ZZon[p];
    const double fcrit = (double)a.fcrit[p];
    const int nshells = a.nshells;
    if (ci < 1 || ci > a.n1 || cj < 1 || cj > a.n2 || ck < 1 || ck > a.n3) {
        // a centre outside the tile has no cells to walk (the reference would fault)
        write_no_collapse(a, p, lane);
        return;
    }

    // last shell that is finalised (nshells - 1: the reference's per-cell loop never
    // closes the last shell), optionally limited by rmax2rs (ext/CUDAExt.jl:2192-2200)
    int m = nshells - 1;
    if (a.rmax2rs > 0.0) {
        const double lim = a.rmax2rs * Rf / a.alatt;
        const double r2lim = lim * lim;
        int cnt = 0;
        for (int s = 1; s <= nshells - 1; ++s) {
            if (!((double)a.r2[s] <= r2lim)) break;
            cnt = s;
        }
        m = cnt;
    }
    if (m < 2) { write_no_collapse(a, p, lane); return; }

    // data-independent shell indices
    int m0_init = m;
    {
        int lo = 2, hi = m;
        while (lo <= hi) {
            int mid = (lo + hi) >> 1;
            if (a.r2[mid] > ir2min) { m0_init = mid; hi = mid - 1; } else { lo = mid + 1; }
        }
    }
    const double RR = Rf / a.alatt;
    const int mrf = find_mrf(a, RR * RR, a.conv == HT_CONV_GPU ? m : nshells, a.conv);
    const int need_rf = max(mrf, last_below(rad, 1, m, rad[mrf] + 2.0));

    // ---------------------------------------------------------------- walk ----
    // centre cell (shell 1)
    float cv[8];
    CellLoader<PACKED>::load(a, ci, cj, ck, cv);
    const double Fbar1 = (double)cv[0];
    {
        double* q = P + kRec;
        if (lane < kRec) {
            double v = 0.0;
            if (lane == P_FBAR) v = Fbar1;
            else if (lane >= P_CS && lane < P_CS + 3) v = (double)cv[2 + lane - P_CS];
            else if (lane >= P_CS2 && lane < P_CS2 + 3) v = (double)cv[5 + lane - P_CS2];
            else if (lane == P_CN) v = 1.0;
            q[lane] = v;
        }
    }
    double Fbarp = Fbar1, dFbarp = Fbar1, radp = 0.0, rad5p = 0.0, csrb = 0.0;
    // running sums held by the lane that owns the value after the reduction
    double cum = 0.0;
    if (lane >= V_S && lane < V_S + 3) cum = (double)cv[2 + lane - V_S];
    if (lane >= V_S2 && lane < V_S2 + 3) cum = (double)cv[5 + lane - V_S2];
    if (lane == V_N) cum = 1.0;

    int m_c = 0;          // first shell >= m0_init with Fbar < fcrit (0: none yet)
    int stop_at = m + 1;  // walk ends after this shell
    int s_end = 1;
    unsigned long long cells_in = 1;

    for (int s = 2; s <= m; ++s) {
        const int st = __ldg(a.start + s);
        const int cnt = __ldg(a.count + s);
        Kahan acc[22];
#pragma unroll
        for (int i = 0; i < 22; ++i) acc[i].zero();
        int nin = 0;
        for (int c = lane; c < cnt; c += 32) {
            const char4 o = __ldg(a.off + st + c);
            const int iv1 = ci + o.x, iv2 = cj + o.y, iv3 = ck + o.z;
            if (iv1 < 1 || iv1 > a.n1 || iv2 < 1 || iv2 > a.n2 || iv3 < 1 || iv3 > a.n3) continue;
            float v[8];
            CellLoader<PACKED>::load(a, iv1, iv2, iv3, v);
            const float d[3] = {(float)o.x, (float)o.y, (float)o.z};
            ++nin;
            acc[0].add(v[0]);
#pragma unroll
            for (int L = 0; L < 3; ++L) {
                acc[1 + L].add(v[2 + L]);
                acc[4 + L].add(v[5 + L]);
                acc[7 + L].add(v[0] * d[L]);
                acc[10 + L].add(v[1] * d[L]);
#pragma unroll
                for (int K = 0; K < 3; ++K) acc[13 + 3 * L + K].add(v[2 + L] * d[K]);
            }
        }
        R[V_F * kRedPitch + lane] = acc[0].value();
        R[V_N * kRedPitch + lane] = (double)nin;
#pragma unroll
        for (int L = 0; L < 3; ++L) {
            R[(V_S + L) * kRedPitch + lane] = acc[1 + L].value();
            R[(V_S2 + L) * kRedPitch + lane] = acc[4 + L].value();
            R[(V_G + L) * kRedPitch + lane] = acc[7 + L].value();
            R[(V_GF + L) * kRedPitch + lane] = acc[10 + L].value();
        }
#pragma unroll
        for (int i = 0; i < 9; ++i) R[(V_SR + i) * kRedPitch + lane] = acc[13 + i].value();
        const double mine = warp_column_sum(R, lane);

        // finalise shell s (ShellAnalysisGPU.jl:197-228)
        const double Fs = __shfl_sync(0xffffffffu, mine, V_F);
        const double ns = __shfl_sync(0xffffffffu, mine, V_N);
        const double rs = rad[s];
        const double dF = ns > 0.0 ? Fs / ns : 0.0;
        const double r3p = radp * radp * radp, r3 = rs * rs * rs;
        const double Fbar_s = (r3p * Fbarp + 0.5 * (dFbarp + dF) * (r3 - r3p)) / r3;
        const double r5 = rs * rs * rs * rs * rs;
        csrb += 0.5 * (Fbarp + Fbar_s) * (r5 - rad5p);

        // strain sums: lane 14 + 3L + K holds SR_LK; symmetrise with the partner KL
        const int srl = lane - V_SR;
        int partner = lane;
        if (srl >= 0 && srl < 9) partner = V_SR + 3 * (srl % 3) + srl / 3;
        const double norm = mine / rs;
        const double pnorm = __shfl_sync(0xffffffffu, norm, partner);
        double* q = P + (size_t)s * kRec;
        if (lane == V_F) q[P_FBAR] = Fbar_s;
        if (lane >= V_G && lane < V_G + 6) q[P_G + (lane - V_G)] = norm;   // G then Gf
        if (srl >= 0 && srl < 9) {
            const int L = srl / 3, K = srl % 3;
            int slot = -1;
            if (L == K) slot = L;                      // 11, 22, 33
            else if (L == 0 && K == 1) slot = 3;       // 12
            else if (L == 0 && K == 2) slot = 4;       // 13
            else if (L == 1 && K == 2) slot = 5;       // 23
            if (slot >= 0) q[P_SR + slot] = norm + pnorm;
        }
        if ((lane >= V_S && lane < V_S + 6) || lane == V_N) {
            cum += mine;
            const int slot = lane == V_N ? P_CN : P_CS + (lane - V_S);
            q[slot] = cum;
        }
        if (lane == 31) q[P_CSRB] = csrb;
        cells_in += (unsigned long long)ns;

        Fbarp = Fbar_s; dFbarp = dF; radp = rs; rad5p = r5;
        s_end = s;

        // early exit: stop once every shell the post-processing reads is present --
        // Fbar up to the crossing m_c, gradients/strain of shells within r < rad[m0]+2
        // plus the first shell beyond it (zvir_half windows), and the mrf window.
        if (m_c == 0 && s >= m0_init && Fbar_s < fcrit) {
            m_c = s;
            const int q2 = first_above(rad, s + 1, m, rad[s] + 2.0);
            stop_at = max(q2, need_rf);
        }
        if (s >= stop_at) break;
    }
    __syncwarp();
    if (lane == 0 && a.stats) {
        atomicAdd(a.stats, cells_in);
        atomicAdd(a.stats + 1, (unsigned long long)s_end);
    }

    // ------------------------------------------------------ post-processing ----
    // gradient at the filter scale (RadialShell.jl:466-482)
    double gradpkrf[3];
    {
        int lo, hi;
        if (mrf > 1) {
            lo = first_above(rad, 1, mrf, fmax(rad[mrf] - 2.0, 0.0));
            if (lo > mrf) lo = mrf;
        } else {
            lo = 1;
        }
        hi = max(mrf, last_below(rad, mrf, m, rad[mrf] + 2.0));
        Strain k = kernel_strain(P, rad, a.akk, mrf, lo, hi, a.wRnor, a.aRnor);
        gradpkrf[0] = k.g[0]; gradpkrf[1] = k.g[1]; gradpkrf[2] = k.g[2];
    }

    // crossing (RadialShell.jl:485-526)
    int m0 = m0_init;
    if (P[(size_t)m0 * kRec + P_FBAR] >= fcrit) {
        if (m_c != 0) m0 = m_c;   // else: no crossing, m0 stays, window up to m
    } else {
        // inward: first shell below m0_init (from the top) with Fbar >= fcrit
        int found = 0;
        for (int base = m0_init - 1; base >= 1 && !found; base -= 32) {
            const int mp = base - lane;
            const bool ge = mp >= 1 && P[(size_t)mp * kRec + P_FBAR] >= fcrit;
            const unsigned bal = __ballot_sync(0xffffffffu, ge);
            if (bal) {
                const int l = __ffs(bal) - 1;
                m0 = base - l + 1;
                found = 1;
            }
        }
        if (!found) { write_no_collapse(a, p, lane); return; }
    }

    // inward walk (RadialShell.jl:529-686): step t evaluates shell m0 - t; step 0 is
    // m0 itself with zvir forced to -1 (RadialShell.jl:566-567).  Lanes evaluate 32
    // consecutive steps at once; the first step with zvir >= ZZon collapses.  Step
    // results are staged in R (row = lane, row 32 = last step of the previous group).
    int tstar = -1, lrow = 0, prow = 0;
    for (int base = 0; base < m0; base += 32) {
        const int t = base + lane;
        double* row = R + lane * kStepW;
        bool hit = false;
        if (t < m0) {
            const Step st = eval_step(a, P, m0 - t, m, t == 0);
#pragma unroll
            for (int i = 0; i < 6; ++i) row[i] = st.k.E[i];
#pragma unroll
            for (int i = 0; i < 3; ++i) { row[6 + i] = st.k.g[i]; row[9 + i] = st.k.gf[i]; }
            row[12] = st.trace;
            row[13] = st.zvir;
            hit = st.zvir >= ZZon;
        }
        const unsigned bal = __ballot_sync(0xffffffffu, hit);
        __syncwarp();
        if (bal) {
            const int l = __ffs(bal) - 1;
            tstar = base + l;
            lrow = l;
            prow = l > 0 ? l - 1 : 32;
            break;
        }
        if (lane < 14) R[32 * kStepW + lane] = R[31 * kStepW + lane];
        __syncwarp();
    }
    if (tstar < 0 || (tstar == 0 && m0 == 1)) { write_no_collapse(a, p, lane); return; }
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
    if (RTHL <= 0.0) { write_no_collapse(a, p, lane); return; }

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
    // Sbar (RadialShell.jl:739-754) from the running sums at shell m0f - 1
    const double* qp = P + (size_t)(m0f - 1) * kRec;
    const double nS = qp[P_CN];
    // Srb (RadialShell.jl:757-771)
    double Srb = qp[P_CSRB];
    const double r5p = m0f - 1 >= 2 ? rp * rp * rp * rp * rp : 0.0;
    if (zvir1 > 0.0 && dZ != 0.0) Srb += 0.5 * (Fb_p + Fbarx) * (RTHL5 - r5p);
    if (Fbarx * RTHL5 > 0.0) Srb /= (Fbarx * RTHL5);

    // cells with r <= RTHL: shells 1..s_in form a contiguous prefix of the cell list
    const int s_in = last_le(rad, 1, nshells, RTHL);
    const int ncell_in = s_in >= 1 ? __ldg(a.start + s_in) + __ldg(a.count + s_in) : 0;

    // d2F
    double d2F = 0.0;
    if (a.lapd) {
        Kahan ks; ks.zero();
        int nloc = 0;
        if (a.conv == HT_CONV_GPU) {
            // all in-tile cells of shells with r <= RTHL, centre included
            // (ShellAnalysisGPU.jl:496-511)
            for (int c = lane; c < ncell_in; c += 32) {
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
            for (int base = 1; base < ncell_in; base += 32) {
                const int c = base + lane;
                bool oob = false;
                int iv1 = 0, iv2 = 0, iv3 = 0;
                if (c < ncell_in) {
                    const char4 o = __ldg(a.off + c);
                    iv1 = ci + o.x; iv2 = cj + o.y; iv3 = ck + o.z;
                    oob = iv1 < 1 || iv1 > a.n1 || iv2 < 1 || iv2 > a.n2 || iv3 < 1 || iv3 > a.n3;
                }
                const unsigned bal = __ballot_sync(0xffffffffu, oob);
                const int lim = bal ? __ffs(bal) - 1 : 32;
                if (c < ncell_in && lane < lim) {
                    const long long idx = (long long)(iv1 - 1) + (long long)a.n1 * (iv2 - 1) +
                                          a.s2 * (iv3 - 1);
                    ks.add(__ldg(a.lapd + idx));
                    ++nloc;
                }
                if (bal) break;
            }
        }
        const double tot = warp_sum(ks.value());
        const double nt = warp_sum((double)nloc);
        if (nt > 0.0) d2F = tot / nt;
    }

    // mask: core cells within RTHL (ShellAnalysisGPU.jl:513-528, RadialShell.jl:773-782)
    if (a.mask) {
        for (int c = lane; c < ncell_in; c += 32) {
            const char4 o = __ldg(a.off + c);
            const int iv1 = ci + o.x, iv2 = cj + o.y, iv3 = ck + o.z;
            if (iv1 > a.nbuff && iv1 <= a.n1 - a.nbuff && iv2 > a.nbuff &&
                iv2 <= a.n2 - a.nbuff && iv3 > a.nbuff && iv3 <= a.n3 - a.nbuff) {
                const long long idx = (long long)(iv1 - 1) + (long long)a.n1 * (iv2 - 1) +
                                      a.s2 * (iv3 - 1);
                a.mask[idx] = 1;
            }
        }
    }

    // zvir_half (RadialShell.jl:801-859): lane jj-1 handles radius jj
    double zvir_half = -1.0;
    if (RTHL >= 3.0) {
        double zl = -1.0;
        bool nan = false;
        if (lane < 10) {
            const double rcur = RTHL * pow(lane / 9.0 * 0.5 + 0.5, 1.0 / 3.0);
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
            const Strain k = kernel_strain(P, rad, a.akk, m0_rc, mlow_rc, mupp_rc, a.wRnor,
                                           a.aRnor);
            const Shape sh = shape_of(k.E);
            const double Fc = P[(size_t)m0_rc * kRec + P_FBAR];
            const double poe = sh.e_v < 1e-5 ? 0.0 : sh.p_v / sh.e_v;
            double z = -1.0;
            if (Fc > 0.0) z = interp3(a, log10(Fc), sh.e_v, poe);
            zl = z - 1.0;
            nan = isnan(zl);
        }
        // Julia's max propagates NaN
        const bool anynan = __any_sync(0xffffffffu, nan);
        double mx = zl;
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        zvir_half = anynan ? __longlong_as_double(0x7ff8000000000000ULL) : fmax(mx, -1.0);
    }

    // outputs
    const ht_results& o = a.out;
    if (lane == 0) {
        o.RTHL[p] = (float)RTHL;
        o.Fbarx[p] = (float)Fbarx;
        o.e_v[p] = (float)fin.e_v;
        o.p_v[p] = (float)fin.p_v;
        o.Srb[p] = (float)Srb;
        o.d2F[p] = (float)d2F;
        o.zvir_half[p] = (float)zvir_half;
    }
    if (lane < 9) {
        const int L = lane % 3, K = lane / 3;   // column-major (L, K)
        int idx6;
        if (L == K) idx6 = L;
        else if (L + K == 1) idx6 = 3;
        else if (L + K == 2) idx6 = 4;
        else idx6 = 5;
        o.strain[9 * p + lane] = (float)sfin[idx6];
    }
    if (lane < 3) {
        const double cs = qp[P_CS + lane], cs2 = qp[P_CS2 + lane];
        o.Sbar[3 * p + lane] = (float)(nS > 0.0 ? cs / nS : 0.0);
        o.Sbar2[3 * p + lane] = (float)(nS > 0.0 ? cs2 / nS : 0.0);
        o.gradpk[3 * p + lane] = (float)gpk[lane];
        o.gradpkf[3 * p + lane] = (float)gpkf[lane];
        o.gradpkrf[3 * p + lane] = (float)gradpkrf[lane];
        o.eigs[3 * p + lane] = (float)fin.lam[lane];
    }
}

template <bool PACKED>
__global__ void __launch_bounds__(kThreads) walk_kernel(const WalkArgs a) {
    extern __shared__ double smem[];
    const int lane = threadIdx.x & 31;
    double* R = smem + (threadIdx.x >> 5) * kWarpSmemDoubles;
    const long long gw = (long long)blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5);
    const long long nw = (long long)gridDim.x * kWarpsPerBlock;
    double* P = a.scratch + gw * a.scratch_stride;
    long long p;
    if (a.dynamic) {
        int q = 0;
        if (lane == 0) q = atomicAdd(a.queue, 1);
        p = __shfl_sync(0xffffffffu, q, 0);
    } else {
        p = gw;
    }
    while (p < a.npeaks) {
        process_peak<PACKED>(a, p, P, R, lane);
        __syncwarp();
        if (a.dynamic) {
            int q = 0;
            if (lane == 0) q = atomicAdd(a.queue, 1);
            p = __shfl_sync(0xffffffffu, q, 0);
        } else {
            p += nw;
        }
    }
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

int ht_launch_walk(ht_ctx* ctx, const ht_peak_batch* b, double alatt, double rmax2rs,
                   int32_t nbuff, int8_t* d_mask, int32_t conv, int32_t mode,
                   const ht_results* out, cudaStream_t st) {
    const bool packed = mode == HT_MODE_BATCHED;
    const size_t smem = (size_t)kWarpsPerBlock * kWarpSmemDoubles * sizeof(double);
    int bpsm = 0;
    cudaError_t e;
    if (packed) {
        e = cudaFuncSetAttribute(walk_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem);
        if (e == cudaSuccess)
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bpsm, walk_kernel<true>, kThreads,
                                                              smem);
    } else {
        e = cudaFuncSetAttribute(walk_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem);
        if (e == cudaSuccess)
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bpsm, walk_kernel<false>, kThreads,
                                                              smem);
    }
    if (e != cudaSuccess) return ht_cuda_fail(e, "occupancy query");
    if (bpsm < 1) bpsm = 1;
    long long blocks = (long long)ctx->num_sms * bpsm;
    const long long warps_needed = (b->npeaks + 0);
    if (!packed) {
        // static schedule: no more warps than peaks
        long long bl = (warps_needed + kWarpsPerBlock - 1) / kWarpsPerBlock;
        if (bl < blocks) blocks = bl;
    } else {
        long long bl = (warps_needed + kWarpsPerBlock - 1) / kWarpsPerBlock;
        if (bl < blocks) blocks = bl;
    }
    if (blocks < 1) blocks = 1;
    const long long nwarps = blocks * kWarpsPerBlock;
    const long long stride = (long long)(ctx->nshells + 2) * kRec;
    const size_t need = (size_t)nwarps * stride * sizeof(double);
    int rc = ht_grow((void**)&ctx->d_scratch, &ctx->scratch_bytes, need, "shell-walk scratch");
    if (rc != HT_OK) return rc;

    WalkArgs a;
    const ht_fields& f = ctx->fields;
    a.rec = ctx->d_rec;
    a.delta = f.delta; a.ex = f.etax; a.ey = f.etay; a.ez = f.etaz;
    a.e2x = f.eta2x; a.e2y = f.eta2y; a.e2z = f.eta2z; a.lapd = f.lapd;
    a.n1 = f.n1; a.n2 = f.n2; a.n3 = f.n3;
    a.s2 = (long long)f.n1 * f.n2;
    a.off = ctx->d_off; a.start = ctx->d_start; a.count = ctx->d_count; a.r2 = ctx->d_r2;
    a.rad = ctx->d_rad; a.nshells = ctx->nshells;
    a.ct = ctx->d_ct; a.nx = ctx->nx; a.ny = ctx->ny; a.nz = ctx->nz;
    a.X1 = ctx->X1; a.X2 = ctx->X2; a.Y1 = ctx->Y1; a.Y2 = ctx->Y2; a.Z1 = ctx->Z1;
    a.Z2 = ctx->Z2; a.out_val = ctx->out_val; a.akk = ctx->d_akk;
    a.pi = b->pi; a.pj = b->pj; a.pk = b->pk; a.Rf = b->Rf; a.ir2min = b->ir2min;
    a.ZZon = b->ZZon; a.fcrit = b->fcrit; a.npeaks = b->npeaks;
    a.alatt = alatt;
    const double pi = 3.14159265358979323846;
    a.aRnor = 3.0 / alatt;                   // RadialShell.jl:296-300 with hlatt = 1
    a.wRnor = 3.0 * (1.0 / (4.0 * pi)) / alatt;
    a.rmax2rs = rmax2rs; a.nbuff = nbuff; a.conv = conv; a.mask = d_mask; a.out = *out;
    a.scratch = ctx->d_scratch; a.scratch_stride = stride;
    a.queue = ctx->d_queue; a.dynamic = packed ? 1 : 0;
    a.stats = ctx->d_stats;

    HT_CUDA_TRY(cudaMemsetAsync(ctx->d_queue, 0, sizeof(int32_t), st), "queue reset");
    HT_CUDA_TRY(cudaMemsetAsync(ctx->d_stats, 0, 2 * sizeof(unsigned long long), st),
                "stats reset");
    if (packed) walk_kernel<true><<<(unsigned)blocks, kThreads, smem, st>>>(a);
    else walk_kernel<false><<<(unsigned)blocks, kThreads, smem, st>>>(a);
    HT_CUDA_TRY(cudaGetLastError(), "walk_kernel launch");
    ctx->last_kernels = 1;
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
// device current (a host-side name of a __device__ array is not a device address).
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
    // one 8-warp block must fit the static scratch
    const long long stride = (long long)(ctx->nshells + 2) * kRec;
    const size_t per_block = (size_t)kWarpsPerBlock * stride * sizeof(double);
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

    const size_t smem = (size_t)kWarpsPerBlock * kWarpSmemDoubles * sizeof(double);
    cudaError_t e = cudaFuncSetAttribute(walk_kernel<false>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return ht_cuda_fail(e, "cudaFuncSetAttribute");
    int bpsm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bpsm, walk_kernel<false>, kThreads, smem);
    if (e != cudaSuccess) return ht_cuda_fail(e, "occupancy query");
    long long blocks = (long long)ctx->num_sms * (bpsm > 0 ? bpsm : 1);
    const long long fit = (long long)(kStaticScratchBytes / per_block);
    const long long need = (b->npeaks + kWarpsPerBlock - 1) / kWarpsPerBlock;
    if (blocks > fit) blocks = fit;
    if (blocks > need) blocks = need;

    WalkArgs a;
    a.rec = nullptr;
    a.delta = f->delta; a.ex = f->etax; a.ey = f->etay; a.ez = f->etaz;
    a.e2x = f->eta2x; a.e2y = f->eta2y; a.e2z = f->eta2z; a.lapd = f->lapd;
    a.n1 = f->n1; a.n2 = f->n2; a.n3 = f->n3;
    a.s2 = (long long)f->n1 * f->n2;
    a.off = ctx->d_off; a.start = ctx->d_start; a.count = ctx->d_count; a.r2 = ctx->d_r2;
    a.rad = ctx->d_rad; a.nshells = ctx->nshells;
    a.ct = ctx->d_ct; a.nx = ctx->nx; a.ny = ctx->ny; a.nz = ctx->nz;
    a.X1 = ctx->X1; a.X2 = ctx->X2; a.Y1 = ctx->Y1; a.Y2 = ctx->Y2; a.Z1 = ctx->Z1;
    a.Z2 = ctx->Z2; a.out_val = ctx->out_val; a.akk = ctx->d_akk;
    a.pi = b->pi; a.pj = b->pj; a.pk = b->pk; a.Rf = b->Rf; a.ir2min = b->ir2min;
    a.ZZon = b->ZZon; a.fcrit = b->fcrit; a.npeaks = b->npeaks;
    a.alatt = alatt;
    const double pi = 3.14159265358979323846;
    a.aRnor = 3.0 / alatt;
    a.wRnor = 3.0 * (1.0 / (4.0 * pi)) / alatt;
    a.rmax2rs = rmax2rs; a.nbuff = nbuff; a.conv = conv; a.mask = d_mask; a.out = *out;
    a.scratch = (double*)scratch; a.scratch_stride = stride;
    a.queue = nullptr; a.dynamic = 0;   // static peak-to-warp schedule: no counter to clear
    a.stats = nullptr;
    walk_kernel<false><<<(unsigned)blocks, kThreads, smem, (cudaStream_t)stream>>>(a);
    HT_CUDA_TRY(cudaGetLastError(), "walk_kernel launch (static scratch)");
    ctx->last_kernels = 1;
    return HT_OK;
}
