// Lagrangian exclusion, volume reduction and the Eulerian finalisation of a halo catalog on
// the device (src/Merger/Merger.jl:38-104,114-146; src/Merger/Exclusion.jl:81-206).
//
// Exclusion.  The reference visits halos in decreasing radius (ties by x, y, z, then input
// order); a halo that is still alive kills every smaller halo whose centre lies inside its
// radius.  So a halo survives iff no surviving halo earlier in that order covers it, a
// recursive rule with a unique solution that can be settled in parallel rounds: a halo still
// undecided becomes dead when a halo decided alive covers it, and alive when no undecided or
// alive halo earlier in the order covers it.  Each round settles at least the first undecided
// halo, and every decision agrees with the sequential sweep, so the survivors are the same
// set.  Covering pairs are found through a uniform cell grid (halos sorted by cell): the
// search is exhaustive within each radius, as the reference's linked-list hash is.
//
// Volume reduction (optional, as in the reference): every overlapping pair of survivors,
// visited once from its earlier member, adds each its own cap volume (sphere_overlap) to a
// FP64 deficit; radii then shrink to keep r^3 - 3 dV / (4 pi).  The deficits are summed with
// atomics, so their last bits depend on the order of the additions (the reference sums in
// its sweep order); the exclusion itself is exact.
//
// FP64 arithmetic uses explicitly rounded operations (no contraction into FMAs), as the
// reference evaluates these expressions.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_reduce.cuh>
#include <cub/device/device_scan.cuh>
#include <cub/device/device_select.cuh>
#include <thrust/iterator/counting_iterator.h>
#include <math.h>

#include <algorithm>
#include <string>
#include <vector>

#include "ht_internal.cuh"

namespace {

constexpr double kPi = 3.141592653589793;

__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double ddiv(double a, double b) { return __ddiv_rn(a, b); }

// Float32 -> unsigned key with the same order (negatives reversed, then positives).
__device__ __forceinline__ uint32_t fkey(float v) {
    const uint32_t b = __float_as_uint(v);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

__device__ __forceinline__ double dist3(double ax, double ay, double az, double bx, double by,
                                        double bz) {
    const double dx = dsub(bx, ax), dy = dsub(by, ay), dz = dsub(bz, az);
    return __dsqrt_rn(dadd(dadd(dmul(dx, dx), dmul(dy, dy)), dmul(dz, dz)));
}

__global__ void extract_kernel(const float* __restrict__ rec, long long n, int width,
                               float* __restrict__ x, float* __restrict__ y,
                               float* __restrict__ z, float* __restrict__ r,
                               int32_t* __restrict__ idx) {
    const long long h = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= n) return;
    const float* q = rec + h * width;
    x[h] = q[0];
    y[h] = q[1];
    z[h] = q[2];
    r[h] = q[6];
    idx[h] = (int32_t)h;
}

// keys[q] = the sort key of component `which` of halo idx[q] (0..2: x, y, z ascending;
// 3: r descending)
__global__ void key_kernel(const float* __restrict__ v, const int32_t* __restrict__ idx,
                           long long n, bool descending, uint32_t* __restrict__ keys) {
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    const uint32_t k = fkey(v[idx[q]]);
    keys[q] = descending ? ~k : k;
}

struct Grid {
    double x0, y0, z0, cs;
    int nc;
};

__device__ __forceinline__ int cell1(double v, double v0, double cs, int nc) {
    // clamp(floor((v - v0) / cs) + 1, 1, nc) - 1  (Exclusion.jl:68-73, 0-based)
    const double t = floor(ddiv(dsub(v, v0), cs));
    return (int)fmin(fmax(t, 0.0), (double)(nc - 1));
}

// rank-ordered coordinates and the cell of each rank
__global__ void rank_kernel(const int32_t* __restrict__ order, long long n,
                            const float* __restrict__ x, const float* __restrict__ y,
                            const float* __restrict__ z, const float* __restrict__ r, Grid g,
                            float4* __restrict__ xyzr, uint32_t* __restrict__ cell,
                            int32_t* __restrict__ counts) {
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    const int h = order[q];
    const float4 v = make_float4(x[h], y[h], z[h], r[h]);
    xyzr[q] = v;
    const int cx = cell1(v.x, g.x0, g.cs, g.nc), cy = cell1(v.y, g.y0, g.cs, g.nc),
              cz = cell1(v.z, g.z0, g.cs, g.nc);
    const uint32_t c = ((uint32_t)cz * g.nc + cy) * g.nc + cx;
    cell[q] = c;
    atomicAdd(counts + c, 1);
}

__global__ void iota_kernel(int32_t* __restrict__ v, long long n) {
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q < n) v[q] = (int32_t)q;
}

enum : uint8_t { kUndecided = 0, kAlive = 1, kDead = 2 };

struct Nbr {
    const float4* xyzr;        // rank order
    const int32_t* cstart;     // nc^3 + 1
    const int32_t* list;       // ranks sorted by cell
    Grid g;
};

// Calls f(p) for every rank p > q (rank order) in the cells within `reach` of q's centre.
template <class F>
__device__ __forceinline__ void for_neighbours(const Nbr& nb, int q, double reach, F&& f) {
    const float4 v = nb.xyzr[q];
    const int dc = (int)ceil(ddiv(reach, nb.g.cs));
    const int cx = cell1(v.x, nb.g.x0, nb.g.cs, nb.g.nc), cy = cell1(v.y, nb.g.y0, nb.g.cs, nb.g.nc),
              cz = cell1(v.z, nb.g.z0, nb.g.cs, nb.g.nc);
    const int nc = nb.g.nc;
    for (int kz = max(cz - dc, 0); kz <= min(cz + dc, nc - 1); ++kz)
        for (int ky = max(cy - dc, 0); ky <= min(cy + dc, nc - 1); ++ky) {
            const long long row = ((long long)kz * nc + ky) * nc;
            const int b = nb.cstart[row + max(cx - dc, 0)];
            const int e = nb.cstart[row + min(cx + dc, nc - 1) + 1];
            for (int s = b; s < e; ++s) {
                const int p = nb.list[s];
                if (p > q) f(p);
            }
        }
}

// One exclusion round, push side: every undecided halo, and every halo made alive in the
// previous round, marks the undecided later halos it covers (blocked / killed).
__global__ void push_kernel(Nbr nb, long long n, const uint8_t* __restrict__ status,
                            const int32_t* __restrict__ alive_round, int round,
                            uint8_t* __restrict__ blocked, uint8_t* __restrict__ killed) {
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    const uint8_t sq = status[q];
    const bool fresh = sq == kAlive && alive_round[q] == round - 1;
    if (sq != kUndecided && !fresh) return;
    const float4 v = nb.xyzr[q];
    const double rq = v.w;
    for_neighbours(nb, (int)q, rq, [&](int p) {
        if (status[p] != kUndecided) return;
        const float4 w = nb.xyzr[p];
        if (dist3(v.x, v.y, v.z, w.x, w.y, w.z) < rq) {
            if (fresh) killed[p] = 1; else blocked[p] = 1;
        }
    });
}

__global__ void decide_kernel(long long n, uint8_t* __restrict__ status,
                              int32_t* __restrict__ alive_round, int round,
                              const uint8_t* __restrict__ blocked,
                              const uint8_t* __restrict__ killed,
                              unsigned long long* __restrict__ left) {
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n || status[p] != kUndecided) return;
    if (killed[p]) {
        status[p] = kDead;
    } else if (!blocked[p]) {
        status[p] = kAlive;
        alive_round[p] = round;
    } else {
        atomicAdd(left, 1ull);
    }
}

// Exclusion.sphere_overlap (Exclusion.jl:81-97)
__device__ __forceinline__ void sphere_overlap(double d, double r1, double r2, double* v1,
                                               double* v2) {
    *v1 = 0.0;
    *v2 = 0.0;
    if (d >= dadd(r1, r2) || d <= fabs(dsub(r1, r2))) return;
    const double h1 = ddiv(dmul(dadd(dsub(r2, r1), d), dsub(dadd(r2, r1), d)), dmul(2.0, d));
    const double h2 = ddiv(dmul(dadd(dsub(r1, r2), d), dsub(dadd(r1, r2), d)), dmul(2.0, d));
    *v1 = dmul(dmul(kPi / 3.0, dmul(h1, h1)), dsub(dmul(3.0, r1), h1));
    *v2 = dmul(dmul(kPi / 3.0, dmul(h2, h2)), dsub(dmul(3.0, r2), h2));
}

__global__ void overlap_kernel(Nbr nb, long long n, const uint8_t* __restrict__ status,
                               bool fortran_ties, double* __restrict__ dV) {
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n || status[q] != kAlive) return;
    const float4 v = nb.xyzr[q];
    const double rq = v.w;
    double acc = 0.0;
    for_neighbours(nb, (int)q, dmul(2.0, rq), [&](int p) {
        if (status[p] != kAlive) return;
        const float4 w = nb.xyzr[p];
        const double rp = w.w;
        const double d = dist3(v.x, v.y, v.z, w.x, w.y, w.z);
        if (d < dadd(rq, rp)) {
            double v1, v2;
            sphere_overlap(d, rq, rp, &v1, &v2);
            const double wt = (fortran_ties && rp == rq) ? 2.0 : 1.0;
            acc = dadd(acc, dmul(wt, v1));
            atomicAdd(dV + p, dmul(wt, v2));
        }
    });
    if (acc != 0.0) atomicAdd(dV + q, acc);
}

// New radius and survival by original index (Exclusion.jl:191-205; Merger.jl:79-85).
__global__ void radius_kernel(const int32_t* __restrict__ order, long long n,
                              const float4* __restrict__ xyzr, uint8_t* __restrict__ status,
                              const double* __restrict__ dV, bool reduce,
                              uint8_t* __restrict__ surv, float* __restrict__ new_r) {
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    const int h = order[q];
    const double r = xyzr[q].w;
    bool alive = status[q] == kAlive;
    float nr = (float)r;
    if (alive && reduce) {
        const double vol = dsub(dmul(4.0 * kPi / 3.0, dmul(dmul(r, r), r)), dV[q]);
        if (vol <= 0.0) {
            alive = false;
            nr = 0.0f;
        } else {
            nr = (float)cbrt(ddiv(dmul(vol, 3.0), 4.0 * kPi));
        }
    }
    surv[h] = alive ? 1 : 0;
    new_r[h] = nr;
}

__global__ void copy_survivors_kernel(const float* __restrict__ rec, int width,
                                      const int32_t* __restrict__ idx,
                                      const long long* __restrict__ nout,
                                      const float* __restrict__ new_r,
                                      float* __restrict__ out) {
    const long long h = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= *nout) return;
    const long long s = idx[h];
    for (int c = 0; c < width; ++c) out[h * width + c] = c == 6 ? new_r[s] : rec[s * width + c];
}

// Merger.finalize_eulerian (Merger.jl:114-146): Eulerian position q + d1 + d2, velocity
// a 100 E(a) f(a) (d1 + 2 d2) in km/s with f = dlnD/dlna of Dlinear_ab, the 2LPT fields
// zeroed; on a lightcone a = 1 / (1 + z(|x - obs|)).
struct EulerArgs {
    const double *chi, *zchi;
    int n_chi;
    double zmax;
    const double *atab, *dlnD;
    int ntab;
    double amintab, amaxtab, HD_Hainfty, HD_Ha0, Om, OL;
};

__device__ double chi_to_z_e(const EulerArgs& c, double chi) {
    if (chi <= c.chi[0]) return 0.0;
    if (chi >= c.chi[c.n_chi - 1]) return c.zmax;
    int lo = 0, hi = c.n_chi - 1;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (c.chi[mid] <= chi) lo = mid; else hi = mid;
    }
    const double frac = ddiv(dsub(chi, c.chi[lo]), dsub(c.chi[hi], c.chi[lo]));
    return dadd(c.zchi[lo], dmul(frac, dsub(c.zchi[hi], c.zchi[lo])));
}

// second value of Dlinear_ab: dlnD/dlna by the same Lagrange weights (Cosmology.jl:286-306)
__device__ double growth_f(const EulerArgs& c, double ai) {
    if (ai > c.amintab && ai < c.amaxtab) {
        const bool ascnd = c.atab[c.ntab - 1] > c.atab[0];
        int jlo = 0, jhi = c.ntab + 1;
        while (jhi - jlo > 1) {
            const int jm = (jhi + jlo) / 2;
            if ((ai > c.atab[jm - 1]) == ascnd) jlo = jm; else jhi = jm;
        }
        const int kk = jlo;
        int nlint, kkl;
        if (kk < 2 || kk >= c.ntab) { nlint = 2; kkl = max(kk - 1, 1); }
        else { nlint = 4; kkl = max(kk - 2, 1); }
        const double* xa = c.atab + (kkl - 1);
        const double* va = c.dlnD + (kkl - 1);
        if (nlint == 4) {
            auto coef = [&](int i, int a_, int b_, int c_) {
                double a = ddiv(dsub(ai, xa[a_]), dsub(xa[i], xa[a_]));
                a = ddiv(dmul(a, dsub(ai, xa[b_])), dsub(xa[i], xa[b_]));
                return ddiv(dmul(a, dsub(ai, xa[c_])), dsub(xa[i], xa[c_]));
            };
            const double a1 = coef(0, 1, 2, 3), a2 = coef(1, 0, 2, 3), a3 = coef(2, 0, 1, 3),
                         a4 = coef(3, 0, 1, 2);
            return dadd(dadd(dadd(dmul(a1, va[0]), dmul(a2, va[1])), dmul(a3, va[2])),
                        dmul(a4, va[3]));
        }
        const double a1 = ddiv(dsub(ai, xa[1]), dsub(xa[0], xa[1]));
        return dadd(dmul(a1, va[0]), dmul(dsub(1.0, a1), va[1]));
    }
    return ai >= c.amaxtab ? c.HD_Ha0 : c.HD_Hainfty;
}

__global__ void eulerian_kernel(float* __restrict__ rec, long long n, int width, EulerArgs c,
                                double ox, double oy, double oz, int ievol, double a_snap) {
    const long long h = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= n) return;
    float* q = rec + h * width;
    const double d1x = q[3], d1y = q[4], d1z = q[5], d2x = q[7], d2y = q[8], d2z = q[9];
    const double ex = dadd(dadd((double)q[0], d1x), d2x);
    const double ey = dadd(dadd((double)q[1], d1y), d2y);
    const double ez = dadd(dadd((double)q[2], d1z), d2z);
    double a = a_snap;
    if (ievol == 1) {
        const double r = dist3(ox, oy, oz, ex, ey, ez);
        a = r > 0.0 ? ddiv(1.0, dadd(1.0, chi_to_z_e(c, r))) : 1.0;
    }
    // E = sqrt(Om a^-3 + OL) with a^-3 = 1 / (a a a); vfac = ((a 100) E) f
    const double E = __dsqrt_rn(dadd(dmul(c.Om, ddiv(1.0, dmul(dmul(a, a), a))), c.OL));
    const double vfac = dmul(dmul(dmul(a, 100.0), E), growth_f(c, a));
    q[0] = (float)ex;
    q[1] = (float)ey;
    q[2] = (float)ez;
    q[3] = (float)dmul(vfac, dadd(d1x, dmul(2.0, d2x)));
    q[4] = (float)dmul(vfac, dadd(d1y, dmul(2.0, d2y)));
    q[5] = (float)dmul(vfac, dadd(d1z, dmul(2.0, d2z)));
    q[7] = 0.0f;
    q[8] = 0.0f;
    q[9] = 0.0f;
}

// carve `bytes` (256-aligned) from a workspace cursor
template <class T>
T* carve(char*& cur, size_t count) {
    T* p = (T*)cur;
    cur += ((count * sizeof(T)) + 255) & ~(size_t)255;
    return p;
}

}  // namespace

extern "C" HT_API int ht_merge_halos(ht_ctx* ctx, const float* d_records, int64_t nhalo,
                                     int32_t width, int32_t volume_reduction,
                                     int32_t fortran_ties, float* d_out, int64_t* d_nout,
                                     void* stream) {
    HT_RANGE("ht_merge_halos");
    if (!ctx || !d_nout || (nhalo > 0 && (!d_records || !d_out)))
        return ht_fail(HT_ERR_INVALID, "ht_merge_halos: NULL argument");
    if (width != 11 && width != 33)
        return ht_fail(HT_ERR_INVALID, "ht_merge_halos: width must be 11 or 33");
    if (nhalo < 0 || nhalo > 0x7fffffffLL)
        return ht_fail(HT_ERR_CAPACITY, "ht_merge_halos: nhalo must be in [0, 2^31)");
    if (ht_fault_injected("launch")) return ht_fail(HT_ERR_FAULT, "injected launch fault: ht_merge_halos");
    HT_CUDA_TRY(cudaSetDevice(ctx->device), "cudaSetDevice");
    cudaStream_t st = (cudaStream_t)stream;
    const long long n = nhalo;
    if (n == 0) {
        HT_CUDA_TRY(cudaMemsetAsync(d_nout, 0, sizeof(int64_t), st), "nout reset");
        return HT_OK;
    }
    const int ni = (int)n;
    const unsigned blocks = (unsigned)((n + 255) / 256);
    // ---- workspace: one layout pass sizes it (base 0), a second assigns the pointers ----
    size_t tb = 0, t1 = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, t1, (uint32_t*)nullptr, (uint32_t*)nullptr,
                                    (int32_t*)nullptr, (int32_t*)nullptr, ni, 0, 32, st);
    tb = std::max(tb, t1);
    t1 = 0;
    cub::DeviceReduce::Max(nullptr, t1, (float*)nullptr, (float*)nullptr, ni, st);
    tb = std::max(tb, t1);
    t1 = 0;
    thrust::counting_iterator<int32_t> it(0);
    cub::DeviceSelect::Flagged(nullptr, t1, it, (const uint8_t*)nullptr, (int32_t*)nullptr,
                               (long long*)nullptr, ni, st);
    tb = std::max(tb, t1);
    float *x, *y, *z, *r, *new_r, *ext;
    uint32_t *k0, *k1, *c0, *c1;
    int32_t *i0, *i1, *l0, *l1, *alive_round, *sidx;
    float4* xyzr;
    uint8_t* flags;
    double* dV;
    void* temp;
    auto layout = [&](char* base) {
        char* cur = base;
        x = carve<float>(cur, n);
        y = carve<float>(cur, n);
        z = carve<float>(cur, n);
        r = carve<float>(cur, n);
        k0 = carve<uint32_t>(cur, n);
        k1 = carve<uint32_t>(cur, n);
        i0 = carve<int32_t>(cur, n);
        i1 = carve<int32_t>(cur, n);
        xyzr = carve<float4>(cur, n);
        c0 = carve<uint32_t>(cur, n);
        c1 = carve<uint32_t>(cur, n);
        l0 = carve<int32_t>(cur, n);
        l1 = carve<int32_t>(cur, n);
        alive_round = carve<int32_t>(cur, n);
        flags = carve<uint8_t>(cur, 4 * (size_t)n);
        dV = carve<double>(cur, n);
        new_r = carve<float>(cur, n);
        sidx = carve<int32_t>(cur, n);
        ext = carve<float>(cur, 16);   // 8 extents, then a 64-bit counter at ext + 8
        temp = carve<char>(cur, tb);
        return (size_t)(cur - base);
    };
    const size_t need = layout((char*)nullptr) + 256;
    int rc = ht_grow(&ctx->d_merge_ws, &ctx->merge_ws_bytes, need, "merge workspace");
    if (rc != HT_OK) return rc;
    layout((char*)ctx->d_merge_ws);
    uint8_t *status = flags, *blocked = flags + n, *killed = flags + 2 * n, *surv = flags + 3 * n;
    unsigned long long* left = (unsigned long long*)(ext + 8);

    extract_kernel<<<blocks, 256, 0, st>>>(d_records, n, width, x, y, z, r, i0);
    HT_CUDA_TRY(cudaGetLastError(), "extract_kernel launch");
    // ---- order: (-r, x, y, z) ascending, stable: LSD passes z, y, x, r ----
    const float* comp[4] = {z, y, x, r};
    int32_t* ia = i0;
    int32_t* ib = i1;
    for (int pass = 0; pass < 4; ++pass) {
        key_kernel<<<blocks, 256, 0, st>>>(comp[pass], ia, n, pass == 3, k0);
        HT_CUDA_TRY(cudaGetLastError(), "key_kernel launch");
        size_t t = tb;
        HT_CUDA_TRY(cub::DeviceRadixSort::SortPairs(temp, t, k0, k1, ia, ib, ni, 0, 32, st),
                    "cub::DeviceRadixSort::SortPairs (order)");
        std::swap(ia, ib);
    }
    const int32_t* order = ia;   // order[q] = original index of rank q
    // ---- grid: extents padded by 2 rmax (Merger.jl:48-56), about one halo per cell ----
    for (int a = 0; a < 4; ++a) {
        size_t t = tb;
        HT_CUDA_TRY(cub::DeviceReduce::Min(temp, t, comp[a], ext + a, ni, st), "cub::DeviceReduce::Min");
        t = tb;
        HT_CUDA_TRY(cub::DeviceReduce::Max(temp, t, comp[a], ext + 4 + a, ni, st), "cub::DeviceReduce::Max");
    }
    float hx[8];
    HT_CUDA_TRY(cudaMemcpyAsync(hx, ext, sizeof hx, cudaMemcpyDeviceToHost, st), "extent copy");
    HT_CUDA_TRY(cudaStreamSynchronize(st), "extent sync");
    // hx: min z, y, x, r, max z, y, x, r
    const double rmax = hx[7], pad = 2.0 * rmax;
    const double lo[3] = {hx[2] - pad, hx[1] - pad, hx[0] - pad};
    const double hi[3] = {hx[6] + pad, hx[5] + pad, hx[4] + pad};
    const double L = std::max({hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]});
    const int nc = std::min(std::max((int)std::lround(std::cbrt((double)n)), 16), 1024);
    const size_t ncell = (size_t)nc * nc * nc;
    if (!(L > 0.0) || !(rmax >= 0.0))
        return ht_fail(HT_ERR_INVALID, "ht_merge_halos: positions or radii are not finite");
    Grid g{lo[0], lo[1], lo[2], L / nc, nc};
    rc = ht_grow(&ctx->d_merge_cells, &ctx->merge_cells_bytes, (2 * ncell + 2) * sizeof(int32_t),
                 "merge cell table");
    if (rc != HT_OK) return rc;
    int32_t* counts = (int32_t*)ctx->d_merge_cells;
    int32_t* cstart = counts + ncell + 1;
    HT_CUDA_TRY(cudaMemsetAsync(counts, 0, (ncell + 1) * sizeof(int32_t), st), "cell counts reset");
    rank_kernel<<<blocks, 256, 0, st>>>(order, n, x, y, z, r, g, xyzr, c0, counts);
    HT_CUDA_TRY(cudaGetLastError(), "rank_kernel launch");
    {
        size_t t = 0;
        cub::DeviceScan::ExclusiveSum(nullptr, t, counts, cstart, (int)(ncell + 1), st);
        void* scan_temp = nullptr;
        // the scan runs over the cell table: temp from the generic workspace if it fits
        rc = HT_OK;
        if (t <= tb) {
            scan_temp = temp;
        } else {
            rc = ht_grow(&ctx->d_merge_scan, &ctx->merge_scan_bytes, t, "merge scan temp");
            scan_temp = ctx->d_merge_scan;
        }
        if (rc != HT_OK) return rc;
        HT_CUDA_TRY(cub::DeviceScan::ExclusiveSum(scan_temp, t, counts, cstart, (int)(ncell + 1), st),
                    "cub::DeviceScan::ExclusiveSum");
    }
    iota_kernel<<<blocks, 256, 0, st>>>(l0, n);
    HT_CUDA_TRY(cudaGetLastError(), "iota_kernel launch");
    {
        size_t t = tb;
        int bits = 1;
        while (bits < 32 && (1ull << bits) < ncell) ++bits;
        HT_CUDA_TRY(cub::DeviceRadixSort::SortPairs(temp, t, c0, c1, l0, l1, ni, 0, bits, st),
                    "cub::DeviceRadixSort::SortPairs (cells)");
    }
    Nbr nb{xyzr, cstart, l1, g};
    // ---- exclusion rounds ----
    HT_CUDA_TRY(cudaMemsetAsync(status, kUndecided, n, st), "status reset");
    HT_CUDA_TRY(cudaMemsetAsync(alive_round, 0xff, n * sizeof(int32_t), st), "rounds reset");
    int rounds = 0;
    for (int round = 0;; ++round) {
        HT_CUDA_TRY(cudaMemsetAsync(blocked, 0, 2 * (size_t)n, st), "marks reset");
        HT_CUDA_TRY(cudaMemsetAsync(left, 0, sizeof(unsigned long long), st), "counter reset");
        push_kernel<<<blocks, 256, 0, st>>>(nb, n, status, alive_round, round, blocked, killed);
        HT_CUDA_TRY(cudaGetLastError(), "push_kernel launch");
        decide_kernel<<<blocks, 256, 0, st>>>(n, status, alive_round, round, blocked, killed, left);
        HT_CUDA_TRY(cudaGetLastError(), "decide_kernel launch");
        unsigned long long h_left = 0;
        HT_CUDA_TRY(cudaMemcpyAsync(&h_left, left, sizeof h_left, cudaMemcpyDeviceToHost, st),
                    "round counter copy");
        HT_CUDA_TRY(cudaStreamSynchronize(st), "round sync");
        rounds = round + 1;
        if (h_left == 0) {
            // the halos made alive in this last round still kill in the next push, but
            // every halo is decided: nothing is left to kill
            break;
        }
        if (round > ni) return ht_fail(HT_ERR_STATE, "ht_merge_halos: exclusion did not settle");
    }
    // ---- volume reduction ----
    const bool reduce = volume_reduction != 0;
    if (reduce) {
        HT_CUDA_TRY(cudaMemsetAsync(dV, 0, n * sizeof(double), st), "dV reset");
        overlap_kernel<<<blocks, 256, 0, st>>>(nb, n, status, fortran_ties != 0, dV);
        HT_CUDA_TRY(cudaGetLastError(), "overlap_kernel launch");
    }
    radius_kernel<<<blocks, 256, 0, st>>>(order, n, xyzr, status, dV, reduce, surv, new_r);
    HT_CUDA_TRY(cudaGetLastError(), "radius_kernel launch");
    {
        size_t t = tb;
        HT_CUDA_TRY(cub::DeviceSelect::Flagged(temp, t, it, surv, sidx, (long long*)d_nout, ni, st),
                    "cub::DeviceSelect::Flagged (survivors)");
    }
    copy_survivors_kernel<<<blocks, 256, 0, st>>>(d_records, width, sidx,
                                                  (const long long*)d_nout, new_r, d_out);
    HT_CUDA_TRY(cudaGetLastError(), "copy_survivors_kernel launch");
    ctx->last_kernels = 2 * rounds + 8;
    return HT_OK;
}

extern "C" HT_API int ht_finalize_eulerian(ht_ctx* ctx, float* d_records, int64_t nhalo,
                                           int32_t width, const double* obs, int32_t ievol,
                                           double z_out, void* stream) {
    HT_RANGE("ht_finalize_eulerian");
    if (!ctx || (nhalo > 0 && !d_records) || (ievol == 1 && !obs))
        return ht_fail(HT_ERR_INVALID, "ht_finalize_eulerian: NULL argument");
    if (width != 11 && width != 33)
        return ht_fail(HT_ERR_INVALID, "ht_finalize_eulerian: width must be 11 or 33");
    if (!ctx->cosmo_set) return ht_fail(HT_ERR_STATE, "ht_finalize_eulerian: call ht_ctx_set_cosmo first");
    if (nhalo < 0) return ht_fail(HT_ERR_INVALID, "ht_finalize_eulerian: nhalo < 0");
    if (ht_fault_injected("launch")) return ht_fail(HT_ERR_FAULT, "injected launch fault: ht_finalize_eulerian");
    HT_CUDA_TRY(cudaSetDevice(ctx->device), "cudaSetDevice");
    if (nhalo == 0) return HT_OK;
    EulerArgs c{ctx->d_chi, ctx->d_zchi, ctx->n_chi, ctx->cosmo_zmax, ctx->d_atab, ctx->d_dlnD,
                ctx->ntab, ctx->amintab, ctx->amaxtab, ctx->HD_Hainfty, ctx->HD_Ha0,
                ctx->cosmo_Om, ctx->cosmo_OL};
    const double a_snap = 1.0 / (1.0 + z_out);
    eulerian_kernel<<<(unsigned)((nhalo + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
        d_records, nhalo, width, c, ievol == 1 ? obs[0] : 0.0, ievol == 1 ? obs[1] : 0.0,
        ievol == 1 ? obs[2] : 0.0, ievol, a_snap);
    HT_CUDA_TRY(cudaGetLastError(), "eulerian_kernel launch");
    ctx->last_kernels = 1;
    return HT_OK;
}
