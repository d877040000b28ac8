// Per-peak lightcone state and halo-record packing on the device: the host loops of
// MultiResolution.jl:1097-1130 (redshift, ZZon and fcrit of every peak seen from the
// observer, and the z <= z_max cut) and :1159-1219 (HaloRecord / ExtHaloRecord rows of the
// collapsed peaks, src/IO/Catalog.jl:4-48), one thread per peak.
//
// All FP64 arithmetic here is written with explicitly rounded operations (__dmul_rn,
// __dadd_rn, ...) so that the compiler forms no fused multiply-adds: the results are the
// IEEE results of the reference's operation order, which is what the host-side restatement
// computes too.  Order-preserving compaction (cub::DeviceSelect::Flagged) keeps the kept
// peaks and the halos in peak order.
#include <cub/device/device_select.cuh>
#include <thrust/iterator/counting_iterator.h>
#include <math.h>

#include <algorithm>
#include <string>

#include "ht_internal.cuh"

namespace {

struct CosmoDev {
    const double *chi, *zchi;
    int n_chi;
    double zmax;
    const double *atab, *Da, *dlnD;
    int ntab;
    double amintab, amaxtab, D_ainfty, D_a0, HD_Hainfty, HD_Ha0, Om, OL;
};

struct TableDev {   // collapse table (CollapseTable.jl:119-138)
    const float* ct;
    int nx, ny, nz;
    double X1, X2, Y1, Y2, Z1, Z2, out_val;
};

__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double ddiv(double a, double b) { return __ddiv_rn(a, b); }

// Cell centre along one axis: c0 + alatt (i - (n + 1)/2) (ext/CUDAExt.jl:3039-3046).
__device__ __forceinline__ double cell_centre(double c0, double alatt, int i, double cen1) {
    return dadd(c0, dmul(alatt, dsub((double)i, cen1)));
}

// chi_to_z (Cosmology.jl:354-371): clamp, bisection on the ascending chi table, linear
// interpolation in z.
__device__ double chi_to_z(const CosmoDev& c, double chi) {
    if (chi <= __ldg(c.chi)) return 0.0;
    if (chi >= __ldg(c.chi + c.n_chi - 1)) return c.zmax;
    int lo = 0, hi = c.n_chi - 1;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(c.chi + mid) <= chi) lo = mid; else hi = mid;
    }
    const double clo = __ldg(c.chi + lo), chi_hi = __ldg(c.chi + hi);
    const double zlo = __ldg(c.zchi + lo), zhi = __ldg(c.zchi + hi);
    const double frac = ddiv(dsub(chi, clo), dsub(chi_hi, clo));
    return dadd(zlo, dmul(frac, dsub(zhi, zlo)));
}

// Trilinear lookup with -1 outside the closed box (CollapseTable.jl:126-138), FP64 over
// the Float32 table, in the order of the host restatement.
__device__ double table_interp(const TableDev& t, double x, double y, double z) {
    if (!(x >= t.X1 && x <= t.X2 && y >= t.Y1 && y <= t.Y2 && z >= t.Z1 && z <= t.Z2))
        return t.out_val;
    const double tx = ddiv(dsub(x, t.X1), ddiv(dsub(t.X2, t.X1), (double)(t.nx - 1)));
    const double ty = ddiv(dsub(y, t.Y1), ddiv(dsub(t.Y2, t.Y1), (double)(t.ny - 1)));
    const double tz = ddiv(dsub(z, t.Z1), ddiv(dsub(t.Z2, t.Z1), (double)(t.nz - 1)));
    const int ix = min(max((int)floor(tx), 0), t.nx - 2);
    const int iy = min(max((int)floor(ty), 0), t.ny - 2);
    const int iz = min(max((int)floor(tz), 0), t.nz - 2);
    const double fx = dsub(tx, ix), fy = dsub(ty, iy), fz = dsub(tz, iz);
    const long long sy = t.nx, sz = (long long)t.nx * t.ny;
    const float* p = t.ct + ix + iy * sy + iz * sz;
    auto lerp = [](double a, double b, double f) {
        return dadd(dmul(a, dsub(1.0, f)), dmul(b, f));
    };
    const double c00 = lerp(__ldg(p), __ldg(p + 1), fx);
    const double c10 = lerp(__ldg(p + sy), __ldg(p + 1 + sy), fx);
    const double c01 = lerp(__ldg(p + sz), __ldg(p + 1 + sz), fx);
    const double c11 = lerp(__ldg(p + sy + sz), __ldg(p + 1 + sy + sz), fx);
    return lerp(lerp(c00, c10, fy), lerp(c01, c11, fy), fz);
}

// fsc_of_z (RadialShell.jl:181-195): 50 bisection steps of zvir(log10 F, 0, 0) = 1 + z.
__device__ double fsc_of_z(const TableDev& t, double z) {
    const double target = dadd(1.0, z);
    double lo = t.X1, hi = t.X2;
    for (int it = 0; it < 50; ++it) {
        const double mid = dmul(0.5, dadd(lo, hi));
        if (table_interp(t, mid, 0.0, 0.0) > target) hi = mid; else lo = mid;
    }
    return pow(10.0, lo);
}

// _hunt (Cosmology.jl:117-132): 1-based jlo with xx[jlo] < x <= xx[jlo + 1], 0 .. n.
__device__ int hunt(const double* xx, int n, double x) {
    const bool ascnd = __ldg(xx + n - 1) > __ldg(xx);
    int jlo = 0, jhi = n + 1;
    while (jhi - jlo > 1) {
        const int jm = (jhi + jlo) / 2;
        if ((x > __ldg(xx + jm - 1)) == ascnd) jlo = jm; else jhi = jm;
    }
    return jlo;
}

// Dlinear_ab's D(a) (Cosmology.jl:286-306 with _lagrint_2col, :97-115): 4-point Lagrange
// interpolation of D(a)/a around a (2-point at the table ends), times a; constant D/a
// outside the table.  The 4-point window starts two entries below the bracketing one, as
// in the reference; a window that would start before the first entry (a in the second
// table interval, z ~ 900) is moved to start at it.
__device__ double growth_D(const CosmoDev& c, double ai) {
    if (ai > c.amintab && ai < c.amaxtab) {
        const int kk = hunt(c.atab, c.ntab, ai);
        int nlint, kkl;
        if (kk < 2 || kk >= c.ntab) {
            nlint = 2;
            kkl = max(kk - 1, 1);
        } else {
            nlint = 4;
            kkl = max(kk - 2, 1);
        }
        const double* xa = c.atab + (kkl - 1);
        const double* va = c.Da + (kkl - 1);
        double p;
        if (nlint == 4) {
            const double x1 = __ldg(xa), x2 = __ldg(xa + 1), x3 = __ldg(xa + 2), x4 = __ldg(xa + 3);
            // ((((x - x2) / (x1 - x2)) * (x - x3)) / (x1 - x3)) * (x - x4) / (x1 - x4), ...
            auto coef = [&](double xi, double xa_, double xb, double xc) {
                double a = ddiv(dsub(ai, xa_), dsub(xi, xa_));
                a = ddiv(dmul(a, dsub(ai, xb)), dsub(xi, xb));
                return ddiv(dmul(a, dsub(ai, xc)), dsub(xi, xc));
            };
            const double a1 = coef(x1, x2, x3, x4), a2 = coef(x2, x1, x3, x4);
            const double a3 = coef(x3, x1, x2, x4), a4 = coef(x4, x1, x2, x3);
            p = dadd(dadd(dadd(dmul(a1, __ldg(va)), dmul(a2, __ldg(va + 1))),
                          dmul(a3, __ldg(va + 2))),
                     dmul(a4, __ldg(va + 3)));
        } else {
            const double x1 = __ldg(xa), x2 = __ldg(xa + 1);
            const double a1 = ddiv(dsub(ai, x2), dsub(x1, x2));
            const double a2 = dsub(1.0, a1);
            p = dadd(dmul(a1, __ldg(va)), dmul(a2, __ldg(va + 1)));
        }
        return dmul(p, ai);
    }
    if (ai >= c.amaxtab) return dmul(c.D_a0, ai);
    return dmul(c.D_ainfty, ai);
}

__global__ void lightcone_kernel(const int32_t* __restrict__ pi, const int32_t* __restrict__ pj,
                                 const int32_t* __restrict__ pk, long long npeaks,
                                 ht_tile_geom g, double ox, double oy, double oz, double z_max,
                                 CosmoDev c, TableDev t, double* __restrict__ zout,
                                 float* __restrict__ ZZon, float* __restrict__ fcrit,
                                 uint8_t* __restrict__ flag) {
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= npeaks) return;
    const double cen1 = dmul(0.5, (double)(g.n + 1));
    const double x = cell_centre(g.xbx, g.alatt, __ldg(pi + p), cen1);
    const double y = cell_centre(g.ybx, g.alatt, __ldg(pj + p), cen1);
    const double zc = cell_centre(g.zbx, g.alatt, __ldg(pk + p), cen1);
    // peak_redshift (Cosmology.jl:376-385)
    const double dx = dsub(x, ox), dy = dsub(y, oy), dz = dsub(zc, oz);
    const double r = __dsqrt_rn(dadd(dadd(dmul(dx, dx), dmul(dy, dy)), dmul(dz, dz)));
    const double z = chi_to_z(c, r);
    if (zout) zout[p] = z;
    ZZon[p] = (float)dadd(1.0, z);
    fcrit[p] = (float)fsc_of_z(t, z);
    flag[p] = z <= z_max ? 1 : 0;
}

__global__ void halo_flag_kernel(const float* __restrict__ RTHL, const double* __restrict__ z,
                                 long long npeaks, double z_max, uint8_t* __restrict__ flag) {
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= npeaks) return;
    // the reference skips `RTHL <= 0` and `z > z_max` (a NaN passes both tests)
    bool keep = !(__ldg(RTHL + p) <= 0.0f);
    if (z) keep = keep && !(__ldg(z + p) > z_max);
    flag[p] = keep ? 1 : 0;
}

struct PackArgs {
    ht_catalog_peaks pk;
    ht_results r;
    ht_tile_geom g;
    double ZZon;
    int ilpt, width;
    long long cap;
    const int32_t* idx;        // kept peak indices, in order
    const long long* nhalo;    // their number (device)
    float* out;
};

__global__ void halo_record_kernel(PackArgs a, CosmoDev c) {
    const long long h = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= *a.nhalo || h >= a.cap) return;
    const long long p = __ldg(a.idx + h);
    const ht_results& r = a.r;
    const double cen1 = dmul(0.5, (double)(a.g.n + 1));
    const double x = cell_centre(a.g.xbx, a.g.alatt, __ldg(a.pk.i + p), cen1);
    const double y = cell_centre(a.g.ybx, a.g.alatt, __ldg(a.pk.j + p), cen1);
    const double zc = cell_centre(a.g.zbx, a.g.alatt, __ldg(a.pk.k + p), cen1);
    const double ZZon_pk = a.pk.z ? dadd(1.0, __ldg(a.pk.z + p)) : a.ZZon;
    const double a_pk = ddiv(1.0, ZZon_pk);
    const double D_pk = growth_D(c, a_pk);
    const float D32 = (float)D_pk;
    float* o = a.out + h * a.width;
    o[0] = (float)x;
    o[1] = (float)y;
    o[2] = (float)zc;
    o[3] = __fmul_rn(r.Sbar[3 * p], D32);
    o[4] = __fmul_rn(r.Sbar[3 * p + 1], D32);
    o[5] = __fmul_rn(r.Sbar[3 * p + 2], D32);
    o[6] = (float)dmul((double)r.RTHL[p], a.g.alatt);
    float s2c = 0.0f;
    const bool lpt2 = a.ilpt >= 2;
    if (lpt2) {
        // -3/7 Om(a)^(-1/143) D^2, Om(a) = (Om/a^3)/(Om/a^3 + OL) (MultiResolution.jl:1178-1181)
        const double a3 = dmul(dmul(a_pk, a_pk), a_pk);
        const double oma = ddiv(ddiv(c.Om, a3), dadd(ddiv(c.Om, a3), c.OL));
        s2c = (float)dmul(dmul(-3.0 / 7.0, pow(oma, -1.0 / 143)), dmul(D_pk, D_pk));
    }
    o[7] = lpt2 ? __fmul_rn(r.Sbar2[3 * p], s2c) : 0.0f;
    o[8] = lpt2 ? __fmul_rn(r.Sbar2[3 * p + 1], s2c) : 0.0f;
    o[9] = lpt2 ? __fmul_rn(r.Sbar2[3 * p + 2], s2c) : 0.0f;
    o[10] = r.Fbarx[p];
    if (a.width == 11) return;
    o[11] = r.e_v[p];
    o[12] = r.p_v[p];
    const float* st = r.strain + 9 * p;    // column-major (3, 3): (L, K) at L + 3 K
    o[13] = st[0];                           // (1,1)
    o[14] = st[4];                           // (2,2)
    o[15] = st[8];                           // (3,3)
    o[16] = st[7];                           // (2,3)
    o[17] = st[6];                           // (1,3)
    o[18] = st[3];                           // (1,2)
    o[19] = r.d2F[p];
    o[20] = r.zvir_half[p];
    for (int l = 0; l < 3; ++l) {
        o[21 + l] = r.gradpk[3 * p + l];
        o[24 + l] = r.gradpkf[3 * p + l];
        o[30 + l] = r.gradpkrf[3 * p + l];
    }
    o[27] = (float)__ldg(a.pk.Rf + p);
    o[28] = __ldg(a.pk.FcRf + p);
    o[29] = a.pk.d2Rf ? __ldg(a.pk.d2Rf + p) : 0.0f;
}

CosmoDev cosmo_of(const ht_ctx* ctx) {
    return CosmoDev{ctx->d_chi, ctx->d_zchi, ctx->n_chi, ctx->cosmo_zmax, ctx->d_atab,
                    ctx->d_Da, ctx->d_dlnD, ctx->ntab, ctx->amintab, ctx->amaxtab,
                    ctx->D_ainfty, ctx->D_a0, ctx->HD_Hainfty, ctx->HD_Ha0, ctx->cosmo_Om,
                    ctx->cosmo_OL};
}

// Workspace for npeaks: flags, the compacted index list and CUB's temp storage.
int catalog_workspace(ht_ctx* ctx, long long npeaks, uint8_t** flags, int32_t** idx,
                      void** temp, size_t* temp_bytes) {
    size_t tb = 0;
    thrust::counting_iterator<int32_t> it(0);
    cudaError_t e = cub::DeviceSelect::Flagged(nullptr, tb, it, (const uint8_t*)nullptr,
                                               (int32_t*)nullptr, (long long*)nullptr,
                                               (int)npeaks);
    if (e != cudaSuccess) return ht_cuda_fail(e, "cub::DeviceSelect::Flagged (size)");
    const size_t fb = ((size_t)npeaks + 255) & ~(size_t)255;
    const size_t ib = ((size_t)npeaks * 4 + 255) & ~(size_t)255;
    int rc = ht_grow(&ctx->d_cat_ws, &ctx->cat_ws_bytes, fb + ib + tb + 256, "catalog workspace");
    if (rc != HT_OK) return rc;
    char* base = (char*)ctx->d_cat_ws;
    *flags = (uint8_t*)base;
    *idx = (int32_t*)(base + fb);
    *temp = base + fb + ib;
    *temp_bytes = tb;
    return HT_OK;
}

}  // namespace

extern "C" HT_API int ht_ctx_set_cosmo(ht_ctx* ctx, const ht_cosmo* c) {
    HT_RANGE("ht_ctx_set_cosmo");
    if (!ctx || !c) return ht_fail(HT_ERR_INVALID, "ht_ctx_set_cosmo: NULL argument");
    if (!c->chi || !c->zchi || c->n_chi < 2 || !c->atab || !c->D_atab || !c->dlnD_dlna ||
        c->ntab < 4)
        return ht_fail(HT_ERR_INVALID, "ht_ctx_set_cosmo: need n_chi >= 2 and ntab >= 4 tables");
    for (int q = 1; q < c->n_chi; ++q)
        if (!(c->chi[q] > c->chi[q - 1]))
            return ht_fail(HT_ERR_INVALID, "ht_ctx_set_cosmo: chi table must be ascending");
    for (int q = 1; q < c->ntab; ++q)
        if (!(c->atab[q] > c->atab[q - 1]))
            return ht_fail(HT_ERR_INVALID, "ht_ctx_set_cosmo: a table must be ascending");
    if (ht_fault_injected("alloc")) return ht_fail(HT_ERR_FAULT, "injected allocation fault: cosmology tables");
    HT_CUDA_TRY(cudaSetDevice(ctx->device), "cudaSetDevice");
    double** dst[5] = {&ctx->d_chi, &ctx->d_zchi, &ctx->d_atab, &ctx->d_Da, &ctx->d_dlnD};
    const double* src[5] = {c->chi, c->zchi, c->atab, c->D_atab, c->dlnD_dlna};
    const int cnt[5] = {c->n_chi, c->n_chi, c->ntab, c->ntab, c->ntab};
    for (int q = 0; q < 5; ++q) {
        if (*dst[q]) { cudaFree(*dst[q]); *dst[q] = nullptr; }
        int rc = ht_alloc((void**)dst[q], (size_t)cnt[q] * sizeof(double), "cosmology table");
        if (rc != HT_OK) return rc;
        HT_CUDA_TRY(cudaMemcpy(*dst[q], src[q], (size_t)cnt[q] * sizeof(double),
                               cudaMemcpyHostToDevice), "cosmology table upload");
    }
    ctx->n_chi = c->n_chi;
    ctx->cosmo_zmax = c->z_max;
    ctx->ntab = c->ntab;
    ctx->amintab = c->amintab;
    ctx->amaxtab = c->amaxtab;
    ctx->D_ainfty = c->D_ainfty;
    ctx->D_a0 = c->D_a0;
    ctx->HD_Hainfty = c->HD_Hainfty;
    ctx->HD_Ha0 = c->HD_Ha0;
    ctx->cosmo_Om = c->Om;
    ctx->cosmo_OL = c->OL;
    ctx->cosmo_set = true;
    return HT_OK;
}

extern "C" HT_API int ht_peak_lightcone(ht_ctx* ctx, const int32_t* d_i, const int32_t* d_j,
                                        const int32_t* d_k, int64_t npeaks,
                                        const ht_tile_geom* geom, const double* obs,
                                        double z_max, double* d_z, float* d_ZZon,
                                        float* d_fcrit, int32_t* d_keep, int64_t* d_nkeep,
                                        void* stream) {
    HT_RANGE("ht_peak_lightcone");
    if (!ctx || !geom || !obs || !d_ZZon || !d_fcrit || !d_keep || !d_nkeep ||
        (npeaks > 0 && (!d_i || !d_j || !d_k)))
        return ht_fail(HT_ERR_INVALID, "ht_peak_lightcone: NULL argument");
    if (!ctx->cosmo_set) return ht_fail(HT_ERR_STATE, "ht_peak_lightcone: call ht_ctx_set_cosmo first");
    if (npeaks < 0 || npeaks > 0x7fffffffLL)
        return ht_fail(HT_ERR_CAPACITY, "ht_peak_lightcone: npeaks must be in [0, 2^31)");
    if (geom->n < 1 || !(geom->alatt > 0.0))
        return ht_fail(HT_ERR_INVALID, "ht_peak_lightcone: bad tile geometry");
    if (ht_fault_injected("launch")) return ht_fail(HT_ERR_FAULT, "injected launch fault: ht_peak_lightcone");
    HT_CUDA_TRY(cudaSetDevice(ctx->device), "cudaSetDevice");
    cudaStream_t st = (cudaStream_t)stream;
    if (npeaks == 0) {
        HT_CUDA_TRY(cudaMemsetAsync(d_nkeep, 0, sizeof(int64_t), st), "nkeep reset");
        ctx->last_kernels = 0;
        return HT_OK;
    }
    uint8_t* flags;
    int32_t* idx;
    void* temp;
    size_t tb;
    int rc = catalog_workspace(ctx, npeaks, &flags, &idx, &temp, &tb);
    if (rc != HT_OK) return rc;
    const TableDev t{ctx->d_ct, ctx->nx, ctx->ny, ctx->nz, ctx->X1, ctx->X2, ctx->Y1,
                     ctx->Y2, ctx->Z1, ctx->Z2, ctx->out_val};
    const unsigned blocks = (unsigned)((npeaks + 255) / 256);
    lightcone_kernel<<<blocks, 256, 0, st>>>(d_i, d_j, d_k, npeaks, *geom, obs[0], obs[1],
                                             obs[2], z_max, cosmo_of(ctx), t, d_z, d_ZZon,
                                             d_fcrit, flags);
    HT_CUDA_TRY(cudaGetLastError(), "lightcone_kernel launch");
    thrust::counting_iterator<int32_t> it(0);
    HT_CUDA_TRY(cub::DeviceSelect::Flagged(temp, tb, it, flags, d_keep, (long long*)d_nkeep,
                                           (int)npeaks, st),
                "cub::DeviceSelect::Flagged");
    ctx->last_kernels = 2;
    return HT_OK;
}

extern "C" HT_API int ht_pack_halos(ht_ctx* ctx, const ht_catalog_peaks* peaks,
                                    const ht_results* res, const ht_tile_geom* geom,
                                    double ZZon, double z_max, int32_t ilpt,
                                    int32_t ioutshear, float* d_records, int64_t cap,
                                    int64_t* d_nhalo, void* stream) {
    HT_RANGE("ht_pack_halos");
    if (!ctx || !peaks || !res || !geom || !d_nhalo || (cap > 0 && !d_records))
        return ht_fail(HT_ERR_INVALID, "ht_pack_halos: NULL argument");
    if (!ctx->cosmo_set) return ht_fail(HT_ERR_STATE, "ht_pack_halos: call ht_ctx_set_cosmo first");
    const long long npeaks = peaks->npeaks;
    if (npeaks < 0 || npeaks > 0x7fffffffLL || cap < 0)
        return ht_fail(HT_ERR_CAPACITY, "ht_pack_halos: npeaks must be in [0, 2^31), cap >= 0");
    if (npeaks > 0 && (!peaks->i || !peaks->j || !peaks->k || !res->RTHL || !res->Fbarx ||
                       !res->Sbar || !res->Sbar2))
        return ht_fail(HT_ERR_INVALID, "ht_pack_halos: NULL peak or result array");
    if (npeaks > 0 && ioutshear >= 1 &&
        (!peaks->Rf || !peaks->FcRf || !res->e_v || !res->p_v || !res->strain || !res->d2F ||
         !res->zvir_half || !res->gradpk || !res->gradpkf || !res->gradpkrf))
        return ht_fail(HT_ERR_INVALID, "ht_pack_halos: extended records need every result array");
    if (geom->n < 1 || !(geom->alatt > 0.0))
        return ht_fail(HT_ERR_INVALID, "ht_pack_halos: bad tile geometry");
    if (!peaks->z && !(ZZon > 0.0))
        return ht_fail(HT_ERR_INVALID, "ht_pack_halos: ZZon must be > 0 without per-peak z");
    if (ht_fault_injected("launch")) return ht_fail(HT_ERR_FAULT, "injected launch fault: ht_pack_halos");
    HT_CUDA_TRY(cudaSetDevice(ctx->device), "cudaSetDevice");
    cudaStream_t st = (cudaStream_t)stream;
    if (npeaks == 0) {
        HT_CUDA_TRY(cudaMemsetAsync(d_nhalo, 0, sizeof(int64_t), st), "nhalo reset");
        ctx->last_kernels = 0;
        return HT_OK;
    }
    uint8_t* flags;
    int32_t* idx;
    void* temp;
    size_t tb;
    int rc = catalog_workspace(ctx, npeaks, &flags, &idx, &temp, &tb);
    if (rc != HT_OK) return rc;
    const unsigned blocks = (unsigned)((npeaks + 255) / 256);
    halo_flag_kernel<<<blocks, 256, 0, st>>>(res->RTHL, peaks->z, npeaks, z_max, flags);
    HT_CUDA_TRY(cudaGetLastError(), "halo_flag_kernel launch");
    thrust::counting_iterator<int32_t> it(0);
    HT_CUDA_TRY(cub::DeviceSelect::Flagged(temp, tb, it, flags, idx, (long long*)d_nhalo,
                                           (int)npeaks, st),
                "cub::DeviceSelect::Flagged");
    PackArgs a{*peaks, *res, *geom, ZZon, ilpt, ioutshear >= 1 ? 33 : 11, cap, idx,
               (const long long*)d_nhalo, d_records};
    const long long rows = std::min((long long)npeaks, (long long)cap);
    if (rows > 0) {
        halo_record_kernel<<<(unsigned)((rows + 127) / 128), 128, 0, st>>>(a, cosmo_of(ctx));
        HT_CUDA_TRY(cudaGetLastError(), "halo_record_kernel launch");
    }
    ctx->last_kernels = 3;
    return HT_OK;
}
