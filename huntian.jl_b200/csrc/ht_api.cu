// C ABI of huntian_b200: context management, host-side tables, argument checks and
// dispatch to the kernels in ht_peakfind.cu and ht_shell.cu.
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <cstdio>
#include <string>
#include <vector>

#include "ht_internal.cuh"

// ----------------------------------------------------------------- errors ----

static thread_local std::string g_last_error;

int ht_fail(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}

int ht_cuda_fail(cudaError_t e, const char* what) {
    return ht_fail(HT_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

// Host-side fault injection for tests: HT_FAULT_INJECT="alloc" makes every device
// allocation fail, "launch" makes every kernel dispatch fail, before the device is
// touched.  Off unless the variable is set.
bool ht_fault_injected(const char* site) {
    const char* v = getenv("HT_FAULT_INJECT");
    if (!v || !*v) return false;
    std::string s(v);
    size_t pos = 0;
    while (pos <= s.size()) {
        size_t e = s.find(',', pos);
        if (e == std::string::npos) e = s.size();
        if (s.compare(pos, e - pos, site) == 0) return true;
        pos = e + 1;
    }
    return false;
}

int ht_alloc(void** p, size_t bytes, const char* what) {
    if (ht_fault_injected("alloc")) return ht_fail(HT_ERR_FAULT, std::string("injected allocation fault: ") + what);
    cudaError_t e = cudaMalloc(p, bytes ? bytes : 1);
    if (e != cudaSuccess) {
        cudaGetLastError();
        char buf[128];
        snprintf(buf, sizeof buf, " (%zu bytes)", bytes);
        return ht_fail(HT_ERR_NOMEM, std::string("cudaMalloc failed for ") + what + buf + ": " +
                                         cudaGetErrorString(e));
    }
    return HT_OK;
}

int ht_grow(void** p, size_t* have, size_t need, const char* what) {
    if (*p && *have >= need) return HT_OK;
    if (*p) { cudaFree(*p); *p = nullptr; *have = 0; }
    int rc = ht_alloc(p, need, what);
    if (rc == HT_OK) *have = need;
    return rc;
}

extern "C" const char* ht_last_error(void) { return g_last_error.c_str(); }

// ------------------------------------------------------------ host tables ----

// Shell offsets (RadialShell.jl:151-166): all (di, dj, dk) with r^2 <= nhunt^2, in
// dk-outer / dj / di-inner generation order, stably sorted by r^2 (a counting sort is
// stable), grouped into shells by r^2 (ShellAnalysisGPU.jl:44-71).
static void build_shells(ht_ctx* c, int nhunt) {
    const int r2max = nhunt * nhunt;
    std::vector<int64_t> hist((size_t)r2max + 2, 0);
    for (int dk = -nhunt; dk <= nhunt; ++dk)
        for (int dj = -nhunt; dj <= nhunt; ++dj)
            for (int di = -nhunt; di <= nhunt; ++di) {
                int r2 = di * di + dj * dj + dk * dk;
                if (r2 <= r2max) hist[r2 + 1]++;
            }
    std::vector<int64_t> pos(hist.size());
    int64_t acc = 0;
    for (size_t r = 0; r + 1 < hist.size(); ++r) { acc += hist[r + 1]; pos[r] = acc - hist[r + 1]; }
    c->ncells = acc;
    c->h_off.assign((size_t)acc, make_char4(0, 0, 0, 0));
    std::vector<int64_t> wr(pos.begin(), pos.end());
    for (int dk = -nhunt; dk <= nhunt; ++dk)
        for (int dj = -nhunt; dj <= nhunt; ++dj)
            for (int di = -nhunt; di <= nhunt; ++di) {
                int r2 = di * di + dj * dj + dk * dk;
                if (r2 <= r2max) c->h_off[(size_t)wr[r2]++] = make_char4((signed char)di, (signed char)dj, (signed char)dk, 0);
            }
    // shells, 1-based with padding at 0 and nshells + 1
    c->h_r2.assign(1, 0);
    c->h_start.assign(1, 0);
    c->h_count.assign(1, 0);
    for (int r2 = 0; r2 <= r2max; ++r2) {
        if (hist[r2 + 1] == 0) continue;
        c->h_r2.push_back(r2);
        c->h_start.push_back((int32_t)pos[r2]);
        c->h_count.push_back((int32_t)hist[r2 + 1]);
    }
    c->nshells = (int32_t)c->h_r2.size() - 1;
    c->h_r2.push_back(INT32_MAX);
    c->h_start.push_back((int32_t)acc);
    c->h_count.push_back(0);
}

// SPH table atab4 (RadialShell.jl:125-142): akk[i] = W(sqrt(u)), u = i * 0.01 (0-based).
static void build_akk(std::vector<double>& akk) {
    const double pi = 3.14159265358979323846;
    const double ca = 3.0 / (2.0 * pi), cb = 1.0 / (4.0 * pi);
    akk.assign(1101, 0.0);
    for (int i = 0; i < 1100; ++i) {
        const double u = i * 0.01, ru = sqrt(u);
        double v = 0.0;
        if (ru < 1.0) v = ca * (2.0 / 3.0 - u + 0.5 * u * ru);
        else if (ru <= 2.0) { const double t = 2.0 - ru; v = cb * (t * t * t); }
        akk[i] = v;
    }
    akk[1100] = 0.0;
}

// hRinteg (RadialShell.jl:95-121): integral of the SPH kernel 4 pi W(x) x (x^2 - u12)
// from |u0| to 2 (Fortran peakvoidsubs.f90 hRinteg).
static double hRinteg(double u0, double u12) {
    const double x0 = fabs(u0);
    if (x0 >= 2.0) return 0.0;
    const double one7 = 1.0 / 7.0;
    double result = 1.6 * u12 - 6.4 * one7;
    const double x02 = x0 * x0, x04 = x02 * x02;
    if (x0 >= 1.0) {
        const double h1 = x04 * (2.0 - x0 * (2.4 - x0 * (1.0 - x0 * one7)));
        const double h2 = x02 * (4.0 - x0 * (4.0 - x0 * (1.5 - x0 * 0.2)));
        result = result - h2 * u12 + h1;
    } else {
        result = result - 0.2 * (u12 - one7);
        if (x0 > 0.0) {
            const double h1 = x04 * (1.0 - x02 * (1.0 - 3.0 * x0 * one7));
            const double h2 = x02 * (2.0 - x02 * (1.5 - 0.6 * x0));
            result = result - h2 * u12 + h1;
        }
    }
    return result;
}

// Weight table of kernel_strain (RadialShell.jl:225-274, hlatt = 1).  Row mp > 1: the
// shells m1 >= 2 with u0^2 < 4, u0 = rad[mp] - rad[m1], weight
// hRinteg(u0, u12) / (u12 - u0^2)^2 with u12 = rad[mp]^2 + rad[m1]^2.  Row 1 (the central
// branch, used by the inward walk's last step, whose window is shells 2..U(1) with
// U(1) the last shell below radius 2): weight 0.5 * akk(100 rad^2) / rad[m1] with akk
// linearly interpolated.  These are the reference's weights, evaluated once.
static void build_weights(const std::vector<double>& rad, int nshells,
                          const std::vector<double>& akk, std::vector<int32_t>& row,
                          std::vector<int32_t>& m1s, std::vector<double>& wts) {
    row.assign((size_t)nshells + 2, 0);
    m1s.clear();
    wts.clear();
    int lo = 2;
    for (int mp = 1; mp <= nshells; ++mp) {
        row[mp] = (int32_t)m1s.size();
        if (mp == 1) {
            for (int m1 = 2; m1 <= nshells && rad[m1] < 2.0; ++m1) {
                const double r1 = rad[m1];
                const double con = 100.0 * r1 * r1;
                const double fl = floor(con);
                const int icon = (int)fl;
                const double diff = con - fl;
                double aww = 0.0;
                if (icon >= 0 && icon < 1100) aww = akk[icon] + diff * (akk[icon + 1] - akk[icon]);
                m1s.push_back(m1);
                wts.push_back(0.5 * aww / r1);
            }
            continue;
        }
        const double rmp = rad[mp];
        while (lo < mp && (rmp - rad[lo]) * (rmp - rad[lo]) >= 4.0) ++lo;
        for (int m1 = lo; m1 <= nshells; ++m1) {
            const double u0 = rmp - rad[m1];
            const double u02 = u0 * u0;
            if (!(u02 < 4.0)) {
                if (m1 > mp) break;
                continue;
            }
            const double u12 = rmp * rmp + rad[m1] * rad[m1];
            const double den = u12 - u02;
            m1s.push_back(m1);
            wts.push_back(hRinteg(u0, u12) / (den * den));
        }
    }
    row[(size_t)nshells + 1] = (int32_t)m1s.size();
}

// Trilinear lookup on the host copy (CollapseTable.jl:126-138), for fsc_of_z.
static double host_interp(const ht_ctx* c, double x, double y, double z) {
    if (!(x >= c->X1 && x <= c->X2 && y >= c->Y1 && y <= c->Y2 && z >= c->Z1 && z <= c->Z2))
        return c->out_val;
    double tx = (x - c->X1) / ((c->X2 - c->X1) / (c->nx - 1));
    double ty = (y - c->Y1) / ((c->Y2 - c->Y1) / (c->ny - 1));
    double tz = (z - c->Z1) / ((c->Z2 - c->Z1) / (c->nz - 1));
    int ix = std::min(std::max((int)floor(tx), 0), c->nx - 2);
    int iy = std::min(std::max((int)floor(ty), 0), c->ny - 2);
    int iz = std::min(std::max((int)floor(tz), 0), c->nz - 2);
    double fx = tx - ix, fy = ty - iy, fz = tz - iz;
    const size_t sy = c->nx, sz = (size_t)c->nx * c->ny;
    const float* t = c->h_ct.data() + ix + iy * sy + iz * sz;
    double c00 = t[0] * (1.0 - fx) + t[1] * fx;
    double c10 = t[sy] * (1.0 - fx) + t[1 + sy] * fx;
    double c01 = t[sz] * (1.0 - fx) + t[1 + sz] * fx;
    double c11 = t[sy + sz] * (1.0 - fx) + t[1 + sy + sz] * fx;
    double c0 = c00 * (1.0 - fy) + c10 * fy;
    double c1 = c01 * (1.0 - fy) + c11 * fy;
    return c0 * (1.0 - fz) + c1 * fz;
}

static void free_ctx(ht_ctx* c) {
    if (c->fft_n) cufftDestroy(c->fft_plan);
    if (c->tile_n) cufftDestroy(c->tile_plan);
    if (c->tp_n) cufftDestroy(c->tp_plan_n);
    if (c->tp_zc) { cufftDestroy(c->tp_plan_y); cufftDestroy(c->tp_plan_x); }
    void* ptrs[] = {c->d_off, c->d_start, c->d_count, c->d_r2, c->d_rad, c->d_ct, c->d_akk,
                    c->d_wrow, c->d_wpk, c->d_irad, c->d_irad3, c->d_cell,
                    c->d_rec, c->d_pf_ws, c->d_scratch, c->d_win, c->d_cwork, c->d_order_ws,
                    c->d_mlp_ws, c->d_cwork2, c->d_tw, c->d_ftw, c->d_wb, c->d_wu, c->d_queue,
                    c->d_stats, c->d_chi, c->d_zchi, c->d_atab, c->d_Da, c->d_dlnD,
                    c->d_cat_ws, c->d_merge_ws, c->d_merge_cells, c->d_merge_scan};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    delete c;
}

template <typename T>
static int upload(T** dst, const T* src, size_t n, const char* what) {
    int rc = ht_alloc((void**)dst, n * sizeof(T), what);
    if (rc != HT_OK) return rc;
    HT_CUDA_TRY(cudaMemcpy(*dst, src, n * sizeof(T), cudaMemcpyHostToDevice), what);
    return HT_OK;
}

// ------------------------------------------------------------------- ABI ----

extern "C" int ht_ctx_create(int device, int nhunt, const float* ct_table_host, int nx, int ny,
                             int nz, double X1, double X2, double Y1, double Y2, double Z1,
                             double Z2, double out_val, ht_ctx** out) {
    HT_RANGE("ht_ctx_create");
    if (!out) return ht_fail(HT_ERR_INVALID, "ht_ctx_create: out is NULL");
    *out = nullptr;
    if (nhunt < 1 || nhunt > 127)
        return ht_fail(HT_ERR_INVALID, "ht_ctx_create: nhunt must be in 1..127 (offsets are 8-bit)");
    if (!ct_table_host || nx < 2 || ny < 2 || nz < 2)
        return ht_fail(HT_ERR_INVALID, "ht_ctx_create: collapse table must be at least 2x2x2");
    if (!(X2 > X1) || !(Y2 > Y1) || !(Z2 > Z1))
        return ht_fail(HT_ERR_INVALID, "ht_ctx_create: collapse-table axes must be increasing");
    HT_CUDA_TRY(cudaSetDevice(device), "cudaSetDevice");
    ht_ctx* c = new ht_ctx();
    c->device = device;
    c->nhunt = nhunt;
    cudaError_t e = cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) { free_ctx(c); return ht_cuda_fail(e, "cudaDeviceGetAttribute"); }
    build_shells(c, nhunt);
    std::vector<double> rad(c->h_r2.size());
    for (size_t m = 0; m < rad.size(); ++m)
        rad[m] = (m == 0 || m + 1 == rad.size()) ? (m == 0 ? 0.0 : INFINITY) : sqrt((double)c->h_r2[m]);
    c->h_ct.assign(ct_table_host, ct_table_host + (size_t)nx * ny * nz);
    c->nx = nx; c->ny = ny; c->nz = nz;
    c->X1 = X1; c->X2 = X2; c->Y1 = Y1; c->Y2 = Y2; c->Z1 = Z1; c->Z2 = Z2;
    c->out_val = out_val;
    std::vector<double> akk;
    build_akk(akk);
    std::vector<int32_t> wrow, wm1;
    std::vector<double> wwt;
    build_weights(rad, c->nshells, akk, wrow, wm1, wwt);
    std::vector<double> irad(rad.size(), 0.0), irad3(rad.size(), 0.0);
    for (size_t m = 0; m < rad.size(); ++m)
        if (rad[m] > 0.0) { irad[m] = 1.0 / rad[m]; irad3[m] = 1.0 / (rad[m] * rad[m] * rad[m]); }
    c->nweights = (int64_t)wm1.size();
    std::vector<double2> wpk(wm1.size());
    for (size_t e = 0; e < wm1.size(); ++e) wpk[e] = make_double2(wwt[e], (double)wm1[e]);
    int rc;
    if ((rc = upload(&c->d_off, c->h_off.data(), c->h_off.size(), "shell offsets")) ||
        (rc = upload(&c->d_start, c->h_start.data(), c->h_start.size(), "shell starts")) ||
        (rc = upload(&c->d_count, c->h_count.data(), c->h_count.size(), "shell counts")) ||
        (rc = upload(&c->d_r2, c->h_r2.data(), c->h_r2.size(), "shell r2")) ||
        (rc = upload(&c->d_rad, rad.data(), rad.size(), "shell radii")) ||
        (rc = upload(&c->d_irad, irad.data(), irad.size(), "inverse shell radii")) ||
        (rc = upload(&c->d_irad3, irad3.data(), irad3.size(), "inverse cubed radii")) ||
        (rc = upload(&c->d_ct, c->h_ct.data(), c->h_ct.size(), "collapse table")) ||
        (rc = upload(&c->d_akk, akk.data(), akk.size(), "SPH table")) ||
        (rc = upload(&c->d_wrow, wrow.data(), wrow.size(), "weight rows")) ||
        (rc = upload(&c->d_wpk, wpk.data(), wpk.size(), "weights")) ||
        (rc = ht_alloc((void**)&c->d_queue, 256, "work queue")) ||
        (rc = ht_alloc((void**)&c->d_stats, 256, "launch stats"))) {
        free_ctx(c);
        return rc;
    }
    HT_CUDA_TRY(cudaMemset(c->d_stats, 0, 256), "stats init");
    *out = c;
    return HT_OK;
}

extern "C" int ht_ctx_destroy(ht_ctx* ctx) {
    HT_RANGE("ht_ctx_destroy");
    if (!ctx) return HT_OK;
    cudaSetDevice(ctx->device);
    free_ctx(ctx);
    return HT_OK;
}

extern "C" int ht_ctx_shell_info(const ht_ctx* ctx, int32_t* nshells, int64_t* ncells) {
    if (!ctx) return ht_fail(HT_ERR_INVALID, "ht_ctx_shell_info: ctx is NULL");
    if (nshells) *nshells = ctx->nshells;
    if (ncells) *ncells = ctx->ncells;
    return HT_OK;
}

extern "C" int ht_ctx_shell_r2(const ht_ctx* ctx, int32_t* r2_host, int32_t cap) {
    if (!ctx || !r2_host) return ht_fail(HT_ERR_INVALID, "ht_ctx_shell_r2: NULL argument");
    if (cap < ctx->nshells) return ht_fail(HT_ERR_CAPACITY, "ht_ctx_shell_r2: cap < nshells");
    memcpy(r2_host, ctx->h_r2.data() + 1, sizeof(int32_t) * (size_t)ctx->nshells);
    return HT_OK;
}

extern "C" int ht_fsc_of_z(const ht_ctx* ctx, double z, double* fcrit_out) {
    if (!ctx || !fcrit_out) return ht_fail(HT_ERR_INVALID, "ht_fsc_of_z: NULL argument");
    double target = 1.0 + z, lo = ctx->X1, hi = ctx->X2;
    for (int it = 0; it < 50; ++it) {
        double mid = 0.5 * (lo + hi);
        if (host_interp(ctx, mid, 0.0, 0.0) > target) hi = mid; else lo = mid;
    }
    *fcrit_out = pow(10.0, lo);
    return HT_OK;
}

extern "C" int ht_peakfind_filter(ht_ctx* ctx, const float* d_delta_s, const float* d_lapd_s,
                                  int8_t* d_mask, int n, int nbuff, float fcrit,
                                  int32_t filter_idx, int64_t max_peaks, const ht_peaks* out,
                                  void* stream) {
    HT_RANGE("ht_peakfind_filter");
    if (!ctx || !d_delta_s || !d_mask || !out)
        return ht_fail(HT_ERR_INVALID, "ht_peakfind_filter: NULL argument");
    if (!out->i || !out->j || !out->k || !out->delta || !out->filter_idx || !out->count)
        return ht_fail(HT_ERR_INVALID, "ht_peakfind_filter: NULL output array");
    if (n < 3 || nbuff < 1 || 2 * nbuff >= n)
        return ht_fail(HT_ERR_INVALID, "ht_peakfind_filter: need n >= 3 and 1 <= nbuff < n/2 "
                                       "(the 3x3x3 stencil reads one cell beyond the inner cube)");
    if ((long long)n * n * n > (1LL << 40))
        return ht_fail(HT_ERR_CAPACITY, "ht_peakfind_filter: n^3 too large");
    if (max_peaks < 0) return ht_fail(HT_ERR_INVALID, "ht_peakfind_filter: max_peaks < 0");
    if (ht_fault_injected("launch")) return ht_fail(HT_ERR_FAULT, "injected launch fault: ht_peakfind_filter");
    HT_CUDA_TRY(cudaSetDevice(ctx->device), "cudaSetDevice");
    return ht_launch_peakfind(ctx, d_delta_s, d_lapd_s, d_mask, n, nbuff, fcrit, filter_idx,
                              max_peaks, out, (cudaStream_t)stream);
}

extern "C" int ht_fields_pack(ht_ctx* ctx, const ht_fields* f, void* stream) {
    HT_RANGE("ht_fields_pack");
    if (!ctx || !f) return ht_fail(HT_ERR_INVALID, "ht_fields_pack: NULL argument");
    if (!f->delta || !f->etax || !f->etay || !f->etaz)
        return ht_fail(HT_ERR_INVALID, "ht_fields_pack: delta and eta x/y/z are required");
    const bool any2 = f->eta2x || f->eta2y || f->eta2z;
    const bool all2 = f->eta2x && f->eta2y && f->eta2z;
    if (any2 && !all2) return ht_fail(HT_ERR_INVALID, "ht_fields_pack: give all of eta2x/y/z or none");
    if (f->n1 < 1 || f->n1 != f->n2 || f->n1 != f->n3)
        return ht_fail(HT_ERR_INVALID, "ht_fields_pack: the tile must be cubic (the gather reads "
                                       "delta[k, i, j], ext/CUDAExt.jl:819)");
    if (ht_fault_injected("launch")) return ht_fail(HT_ERR_FAULT, "injected launch fault: ht_fields_pack");
    HT_CUDA_TRY(cudaSetDevice(ctx->device), "cudaSetDevice");
    const size_t cells = (size_t)f->n1 * f->n2 * f->n3;
    if (!ctx->d_rec || ctx->rec_cells < cells) {
        if (ctx->d_rec) { cudaFree(ctx->d_rec); ctx->d_rec = nullptr; ctx->rec_cells = 0; }
        int rc = ht_alloc((void**)&ctx->d_rec, cells * 2 * sizeof(float4), "cell records");
        if (rc != HT_OK) { ctx->bound = false; return rc; }
        ctx->rec_cells = cells;
    }
    ctx->fields = *f;
    ctx->bound = true;
    return ht_launch_pack(ctx, (cudaStream_t)stream);
}

extern "C" int ht_shell_analyse(ht_ctx* ctx, const ht_peak_batch* b, double alatt,
                                double rmax2rs, int32_t nbuff, int8_t* d_mask, int32_t conv,
                                int32_t mode, const ht_results* out, void* stream) {
    HT_RANGE("ht_shell_analyse");
    if (!ctx || !b || !out) return ht_fail(HT_ERR_INVALID, "ht_shell_analyse: NULL argument");
    if (!ctx->bound) return ht_fail(HT_ERR_STATE, "ht_shell_analyse: call ht_fields_pack first");
    if (b->npeaks < 0) return ht_fail(HT_ERR_INVALID, "ht_shell_analyse: npeaks < 0");
    if (b->npeaks > 0 && (!b->pi || !b->pj || !b->pk || !b->Rf || !b->ir2min || !b->ZZon || !b->fcrit))
        return ht_fail(HT_ERR_INVALID, "ht_shell_analyse: NULL peak array");
    if (b->npeaks > 0 && (!out->RTHL || !out->Fbarx || !out->e_v || !out->p_v || !out->strain ||
                          !out->eigs || !out->Srb || !out->Sbar || !out->Sbar2 || !out->gradpk ||
                          !out->gradpkf || !out->gradpkrf || !out->d2F || !out->zvir_half))
        return ht_fail(HT_ERR_INVALID, "ht_shell_analyse: NULL result array");
    if (!(alatt > 0.0)) return ht_fail(HT_ERR_INVALID, "ht_shell_analyse: alatt must be > 0");
    if (conv != HT_CONV_GPU && conv != HT_CONV_CPU)
        return ht_fail(HT_ERR_INVALID, "ht_shell_analyse: unknown conv");
    if (conv == HT_CONV_CPU && rmax2rs > 0.0)
        return ht_fail(HT_ERR_INVALID, "ht_shell_analyse: HT_CONV_CPU supports rmax2rs == 0 only");
    if (mode != HT_MODE_PLAIN && mode != HT_MODE_BATCHED && mode != HT_MODE_LEARNED)
        return ht_fail(HT_ERR_INVALID, "ht_shell_analyse: unknown mode");
    if (mode == HT_MODE_LEARNED && !b->order && !b->cost && b->npeaks > 0)
        return ht_fail(HT_ERR_INVALID, "ht_shell_analyse: HT_MODE_LEARNED needs batch->cost "
                                       "(ht_bracket_predict) or batch->order");
    if (nbuff < 0) return ht_fail(HT_ERR_INVALID, "ht_shell_analyse: nbuff < 0");
    if (ctx->nshells < 3) return ht_fail(HT_ERR_INVALID, "ht_shell_analyse: hunt radius too small");
    if (ht_fault_injected("launch")) return ht_fail(HT_ERR_FAULT, "injected launch fault: ht_shell_analyse");
    ctx->last_kernels = 0;
    if (b->npeaks == 0) return HT_OK;
    HT_CUDA_TRY(cudaSetDevice(ctx->device), "cudaSetDevice");
    return ht_launch_walk(ctx, b, alatt, rmax2rs, nbuff, d_mask, conv, mode, out,
                          (cudaStream_t)stream);
}

extern "C" int ht_last_launch_stats(const ht_ctx* ctx, int64_t* kernels, int64_t* shells_walked,
                                    int64_t* cells_walked) {
    if (!ctx) return ht_fail(HT_ERR_INVALID, "ht_last_launch_stats: ctx is NULL");
    if (kernels) *kernels = ctx->last_kernels;
    if (shells_walked || cells_walked) {
        unsigned long long h[2] = {0, 0};
        HT_CUDA_TRY(cudaSetDevice(ctx->device), "cudaSetDevice");
        HT_CUDA_TRY(cudaMemcpy(h, ctx->d_stats, sizeof h, cudaMemcpyDeviceToHost), "stats read");
        if (cells_walked) *cells_walked = (int64_t)h[0];
        if (shells_walked) *shells_walked = (int64_t)h[1];
    }
    return HT_OK;
}

extern "C" int ht_reject_counts(const ht_ctx* ctx, int64_t* counts) {
    HT_RANGE("ht_reject_counts");
    if (!ctx || !counts) return ht_fail(HT_ERR_INVALID, "ht_reject_counts: NULL argument");
    unsigned long long h[HT_REJECT_COUNT];
    HT_CUDA_TRY(cudaSetDevice(ctx->device), "cudaSetDevice");
    HT_CUDA_TRY(cudaDeviceSynchronize(), "ht_reject_counts: synchronize");
    HT_CUDA_TRY(cudaMemcpy(h, ctx->d_stats + 16, sizeof h, cudaMemcpyDeviceToHost),
                "reject counters read");
    for (int i = 0; i < HT_REJECT_COUNT; ++i) counts[i] = (int64_t)h[i];
    return HT_OK;
}

extern "C" int ht_reset_reject_counts(ht_ctx* ctx, void* stream) {
    HT_RANGE("ht_reset_reject_counts");
    if (!ctx) return ht_fail(HT_ERR_INVALID, "ht_reset_reject_counts: ctx is NULL");
    HT_CUDA_TRY(cudaSetDevice(ctx->device), "cudaSetDevice");
    HT_CUDA_TRY(cudaMemsetAsync(ht_reject_words(ctx), 0,
                                HT_REJECT_COUNT * sizeof(unsigned long long),
                                (cudaStream_t)stream),
                "reject counters reset");
    return HT_OK;
}

extern "C" int ht_device_status(ht_ctx* ctx, int32_t* status) {
    HT_RANGE("ht_device_status");
    if (!ctx || !status) return ht_fail(HT_ERR_INVALID, "ht_device_status: NULL argument");
    HT_CUDA_TRY(cudaSetDevice(ctx->device), "cudaSetDevice");
    HT_CUDA_TRY(cudaDeviceSynchronize(), "ht_device_status: synchronize");
    int32_t v = 0;
    HT_CUDA_TRY(cudaMemcpy(&v, ht_status_word(ctx), sizeof v, cudaMemcpyDeviceToHost),
                "status read");
    if (v != 0) {
        const int32_t z = 0;
        HT_CUDA_TRY(cudaMemcpy(ht_status_word(ctx), &z, sizeof z, cudaMemcpyHostToDevice),
                    "status clear");
    }
    *status = v;
    return HT_OK;
}

extern "C" int ht_ctx_tune(ht_ctx* ctx, int32_t key, int64_t value) {
    if (!ctx) return ht_fail(HT_ERR_INVALID, "ht_ctx_tune: ctx is NULL");
    switch (key) {
        case HT_TUNE_BLOCK_BITS:
            if (value < 0 || value > 40) return ht_fail(HT_ERR_INVALID, "ht_ctx_tune: block bits must be 0..40");
            ctx->tune_block_bits = (int)value;
            return HT_OK;
        case HT_TUNE_PF_KZ:
            if (value != 0 && (value < 2 || value > 1024))
                return ht_fail(HT_ERR_INVALID, "ht_ctx_tune: planes per CTA must be 0 or 2..1024");
            ctx->tune_pf_kz = (int)value;
            return HT_OK;
        case HT_TUNE_FFT_PATH:
            if (value < 0 || value > 4) return ht_fail(HT_ERR_INVALID, "ht_ctx_tune: FFT path must be 0..4");
            ctx->tune_fft_path = (int)value;
            return HT_OK;
        case HT_TUNE_WALK_BPSM:
            if (value < 0 || value > 32) return ht_fail(HT_ERR_INVALID, "ht_ctx_tune: blocks per SM must be 0..32");
            ctx->tune_walk_bpsm = (int)value;
            return HT_OK;
        case HT_TUNE_WAIT_NS:
            if (value < 1000 || value > 60000000000LL)
                return ht_fail(HT_ERR_INVALID, "ht_ctx_tune: wait limit must be 1e3..6e10 ns");
            ctx->wait_ns = (long long)value;
            return HT_OK;
        case HT_TUNE_INJECT_TX:
            if (value < 0 || value > 4096 || value % 16 != 0)
                return ht_fail(HT_ERR_INVALID, "ht_ctx_tune: injected bytes must be 0..4096, a multiple of 16");
            ctx->inject_tx = (unsigned)value;
            return HT_OK;
        default:
            return ht_fail(HT_ERR_INVALID, "ht_ctx_tune: unknown key " + std::to_string(key));
    }
}
