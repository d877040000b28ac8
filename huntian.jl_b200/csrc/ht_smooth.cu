// k-space smoothing window applied to the rfft of delta before the per-filter inverse
// FFT (Filters.smooth_field, Filters.jl:72-99; GPU _smooth_window_kernel!,
// ext/CUDAExt.jl:2831-2871).  The window depends on |k| only, and on the rfft grid
// k^2 = dk^2 (ix^2 + iy^2 + iz^2) takes at most 3 (n/2)^2 + 1 values, so the FP64 window
// is evaluated once per distinct integer ix^2 + iy^2 + iz^2 into a table (first kernel)
// and the modes are multiplied by Float32(W) from it (second kernel, bandwidth-bound:
// 8 B read + 8 B written per mode).  k = 0 is left unchanged, as in the reference.
#include <cufft.h>
#include <math.h>

#include <string>

#include "ht_internal.cuh"

namespace {

// wsmooth: 0 Gaussian in the Fortran convention exp(-(kR/2)^2 / 2), 3 the same times k^2,
// anything else the top-hat 3 (sin x - x cos x) / x^3 (ext/CUDAExt.jl:2853-2866).
__global__ void window_table_kernel(float* __restrict__ tab, int nvals, double dk, double Rf,
                                    int wsmooth, double scale) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nvals) return;
    double w = 1.0;
    if (q > 0) {
        const double k2 = (double)q * dk * dk;
        const double k = sqrt(k2);
        const double kR = k * Rf;
        if (wsmooth == 0) {
            w = exp(-kR * kR * 0.125);
        } else if (wsmooth == 3) {
            w = exp(-kR * kR * 0.125) * k2;
        } else {
            double s, c;
            sincos(kR, &s, &c);
            w = 3.0 * (s - kR * c) / (kR * kR * kR);
        }
    }
    tab[q] = (float)(w * scale);
}

// One thread per mode; grid (ceil((n/2+1) / 256), n, n) so that the mode's (iy, iz)
// come from the block index instead of 64-bit division.
__global__ void __launch_bounds__(256) window_apply_kernel(const float2* __restrict__ in,
                                                           float2* __restrict__ out, int n,
                                                           const float* __restrict__ tab,
                                                           bool scaled) {
    const int nk = n / 2 + 1;
    const int ix = blockIdx.x * blockDim.x + threadIdx.x;
    if (ix >= nk) return;
    const int iy = blockIdx.y, iz = blockIdx.z;
    const long long li = ((long long)iz * n + iy) * nk + ix;
    const int sy = iy <= n / 2 ? iy : iy - n;
    const int sz = iz <= n / 2 ? iz : iz - n;
    const int q = ix * ix + sy * sy + sz * sz;
    float2 v = __ldg(in + li);
    if (q > 0 || scaled) {
        const float w = __ldg(tab + q);
        v.x *= w;
        v.y *= w;
    }
    out[li] = v;
}

// Window table + apply on stream st; scale multiplies every mode, k = 0 included, when
// scaled is true (the 1/n^3 of the inverse FFT folded into the window).
int launch_window(ht_ctx* ctx, const void* d_delta_k, void* d_out, int n, double boxsize,
                  double Rf, int wsmooth, double scale, bool scaled, cudaStream_t st) {
    const int h = n / 2;
    const int nvals = 3 * h * h + 1;
    int rc = ht_grow(&ctx->d_win, &ctx->win_bytes, (size_t)nvals * sizeof(float),
                     "window table");
    if (rc != HT_OK) return rc;
    const double dk = 2.0 * 3.14159265358979323846 / boxsize;
    window_table_kernel<<<(nvals + 255) / 256, 256, 0, st>>>((float*)ctx->d_win, nvals, dk, Rf,
                                                             wsmooth, scale);
    HT_CUDA_TRY(cudaGetLastError(), "window_table_kernel launch");
    const dim3 agrid((unsigned)((h + 1 + 255) / 256), (unsigned)n, (unsigned)n);
    window_apply_kernel<<<agrid, 256, 0, st>>>((const float2*)d_delta_k, (float2*)d_out, n,
                                                (const float*)ctx->d_win, scaled);
    HT_CUDA_TRY(cudaGetLastError(), "window_apply_kernel launch");
    return HT_OK;
}

int check_window_args(const char* who, double boxsize, double Rf) {
    if (!(boxsize > 0.0) || !(Rf >= 0.0))
        return ht_fail(HT_ERR_INVALID, std::string(who) + ": boxsize must be > 0 and Rf >= 0");
    return HT_OK;
}

}  // namespace

extern "C" HT_API int ht_smooth_window(ht_ctx* ctx, const void* d_delta_k, void* d_out, int n,
                                       double boxsize, double Rf, int wsmooth, void* stream) {
    if (!ctx || !d_delta_k || !d_out) return ht_fail(HT_ERR_INVALID, "ht_smooth_window: NULL argument");
    if (n < 2 || n > 8192) return ht_fail(HT_ERR_INVALID, "ht_smooth_window: need 2 <= n <= 8192");
    int rc = check_window_args("ht_smooth_window", boxsize, Rf);
    if (rc != HT_OK) return rc;
    if (ht_fault_injected("launch")) return ht_fail(HT_ERR_FAULT, "injected launch fault: ht_smooth_window");
    HT_CUDA_TRY(cudaSetDevice(ctx->device), "cudaSetDevice");
    rc = launch_window(ctx, d_delta_k, d_out, n, boxsize, Rf, wsmooth, 1.0, false,
                       (cudaStream_t)stream);
    if (rc != HT_OK) return rc;
    ctx->last_kernels = 2;
    return HT_OK;
}

// ------------------------------------------------------ window + inverse FFT (tile) ----

extern "C" HT_API int ht_smooth_tile(ht_ctx* ctx, const void* d_delta_k, float* d_out, int n,
                                     double boxsize, double Rf, int wsmooth, void* stream) {
    if (!ctx || !d_delta_k || !d_out) return ht_fail(HT_ERR_INVALID, "ht_smooth_tile: NULL argument");
    if (n < 2 || n > 4096) return ht_fail(HT_ERR_INVALID, "ht_smooth_tile: need 2 <= n <= 4096");
    int rc = check_window_args("ht_smooth_tile", boxsize, Rf);
    if (rc != HT_OK) return rc;
    if (ht_fault_injected("launch")) return ht_fail(HT_ERR_FAULT, "injected launch fault: ht_smooth_tile");
    HT_CUDA_TRY(cudaSetDevice(ctx->device), "cudaSetDevice");
    const long long nk = n / 2 + 1;
    const size_t cbytes = (size_t)nk * n * n * 2 * sizeof(float);
    rc = ht_grow(&ctx->d_cwork, &ctx->cwork_bytes, cbytes, "smoothing buffer");
    if (rc != HT_OK) return rc;
    if (ctx->tile_n != n) {
        if (ctx->tile_n) { cufftDestroy(ctx->tile_plan); ctx->tile_n = 0; }
        if (ht_fault_injected("alloc")) return ht_fail(HT_ERR_FAULT, "injected allocation fault: cuFFT plan");
        int dims[3] = {n, n, n};
        int inembed[3] = {n, n, (int)nk};
        int onembed[3] = {n, n, n};
        cufftResult r = cufftPlanMany(&ctx->tile_plan, 3, dims, inembed, 1, (int)(nk * n * n),
                                      onembed, 1, n * n * n, CUFFT_C2R, 1);
        if (r != CUFFT_SUCCESS)
            return ht_fail(HT_ERR_CUDA, "cufftPlanMany(C2R, out of place) failed with code " +
                                            std::to_string((int)r));
        ctx->tile_n = n;
    }
    cudaStream_t st = (cudaStream_t)stream;
    const double scale = 1.0 / ((double)n * n * n);
    rc = launch_window(ctx, d_delta_k, ctx->d_cwork, n, boxsize, Rf, wsmooth, scale, true, st);
    if (rc != HT_OK) return rc;
    if (cufftSetStream(ctx->tile_plan, st) != CUFFT_SUCCESS)
        return ht_fail(HT_ERR_CUDA, "cufftSetStream failed");
    cufftResult r = cufftExecC2R(ctx->tile_plan, (cufftComplex*)ctx->d_cwork, (cufftReal*)d_out);
    if (r != CUFFT_SUCCESS)
        return ht_fail(HT_ERR_CUDA, "cufftExecC2R failed with code " + std::to_string((int)r));
    ctx->last_kernels = 2;
    return HT_OK;
}

// ------------------------------------------------- window + inverse FFT + wrap ----
//
// ht_smooth_filter: the whole per-filter smoothing of a periodic n^3 box, delivered as the
// tile the peak scan reads: the window above into a context-owned complex buffer, an
// in-place cuFFT C2R (plan cached per n; the result is the padded real layout with rows of
// 2 (n/2 + 1) floats), then one kernel that writes tile cell (i, j, k) =
// box((i - nbuff) mod n, ...) / n^3 -- the normalisation of Julia's irfft -- for the
// (n + 2 nbuff)^3 tile with periodic wrap.

namespace {

// One thread per tile cell; grid (ceil(nt / 128), nt, nt): the cell's (j, k) come from
// the block index.
__global__ void __launch_bounds__(128) wrap_pad_kernel(const float* __restrict__ box, int n,
                                                       long long row, int nbuff,
                                                       float* __restrict__ tile, float scale) {
    const int nt = n + 2 * nbuff;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nt) return;
    const int j = blockIdx.y, k = blockIdx.z;
    int bi = i - nbuff, bj = j - nbuff, bk = k - nbuff;
    bi = bi < 0 ? bi + n : (bi >= n ? bi - n : bi);
    bj = bj < 0 ? bj + n : (bj >= n ? bj - n : bj);
    bk = bk < 0 ? bk + n : (bk >= n ? bk - n : bk);
    tile[((long long)k * nt + j) * nt + i] =
        __ldg(box + ((long long)bk * n + bj) * row + bi) * scale;
}

}  // namespace

extern "C" HT_API int ht_smooth_filter(ht_ctx* ctx, const void* d_delta_k, float* d_tile, int n,
                                       int nbuff, double boxsize, double Rf, int wsmooth,
                                       void* stream) {
    if (!ctx || !d_delta_k || !d_tile) return ht_fail(HT_ERR_INVALID, "ht_smooth_filter: NULL argument");
    if (n < 2 || n > 4096 || nbuff < 0 || nbuff > n)
        return ht_fail(HT_ERR_INVALID, "ht_smooth_filter: need 2 <= n <= 4096 and 0 <= nbuff <= n");
    HT_CUDA_TRY(cudaSetDevice(ctx->device), "cudaSetDevice");
    const long long nk = n / 2 + 1;
    const size_t cbytes = (size_t)nk * n * n * 2 * sizeof(float);
    int rc = ht_grow(&ctx->d_cwork, &ctx->cwork_bytes, cbytes, "smoothing buffer");
    if (rc != HT_OK) return rc;
    if (ctx->fft_n != n) {
        if (ctx->fft_n) { cufftDestroy(ctx->fft_plan); ctx->fft_n = 0; }
        if (ht_fault_injected("alloc")) return ht_fail(HT_ERR_FAULT, "injected allocation fault: cuFFT plan");
        cufftResult r = cufftPlan3d(&ctx->fft_plan, n, n, n, CUFFT_C2R);
        if (r != CUFFT_SUCCESS)
            return ht_fail(HT_ERR_CUDA, "cufftPlan3d(C2R) failed with code " + std::to_string((int)r));
        ctx->fft_n = n;
    }
    rc = ht_smooth_window(ctx, d_delta_k, ctx->d_cwork, n, boxsize, Rf, wsmooth, stream);
    if (rc != HT_OK) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    if (cufftSetStream(ctx->fft_plan, st) != CUFFT_SUCCESS)
        return ht_fail(HT_ERR_CUDA, "cufftSetStream failed");
    cufftResult r = cufftExecC2R(ctx->fft_plan, (cufftComplex*)ctx->d_cwork, (cufftReal*)ctx->d_cwork);
    if (r != CUFFT_SUCCESS)
        return ht_fail(HT_ERR_CUDA, "cufftExecC2R failed with code " + std::to_string((int)r));
    const int nt = n + 2 * nbuff;
    const float scale = (float)(1.0 / ((double)n * n * n));
    const dim3 wgrid((unsigned)((nt + 127) / 128), (unsigned)nt, (unsigned)nt);
    wrap_pad_kernel<<<wgrid, 128, 0, st>>>((const float*)ctx->d_cwork, n, 2 * nk, nbuff, d_tile,
                                           scale);
    HT_CUDA_TRY(cudaGetLastError(), "wrap_pad_kernel launch");
    ctx->last_kernels = 3;
    return HT_OK;
}
