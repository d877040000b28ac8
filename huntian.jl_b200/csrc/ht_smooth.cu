// k-space smoothing window applied to the rfft of delta before the per-filter inverse
// FFT (Filters.smooth_field, Filters.jl:72-99; GPU _smooth_window_kernel!,
// ext/CUDAExt.jl:2831-2871).  The window depends on |k| only, and on the rfft grid
// k^2 = dk^2 (ix^2 + iy^2 + iz^2) takes at most 3 (n/2)^2 + 1 values, so the FP64 window
// is evaluated once per distinct integer ix^2 + iy^2 + iz^2 into a table (first kernel)
// and the modes are multiplied by Float32(W) from it (second kernel, bandwidth-bound:
// 8 B read + 8 B written per mode).  k = 0 is left unchanged, as in the reference.
#include <cufft.h>
#include <algorithm>
#include <math.h>

#include <string>
#include <vector>

#include "ht_async.cuh"
#include "ht_fft.cuh"
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

// The window along kz of every distinct b = kx^2 + ky^2 (vals[i], ascending), for the
// pencil Z pass: U[i * UP + kz] = tab[b + kz^2] for kz <= h = n/2, 0 for h < kz < UP.  A
// Z-pass column then reads its window as one contiguous row (a 128-byte line per 32
// values) instead of one line per value (consecutive kz^2 lie more than a line apart
// beyond kz = 16).  A block takes 32 consecutive distinct values: its lanes read tab at
// b_lane + kz^2, a few lines per warp since neighbouring distinct b differ by about 5,
// 16 loads per thread in flight (128 kz per round), and the 128 x 32 tile is written back
// along the rows through shared memory.
__global__ void __launch_bounds__(256) window_rows_kernel(const float* __restrict__ tab,
                                                          const int32_t* __restrict__ vals,
                                                          int nb, int h, int UP,
                                                          float* __restrict__ U) {
    constexpr int KC = 128;
    __shared__ float s[KC][33];
    const int tx = threadIdx.x, ty = threadIdx.y;   // block (32, 8)
    const int i0 = blockIdx.x * 32;
    const bool have = i0 + tx < nb;
    const int b = have ? __ldg(vals + i0 + tx) : 0;
    for (int kc = 0; kc < UP; kc += KC) {
#pragma unroll
        for (int m = 0; m < KC / 8; ++m) {
            const int j = ty + 8 * m, kz = kc + j;
            s[j][tx] = (have && kz <= h) ? __ldg(tab + (b + kz * kz)) : 0.f;
        }
        __syncthreads();
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            const int r = ty + 8 * m;
            if (i0 + r < nb) {
                float* row = U + (long long)(i0 + r) * UP + kc;
#pragma unroll
                for (int q = 0; q < KC / 32; ++q) {
                    const int kz = tx + 32 * q;
                    if (kc + kz < UP) row[kz] = s[kz][r];
                }
            }
        }
        __syncthreads();
    }
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
    HT_RANGE("ht_smooth_window");
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

// ------------------------------------------- transposed inverse FFT of the tile ----
//
// cuFFT's single 3-D C2R plan is slow for tile sides that are not powers of two (19.1 ms
// at 1152^3 against 6.0 ms at 1024^3), while its batched 1-D transforms along a contiguous
// axis run near HBM speed at any size (2.1 ms for all 1152-point columns of a 1152^3
// field).  For such sides the inverse transform is therefore done axis by axis, each axis
// made contiguous by a tiled shared-memory transpose:
//   T1  window (with 1/n^3) + transpose (kz, ky, kx) -> A (ky, kx, kz)
//   F1  1-D C2C along kz, batch n (n/2+1), in place on A
//   T2  transpose A (ky, kx, z) -> B (z, kx, ky)
//   F2  1-D C2C along ky, in place on B
//   T3  transpose B (z, kx, y) -> C (z, y, k) with the half-length real-inverse packing
//       C[k] = (X[k] + conj X[m-k]) + i w^k (X[k] - conj X[m-k]),  m = n/2, w = e^{2 pi i/n}
//       (outputs k and m - k come from the same two rows, so each row is read once)
//   F3  1-D C2C of length m along k, batch n^2, out of place into the output: its complex
//       result c[j] = x[2j] + i x[2j+1] is the real row itself.
// Six HBM passes instead of the 3-D plan's slow decomposition; results agree with it to
// FP32 round-off (different summation order, same transform).

namespace {

__global__ void __launch_bounds__(256) t1_window_kernel(const float2* __restrict__ in,
                                                        float2* __restrict__ A, int N, int NK,
                                                        const float* __restrict__ tab) {
    __shared__ float2 t[32][33];
    const int a0 = blockIdx.x * 32, c0 = blockIdx.y * 32, ky = blockIdx.z;
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int sy = ky <= N / 2 ? ky : ky - N;
    for (int r = ty; r < 32; r += 8) {
        const int kx = a0 + tx, kz = c0 + r;
        if (kx < NK && kz < N) {
            float2 v = __ldg(in + ((long long)kz * N + ky) * NK + kx);
            if (tab) {   // no table: a plain transpose (the pencil layout of the spectrum)
                const int sz = kz <= N / 2 ? kz : kz - N;
                const float w = __ldg(tab + (kx * kx + sy * sy + sz * sz));
                v.x *= w;
                v.y *= w;
            }
            t[r][tx] = v;
        }
    }
    __syncthreads();
    for (int r = ty; r < 32; r += 8) {
        const int kz = c0 + tx, kx = a0 + r;
        if (kx < NK && kz < N) A[((long long)ky * NK + kx) * N + kz] = t[tx][r];
    }
}

// B[(z NK + kx) N + ky] = A[(ky NK + kx) N + z] for z in [zlo, zhi)
__global__ void __launch_bounds__(256) t2_kernel(const float2* __restrict__ A,
                                                 float2* __restrict__ B, int N, int NK,
                                                 int zlo, int zhi) {
    __shared__ float2 t[32][33];
    const int z0 = zlo + blockIdx.x * 32, y0 = blockIdx.y * 32, kx = blockIdx.z;
    const int tx = threadIdx.x, ty = threadIdx.y;
    for (int r = ty; r < 32; r += 8) {
        const int ky = y0 + r, z = z0 + tx;
        if (ky < N && z < zhi) t[r][tx] = __ldg(A + ((long long)ky * NK + kx) * N + z);
    }
    __syncthreads();
    for (int r = ty; r < 32; r += 8) {
        const int z = z0 + r, ky = y0 + tx;
        if (ky < N && z < zhi) B[((long long)z * NK + kx) * N + ky] = t[tx][r];
    }
}

// C[(z N + y) m + k] from X[k] = B[(z NK + k) N + y] and X[m - k], k < m = N/2.  Outputs k
// and m - k need the same two rows (X[k], X[m - k]), so a block loads a tile of "low" k in
// [k0, k0 + 32) (k <= m/2) and its mirror tile once and writes both outputs: B is read once.
__global__ void __launch_bounds__(256) t3_pack_kernel(const float2* __restrict__ B,
                                                      float2* __restrict__ C, int N, int NK,
                                                      const float2* __restrict__ tw, int zlo) {
    __shared__ float2 ta[32][33];
    __shared__ float2 tb[32][33];
    const int m = N / 2, half = m / 2;
    const int k0 = blockIdx.x * 32, y0 = blockIdx.y * 32, z = zlo + blockIdx.z;
    const int tx = threadIdx.x, ty = threadIdx.y;
    for (int r = ty; r < 32; r += 8) {
        const int k = k0 + r, y = y0 + tx;
        if (k <= half && y < N) {
            ta[r][tx] = __ldg(B + ((long long)z * NK + k) * N + y);
            tb[r][tx] = __ldg(B + ((long long)z * NK + (m - k)) * N + y);
        }
    }
    __syncthreads();
    // packed value for output kk from a = X[kk], bb = X[m - kk]
    auto pack = [&](float2 a, float2 bb, int kk) {
        const float2 b = make_float2(bb.x, -bb.y);          // conj X[m - kk]
        const float2 e = make_float2(a.x + b.x, a.y + b.y);
        const float2 d = make_float2(a.x - b.x, a.y - b.y);
        const float2 w = __ldg(tw + kk);
        const float2 o = make_float2(d.x * w.x - d.y * w.y, d.x * w.y + d.y * w.x);
        return make_float2(e.x - o.y, e.y + o.x);
    };
    for (int r = ty; r < 32; r += 8) {
        const int k = k0 + tx, y = y0 + r;
        if (k <= half && y < N) {
            const float2 xa = ta[tx][r], xb = tb[tx][r];
            float2* row = C + ((long long)z * N + y) * m;
            row[k] = pack(xa, xb, k);                       // k < m always (k <= m/2)
            const int kh = m - k;
            if (kh != k && kh < m) row[kh] = pack(xb, xa, kh);
        }
    }
}

}  // namespace

// Build (once per n) the 1-D plans and the twiddles of the transposed path.
// F2 / F3 plans for zc planes (the peak scan needs only the inner planes of the tile)
static int transposed_plane_plans(ht_ctx* ctx, int n, int zc) {
    if (ctx->tp_zc_n == n && ctx->tp_zc == zc) return HT_OK;
    if (ctx->tp_zc) {
        cufftDestroy(ctx->tp_plan_y);
        cufftDestroy(ctx->tp_plan_x);
        ctx->tp_zc = 0;
    }
    const int nk = n / 2 + 1, m = n / 2;
    int len[1] = {n}, lm[1] = {m};
    cufftResult r = cufftPlanMany(&ctx->tp_plan_y, 1, len, len, 1, n, len, 1, n, CUFFT_C2C,
                                  zc * nk);
    if (r != CUFFT_SUCCESS)
        return ht_fail(HT_ERR_CUDA, "cufftPlanMany(C2C, y planes) failed with code " + std::to_string((int)r));
    r = cufftPlanMany(&ctx->tp_plan_x, 1, lm, lm, 1, m, lm, 1, m, CUFFT_C2C, zc * n);
    if (r != CUFFT_SUCCESS) {
        cufftDestroy(ctx->tp_plan_y);
        return ht_fail(HT_ERR_CUDA, "cufftPlanMany(C2C, x planes) failed with code " + std::to_string((int)r));
    }
    ctx->tp_zc = zc;
    ctx->tp_zc_n = n;
    return HT_OK;
}

static int transposed_plans(ht_ctx* ctx, int n) {
    if (ctx->tp_n == n) return HT_OK;
    if (ctx->tp_n) {
        cufftDestroy(ctx->tp_plan_n);
        ctx->tp_n = 0;
    }
    if (ht_fault_injected("alloc")) return ht_fail(HT_ERR_FAULT, "injected allocation fault: cuFFT plan");
    const int nk = n / 2 + 1, m = n / 2;
    int len[1] = {n};
    cufftResult r = cufftPlanMany(&ctx->tp_plan_n, 1, len, len, 1, n, len, 1, n, CUFFT_C2C,
                                  n * nk);
    if (r != CUFFT_SUCCESS)
        return ht_fail(HT_ERR_CUDA, "cufftPlanMany(C2C, n) failed with code " + std::to_string((int)r));
    std::vector<float2> tw((size_t)m);
    for (int k = 0; k < m; ++k) {
        const double ph = 2.0 * 3.14159265358979323846 * (double)k / (double)n;
        tw[k] = make_float2((float)cos(ph), (float)sin(ph));
    }
    int rc = ht_grow(&ctx->d_tw, &ctx->tw_bytes, tw.size() * sizeof(float2), "C2R twiddles");
    if (rc != HT_OK) return rc;
    HT_CUDA_TRY(cudaMemcpy(ctx->d_tw, tw.data(), tw.size() * sizeof(float2), cudaMemcpyHostToDevice),
                "twiddle upload");
    ctx->tp_n = n;
    return HT_OK;
}

static int smooth_tile_transposed(ht_ctx* ctx, const void* d_delta_k, float* d_out, int n,
                                  double boxsize, double Rf, int wsmooth, int zlo, int zhi,
                                  cudaStream_t st) {
    const long long nk = n / 2 + 1;
    const size_t cbytes = (size_t)nk * n * n * sizeof(float2);
    int rc = ht_grow(&ctx->d_cwork, &ctx->cwork_bytes, cbytes, "smoothing buffer");
    if (rc == HT_OK) rc = ht_grow(&ctx->d_cwork2, &ctx->cwork2_bytes, cbytes, "smoothing buffer 2");
    if (rc == HT_OK) rc = transposed_plans(ctx, n);
    if (rc == HT_OK) rc = transposed_plane_plans(ctx, n, zhi - zlo);
    if (rc != HT_OK) return rc;
    // window table (W / n^3 per distinct integer |k|^2), shared with the other paths
    const int h = n / 2;
    const int nvals = 3 * h * h + 1;
    rc = ht_grow(&ctx->d_win, &ctx->win_bytes, (size_t)nvals * sizeof(float), "window table");
    if (rc != HT_OK) return rc;
    const double dk = 2.0 * 3.14159265358979323846 / boxsize;
    window_table_kernel<<<(nvals + 255) / 256, 256, 0, st>>>((float*)ctx->d_win, nvals, dk, Rf,
                                                             wsmooth, 1.0 / ((double)n * n * n));
    HT_CUDA_TRY(cudaGetLastError(), "window_table_kernel launch");
    float2* A = (float2*)ctx->d_cwork;
    float2* B = (float2*)ctx->d_cwork2;
    const dim3 blk(32, 8);
    t1_window_kernel<<<dim3((unsigned)((nk + 31) / 32), (unsigned)((n + 31) / 32), (unsigned)n),
                       blk, 0, st>>>((const float2*)d_delta_k, A, n, (int)nk,
                                     (const float*)ctx->d_win);
    HT_CUDA_TRY(cudaGetLastError(), "t1_window_kernel launch");
    if (cufftSetStream(ctx->tp_plan_n, st) != CUFFT_SUCCESS ||
        cufftSetStream(ctx->tp_plan_y, st) != CUFFT_SUCCESS ||
        cufftSetStream(ctx->tp_plan_x, st) != CUFFT_SUCCESS)
        return ht_fail(HT_ERR_CUDA, "cufftSetStream failed");
    cufftResult r = cufftExecC2C(ctx->tp_plan_n, (cufftComplex*)A, (cufftComplex*)A, CUFFT_INVERSE);
    if (r != CUFFT_SUCCESS) return ht_fail(HT_ERR_CUDA, "cufftExecC2C (z) failed with code " + std::to_string((int)r));
    const int zc = zhi - zlo;
    t2_kernel<<<dim3((unsigned)((zc + 31) / 32), (unsigned)((n + 31) / 32), (unsigned)nk), blk, 0,
                st>>>(A, B, n, (int)nk, zlo, zhi);
    HT_CUDA_TRY(cudaGetLastError(), "t2_kernel launch");
    float2* Bz = B + (size_t)zlo * nk * n;
    r = cufftExecC2C(ctx->tp_plan_y, (cufftComplex*)Bz, (cufftComplex*)Bz, CUFFT_INVERSE);
    if (r != CUFFT_SUCCESS) return ht_fail(HT_ERR_CUDA, "cufftExecC2C (y) failed with code " + std::to_string((int)r));
    const int m = n / 2;
    t3_pack_kernel<<<dim3((unsigned)((m / 2 + 1 + 31) / 32), (unsigned)((n + 31) / 32),
                          (unsigned)zc), blk, 0, st>>>(B, A, n, (int)nk, (const float2*)ctx->d_tw,
                                                       zlo);
    HT_CUDA_TRY(cudaGetLastError(), "t3_pack_kernel launch");
    const size_t off = (size_t)zlo * n * m;   // complex elements of C and of the output
    r = cufftExecC2C(ctx->tp_plan_x, (cufftComplex*)A + off, (cufftComplex*)d_out + off,
                     CUFFT_INVERSE);
    if (r != CUFFT_SUCCESS) return ht_fail(HT_ERR_CUDA, "cufftExecC2C (x) failed with code " + std::to_string((int)r));
    ctx->last_kernels = 4;
    return HT_OK;
}


// --------------------------------------------- fused three-pass inverse FFT (n = 32 T) ----
//
// For tile sides n = 576 and 1152 the six passes of the transposed path can collapse into
// three (ht_fft.cuh): each kernel loads 8 columns along the axis it transforms (64-byte
// segments of 8 neighbours), runs one warp-level inverse FFT per column in shared memory,
// and stores every column contiguously in the next pass's layout (the default at 576 only:
// at 1152 the 64-byte reads keep it slower than the transposed path):
//   Z  window (with 1/n^3) on load, FFT along kz:     (kz, ky, kx) -> A (ky, kx, z)
//   Y  FFT along ky:                                   A (ky, kx, z) -> B (z, kx, y)
//   X  half-length real packing, FFT of n/2 along kx:  B (z, kx, y) -> out (z, y, x)

namespace {

constexpr int kFftCols = 8;   // columns (warps) per CTA

template <int T>
__global__ void __launch_bounds__(256) fft_z_kernel(const float2* __restrict__ in,
                                                    float2* __restrict__ A, int NK,
                                                    const float* __restrict__ tab,
                                                    const float2* __restrict__ twL,
                                                    const float2* __restrict__ tw32) {
    constexpr int N = 32 * T, S = N + 1;
    extern __shared__ float2 sm[];
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int kx0 = blockIdx.x * kFftCols, ky = blockIdx.y;
    const int sy = ky <= N / 2 ? ky : ky - N;
    for (int e = tid; e < kFftCols * N; e += blockDim.x) {
        const int r = e / kFftCols, c = e % kFftCols;      // r = kz
        const int kx = kx0 + c;
        float2 v = make_float2(0.f, 0.f);
        if (kx < NK) {
            const int sz = r <= N / 2 ? r : r - N;
            const float wv = __ldg(tab + (kx * kx + sy * sy + sz * sz));
            v = __ldg(in + ((long long)r * N + ky) * NK + kx);
            v.x *= wv;
            v.y *= wv;
        }
        sm[c * S + r] = v;
    }
    __syncthreads();
    const int kx = kx0 + w;
    if (kx >= NK) return;
    htfft::C2 w32[5];
    htfft::lane_twiddles(lane, tw32, w32);
    float2* col = sm + w * S;
    htfft::warp_ifft<T>(col, twL, lane, w32);
    float2* dst = A + ((long long)ky * NK + kx) * N;
    for (int z = lane; z < N; z += 32) dst[z] = col[z];
}

template <int T>
__global__ void __launch_bounds__(256) fft_y_kernel(const float2* __restrict__ A,
                                                    float2* __restrict__ B, int NK,
                                                    const float2* __restrict__ twL,
                                                    const float2* __restrict__ tw32) {
    constexpr int N = 32 * T, S = N + 1;
    extern __shared__ float2 sm[];
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int z0 = blockIdx.x * kFftCols, kx = blockIdx.y;
    for (int e = tid; e < kFftCols * N; e += blockDim.x) {
        const int r = e / kFftCols, c = e % kFftCols;      // r = ky
        const int z = z0 + c;
        sm[c * S + r] = z < N ? __ldg(A + ((long long)r * NK + kx) * N + z) : make_float2(0.f, 0.f);
    }
    __syncthreads();
    const int z = z0 + w;
    if (z >= N) return;
    htfft::C2 w32[5];
    htfft::lane_twiddles(lane, tw32, w32);
    float2* col = sm + w * S;
    htfft::warp_ifft<T>(col, twL, lane, w32);
    float2* dst = B + ((long long)z * NK + kx) * N;
    for (int y = lane; y < N; y += 32) dst[y] = col[y];
}

// TH = n / 64: the packed rows have m = n / 2 = 32 TH points
template <int TH>
__global__ void __launch_bounds__(256) fft_x_kernel(const float2* __restrict__ B,
                                                    float2* __restrict__ out, int NK,
                                                    const float2* __restrict__ twp,
                                                    const float2* __restrict__ twM,
                                                    const float2* __restrict__ tw32) {
    constexpr int M = 32 * TH, N = 2 * M, S = M + 2;
    extern __shared__ float2 sm[];
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int y0 = blockIdx.x * kFftCols, z = blockIdx.y;
    for (int e = tid; e < kFftCols * NK; e += blockDim.x) {
        const int r = e / kFftCols, c = e % kFftCols;      // r = kx
        const int y = y0 + c;
        sm[c * S + r] = y < N ? __ldg(B + ((long long)z * NK + r) * N + y) : make_float2(0.f, 0.f);
    }
    __syncthreads();
    const int y = y0 + w;
    if (y >= N) return;
    float2* col = sm + w * S;
    // in-place packing: lane handles the pair (k, M - k) for k = lane, lane + 32, ... <= M/2
    for (int k = lane; k <= M / 2; k += 32) {
        const float2 xa = col[k], xb = col[M - k];
        auto pack = [&](float2 a, float2 bb, int kk) {
            const float2 b = make_float2(bb.x, -bb.y);
            const float2 e = make_float2(a.x + b.x, a.y + b.y);
            const float2 d = make_float2(a.x - b.x, a.y - b.y);
            const float2 wv = __ldg(twp + kk);
            const float2 o = make_float2(d.x * wv.x - d.y * wv.y, d.x * wv.y + d.y * wv.x);
            return make_float2(e.x - o.y, e.y + o.x);
        };
        const float2 zk = pack(xa, xb, k);
        const int kh = M - k;
        if (kh != k && kh < M) col[kh] = pack(xb, xa, kh);
        col[k] = zk;
    }
    __syncwarp();
    htfft::C2 w32[5];
    htfft::lane_twiddles(lane, tw32, w32);
    htfft::warp_ifft<TH>(col, twM, lane, w32);
    float2* dst = out + ((long long)z * N + y) * M;
    for (int j = lane; j < M; j += 32) dst[j] = col[j];
}

}  // namespace

// Twiddle tables of the fused and pencil paths for side n (FP64 on the host, stored as
// FP32), at these offsets of ctx->d_ftw (fused_tw):
//   0         e^{2 pi i j / n}, j < n (natural order: the real-packing twiddles)
//   n         e^{2 pi i j / 32}, j < 32 (the cross-lane stages)
//   n + 32    e^{2 pi i l k2 / n} at [32 k2 + l], k2 < n/32 (warp FFT step 2, lane-major)
//   2 n + 32  e^{2 pi i l k2 / (n/2)} at [32 k2 + l], k2 < n/64 (the half-length FFT)
struct FusedTw {
    const float2 *nat, *w32, *lmL, *lmM;
};
static FusedTw fused_tw(const ht_ctx* ctx, int n) {
    const float2* t = (const float2*)ctx->d_ftw;
    return {t, t + n, t + n + 32, t + 2 * n + 32};
}

static int fused_tables(ht_ctx* ctx, int n) {
    if (ctx->fz_n == n) return HT_OK;
    std::vector<float2> t((size_t)n + 32 + n + n / 2);
    auto w = [](double j, double N) {
        const double ph = 2.0 * 3.14159265358979323846 * j / N;
        return make_float2((float)cos(ph), (float)sin(ph));
    };
    for (int j = 0; j < n; ++j) t[j] = w(j, n);
    for (int j = 0; j < 32; ++j) t[n + j] = w(j, 32);
    const size_t oL = (size_t)n + 32, oM = (size_t)2 * n + 32;
    for (int k2 = 0; k2 < n / 32; ++k2)
        for (int l = 0; l < 32; ++l) t[oL + 32 * k2 + l] = w((double)l * k2, n);
    for (int k2 = 0; k2 < n / 64; ++k2)
        for (int l = 0; l < 32; ++l) t[oM + 32 * k2 + l] = w((double)l * k2, n / 2);
    int rc = ht_grow(&ctx->d_ftw, &ctx->ftw_bytes, t.size() * sizeof(float2), "FFT twiddles");
    if (rc != HT_OK) return rc;
    HT_CUDA_TRY(cudaMemcpy(ctx->d_ftw, t.data(), t.size() * sizeof(float2), cudaMemcpyHostToDevice),
                "twiddle upload");
    float2 c8[8], c9[9], c18[18], c32[32], c36[36];
    for (int j = 0; j < 8; ++j) c8[j] = w(j, 8);
    for (int j = 0; j < 9; ++j) c9[j] = w(j, 9);
    for (int j = 0; j < 18; ++j) c18[j] = w(j, 18);
    for (int j = 0; j < 32; ++j) c32[j] = w(j, 32);
    for (int j = 0; j < 36; ++j) c36[j] = w(j, 36);
    HT_CUDA_TRY(cudaMemcpyToSymbol(htfft::c_w8, c8, sizeof c8), "c_w8");
    HT_CUDA_TRY(cudaMemcpyToSymbol(htfft::c_w32, c32, sizeof c32), "c_w32");
    HT_CUDA_TRY(cudaMemcpyToSymbol(htfft::c_w9, c9, sizeof c9), "c_w9");
    HT_CUDA_TRY(cudaMemcpyToSymbol(htfft::c_w18, c18, sizeof c18), "c_w18");
    HT_CUDA_TRY(cudaMemcpyToSymbol(htfft::c_w36, c36, sizeof c36), "c_w36");
    ctx->fz_n = n;
    return HT_OK;
}

template <int T>
static int launch_fused(ht_ctx* ctx, const void* d_delta_k, float* d_out, cudaStream_t st) {
    constexpr int n = 32 * T;
    const int nk = n / 2 + 1, m = n / 2;
    const size_t smz = (size_t)kFftCols * (n + 1) * sizeof(float2);
    const size_t smx = (size_t)kFftCols * (m + 2) * sizeof(float2);
    const FusedTw tw = fused_tw(ctx, n);
    const float2* twL = tw.lmL;
    const float2* twM = tw.lmM;
    const float2* tw32 = tw.w32;
    HT_CUDA_TRY(cudaFuncSetAttribute(fft_z_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smz), "fft_z smem");
    HT_CUDA_TRY(cudaFuncSetAttribute(fft_y_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smz), "fft_y smem");
    HT_CUDA_TRY(cudaFuncSetAttribute(fft_x_kernel<T / 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smx), "fft_x smem");
    float2* A = (float2*)ctx->d_cwork;
    float2* B = (float2*)ctx->d_cwork2;
    fft_z_kernel<T><<<dim3((unsigned)((nk + kFftCols - 1) / kFftCols), (unsigned)n), 256, smz, st>>>(
        (const float2*)d_delta_k, A, nk, (const float*)ctx->d_win, twL, tw32);
    HT_CUDA_TRY(cudaGetLastError(), "fft_z_kernel launch");
    fft_y_kernel<T><<<dim3((unsigned)((n + kFftCols - 1) / kFftCols), (unsigned)nk), 256, smz, st>>>(
        A, B, nk, twL, tw32);
    HT_CUDA_TRY(cudaGetLastError(), "fft_y_kernel launch");
    fft_x_kernel<T / 2><<<dim3((unsigned)((n + kFftCols - 1) / kFftCols), (unsigned)n), 256, smx, st>>>(
        B, (float2*)d_out, nk, (const float2*)ctx->d_tw, twM, tw32);
    HT_CUDA_TRY(cudaGetLastError(), "fft_x_kernel launch");
    (void)m;
    return HT_OK;
}

static int smooth_tile_fused(ht_ctx* ctx, const void* d_delta_k, float* d_out, int n,
                             double boxsize, double Rf, int wsmooth, cudaStream_t st) {
    const long long nk = n / 2 + 1;
    const size_t cbytes = (size_t)nk * n * n * sizeof(float2);
    int rc = ht_grow(&ctx->d_cwork, &ctx->cwork_bytes, cbytes, "smoothing buffer");
    if (rc == HT_OK) rc = ht_grow(&ctx->d_cwork2, &ctx->cwork2_bytes, cbytes, "smoothing buffer 2");
    if (rc == HT_OK) rc = transposed_plans(ctx, n);   // the pack twiddles e^{2 pi i k / n}
    if (rc == HT_OK) rc = fused_tables(ctx, n);
    if (rc != HT_OK) return rc;
    const int h = n / 2;
    const int nvals = 3 * h * h + 1;
    rc = ht_grow(&ctx->d_win, &ctx->win_bytes, (size_t)nvals * sizeof(float), "window table");
    if (rc != HT_OK) return rc;
    const double dk = 2.0 * 3.14159265358979323846 / boxsize;
    window_table_kernel<<<(nvals + 255) / 256, 256, 0, st>>>((float*)ctx->d_win, nvals, dk, Rf,
                                                             wsmooth, 1.0 / ((double)n * n * n));
    HT_CUDA_TRY(cudaGetLastError(), "window_table_kernel launch");
    rc = n == 1152 ? launch_fused<36>(ctx, d_delta_k, d_out, st)
                   : launch_fused<18>(ctx, d_delta_k, d_out, st);
    if (rc != HT_OK) return rc;
    ctx->last_kernels = 4;
    return HT_OK;
}

// ------------------------------------------- pencil three-pass inverse FFT (n = 32 T) ----
//
// The spectrum of a tile is the same for every filter, so it is transposed once into
// pencils P (ky, kx, kz), kz contiguous (ht_spectrum_pencil).  Each filter then runs three
// passes:
//   Z  window (with 1/n^3), FFT along kz:        P (ky, kx, kz) -> B (kx, z, ky)
//   Y  FFT along ky:                             B (kx, z, ky)  -> C (z, y, kx)
//   X  half-length real packing, FFT of n/2:     C (z, y, kx)   -> out (z, y, x)
// B holds only z in [zlo, zlo + Rz) and C only those z with y in [ylo, ylo + Ry): just the
// output rows (z, y) in that range are written.  A peak scan of the region
// [lo + 1, hi - 1)^3 reads the rows (z, y) in [lo, hi)^2 only.  C rows are padded to a
// multiple of 16 complex values (128 bytes).
//
// All three kernels are persistent; columns and rows arrive by 1-D bulk copies
// (cp.async.bulk, completing on an mbarrier that one thread polls with a bounded wait).
// Z and Y: a CTA takes neighbouring columns (one warp each), reads them from its shared-
// memory slot into registers, transforms, writes the results in lane-major order and
// stores them in pieces of the next layout.  Z: 8 columns, the results reuse the slot, the
// next item's columns are requested after the store, two CTAs per SM overlap one's copies
// with the other's arithmetic (64-byte pieces; measured faster than 4 columns, and as fast
// as one CTA per SM with a second slot).  Y: 4 columns with a separate result area, the
// next columns requested as soon as the current ones sit in registers, three CTAs per SM
// (measured 16 % faster than the Z shape on the full Y pass).  X: every warp streams rows
// through a two-slot ring of its own, the next row in flight while the current one is
// transformed.

namespace {

// Z / Y CTA shapes: COLS neighbouring columns (one warp each) per work item; SEP gives the
// bulk-copy destination a buffer of its own, so that the next item's columns are requested
// as soon as the current ones sit in registers (else the row-major outputs reuse the slot
// and the request follows the store); CTAS is the occupancy the launch bounds aim for.
template <int COLS, bool SEP, int CTAS>
struct PencilShape {
    static constexpr int cols = COLS, threads = 32 * COLS, ctas = CTAS;
    static constexpr bool sep = SEP;
};
using PencilZ = PencilShape<8, false, 2>;   // 64-byte pieces of B rows
using PencilY = PencilShape<4, true, 3>;    // 32-byte pieces of C rows

// row-major column of 33 T slots (km_slot), padded so that the COLS columns of a CTA
// start 32 / COLS banks apart (conflict-free transposed reads, 64-bit accesses)
template <int T, int COLS>
__host__ __device__ constexpr int pencil_stride() {
    return 33 * T + (((16 / COLS - 33 * T) % 16) + 16) % 16;
}

// Z / Y shared memory: the bulk-copy destination (COLS columns of N), then the row-major
// outputs (COLS columns of S) after it or over it
template <int T, class Sh>
constexpr size_t pencil_smem_yz() {
    return (size_t)Sh::cols * ((Sh::sep ? 32 * T : 0) + pencil_stride<T, Sh::cols>()) *
           sizeof(float2);
}

// C rows hold the n/2 + 1 modes of one (z, y) padded to a multiple of 16 complex values
// (128 bytes): the Y pass stores 64-byte pieces into them, which then start on 64-byte
// boundaries and cover whole 32-byte sectors (an unaligned pitch made every piece touch a
// third, partly written sector).
__host__ __device__ constexpr int pencil_row_pitch(int n) {
    return (n / 2 + 1 + 15) & ~15;
}

// X: a warp's slot holds 33 TH complex values rounded up to even (16-byte slots), or a
// padded C row if that is longer, two slots per warp
template <int TH>
__host__ __device__ constexpr int pencil_slot_x() {
    return ((33 * TH + 1) & ~1) > pencil_row_pitch(64 * TH) ? ((33 * TH + 1) & ~1)
                                                             : pencil_row_pitch(64 * TH);
}
template <int TH>
constexpr size_t pencil_smem_x() {
    return (size_t)8 * 2 * pencil_slot_x<TH>() * sizeof(float2);
}

// Rows of the 32-point DFTs finished in registers after the transpose: up to 32 per
// column, so that 8 columns give at most one per thread; rows beyond (T > 32) are finished
// across the lanes in the warp.
template <int T>
__host__ __device__ constexpr int pencil_rows() {
    return T < 32 ? T : 32;
}

// The second half of the Z / Y transforms and the transposed store.  On entry warp w < ncol
// holds its column's twiddled inner transform X[lane][k2] in registers, rows k2 >=
// pencil_rows already finished across lanes (y[k2 + T bitrev5(lane)]): it writes every row
// k2 to slots k2 * 33 + (lane or k1), the CTA finishes the remaining 32-point row DFTs one
// per thread, and dst[r * pitch + c] = column c's output lo + r for r < R, c < ncol.
template <int T, int S, int COLS>
__device__ __forceinline__ void pencil_finish(float2* __restrict__ ob,
                                              const htfft::C2 (&v)[T], float2* dst,
                                              long long pitch, int lo, int R, int ncol,
                                              int tid) {
    constexpr int TB = pencil_rows<T>();
    const int lane = tid & 31, w = tid >> 5;
    if (w < ncol) {
#pragma unroll
        for (int k2 = 0; k2 < TB; ++k2) ob[w * S + k2 * 33 + lane] = make_float2(v[k2].x, v[k2].y);
        const int k1 = htfft::bitrev5(lane);
#pragma unroll
        for (int k2 = TB; k2 < T; ++k2) ob[w * S + k2 * 33 + k1] = make_float2(v[k2].x, v[k2].y);
    }
    __syncthreads();
    for (int j = tid; j < ncol * TB; j += 32 * COLS) {
        const int c = j / TB, k2 = j - c * TB;
        htfft::dft32_row(ob + c * S + k2 * 33);
    }
    __syncthreads();
    // thread tid stores column c = tid % COLS of rows r = tid / COLS, r + 32, ...; the slot
    // km_slot(i) = (i mod T) * 33 + i / T of output i = lo + r is advanced by 32 outputs per
    // step without a division
    const int c = tid % COLS;
    if (c < ncol) {
        constexpr int Q = 32 / T, M = 32 % T;
        int r = tid / COLS;
        const int i = lo + r;
        int k1 = i / T, rem = i - k1 * T;
        float2* d = dst + (long long)r * pitch + c;
        const float2* o = ob + c * S;
        const long long step = 32LL * pitch;
        for (; r < R; r += 32) {
            *d = o[rem * 33 + k1];
            d += step;
            k1 += Q;
            rem += M;
            if (rem >= T) {
                rem -= T;
                ++k1;
            }
        }
    }
}

template <int T, class Sh>
__global__ void __launch_bounds__(Sh::threads, Sh::ctas) pz_kernel(
    const float2* __restrict__ P, float2* __restrict__ B, int NK, int zlo, int Rz,
    const float* __restrict__ U, const int32_t* __restrict__ urow, int UP,
    const float2* __restrict__ twL, const float2* __restrict__ tw32,
    int32_t* __restrict__ status, long long wait_ns) {
    constexpr int COLS = Sh::cols, N = 32 * T, S = pencil_stride<T, COLS>(), NB = N / COLS,
                  H = T / 2;
    extern __shared__ __align__(128) float2 sm[];
    float2* in = sm;                          // the input columns, N each
    float2* ob = Sh::sep ? sm + COLS * N : sm;   // the row-major columns, S each
    __shared__ __align__(8) unsigned long long bar;
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int ntasks = NK * NB;               // task = kx * NB + ky block
    if (tid == 0) {
        htasync::bar_init(&bar, 1);
        htasync::bar_init_fence();
    }
    __syncthreads();
    auto issue = [&](int tk) {                // thread 0
        const int kx = tk / NB, ky0 = (tk - kx * NB) * COLS;
        htasync::bar_expect(&bar, COLS * N * (unsigned)sizeof(float2));
        for (int c = 0; c < COLS; ++c)
            htasync::bulk_load(in + c * N, P + ((long long)(ky0 + c) * NK + kx) * N,
                               N * (unsigned)sizeof(float2), &bar);
    };
    int task = blockIdx.x;
    if (tid == 0 && task < ntasks) issue(task);
    htfft::C2 w32[5];
    htfft::lane_twiddles(lane, tw32, w32);
    unsigned parity = 0;
    bool ok = true;
    for (; task < ntasks; task += gridDim.x) {
        const int kx = task / NB, ky0 = (task - kx * NB) * COLS, ky = ky0 + w;
        // Window W(kx^2 + sy^2 + sz^2) from the column's row of U (urow: the row of this
        // (kx, ky)), loaded before the wait (it does not depend on the copy).  Each value
        // is fetched once: kz = lane + 32 t < N/2 for t < H; the upper half kz' = N - kz
        // (same sz^2) is lane 32 - lane's value at t' = T - 1 - t, handed over by a
        // shuffle.  Lane 0's upper half kz = 32 t has |sz| = 32 (T - t): its own lower-
        // half value, or N/2 (wmid) at t = H.
        const float* wrow = U + (long long)__ldg(urow + (long long)kx * N + ky) * UP;
        float wl[H];
#pragma unroll
        for (int t = 0; t < H; ++t) wl[t] = __ldg(wrow + lane + 32 * t);
        const float wmid = __ldg(wrow + N / 2);
        ok = tid == 0 ? htasync::bar_wait(&bar, parity, wait_ns) : true;
        if (__syncthreads_or(!ok)) {
            ok = false;
            break;
        }
        parity ^= 1;
        htfft::C2 v[T];
        const float2* col = in + w * N;
#pragma unroll
        for (int t = 0; t < T; ++t) v[t] = htfft::to_c2(col[lane + 32 * t]);
        __syncthreads();                      // every column is in registers
        if (Sh::sep && tid == 0 && task + (int)gridDim.x < ntasks) {
            htasync::fence_async_smem();
            issue(task + (int)gridDim.x);
        }
#pragma unroll
        for (int t = 0; t < T; ++t) {
            float wv;
            if (t < H) {
                wv = wl[t];
            } else {
                const float sh = __shfl_sync(0xffffffffu, wl[T - 1 - t], (32 - lane) & 31);
                const float own = t == H ? wmid : wl[(T - t) % H];
                wv = lane == 0 ? own : sh;
            }
            v[t].x *= wv;
            v[t].y *= wv;
        }
        htfft::warp_ifft_inner<T>(v, twL, lane);
        htfft::cross32<T, pencil_rows<T>()>(v, lane, w32);
        pencil_finish<T, S, COLS>(ob, v, B + (long long)kx * Rz * N + ky0, N, zlo, Rz, COLS,
                                  tid);
        // with a separate slot the barrier at the top of the next item orders these reads
        // of ob before its writes; else the slot is refilled once every thread is done
        if (!Sh::sep) {
            __syncthreads();
            if (tid == 0 && task + (int)gridDim.x < ntasks) {
                htasync::fence_async_smem();
                issue(task + (int)gridDim.x);
            }
        }
    }
    if (!ok && tid == 0) {
        // record the timeout, then wait (bounded) for the copy still in flight
        atomicExch(status, kStatusWaitTimeout);
        htasync::bar_wait(&bar, parity, wait_ns);
    }
}

template <int T, class Sh>
__global__ void __launch_bounds__(Sh::threads, Sh::ctas) py_kernel(
    const float2* __restrict__ B, float2* __restrict__ C, int NK, int NKP, int Rz, int ylo,
    int Ry, const float2* __restrict__ twL, const float2* __restrict__ tw32,
    int32_t* __restrict__ status, long long wait_ns) {
    constexpr int COLS = Sh::cols, N = 32 * T, S = pencil_stride<T, COLS>();
    extern __shared__ __align__(128) float2 sm[];
    float2* in = sm;
    float2* ob = Sh::sep ? sm + COLS * N : sm;
    __shared__ __align__(8) unsigned long long bar;
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int NKB = (NK + COLS - 1) / COLS;
    const int ntasks = Rz * NKB;              // task = zr * NKB + kx block
    if (tid == 0) {
        htasync::bar_init(&bar, 1);
        htasync::bar_init_fence();
    }
    __syncthreads();
    auto issue = [&](int tk) {                // thread 0
        const int zr = tk / NKB, kx0 = (tk - zr * NKB) * COLS;
        const int ncol = min(COLS, NK - kx0);
        htasync::bar_expect(&bar, ncol * N * (unsigned)sizeof(float2));
        for (int c = 0; c < ncol; ++c)
            htasync::bulk_load(in + c * N, B + ((long long)(kx0 + c) * Rz + zr) * N,
                               N * (unsigned)sizeof(float2), &bar);
    };
    int task = blockIdx.x;
    if (tid == 0 && task < ntasks) issue(task);
    htfft::C2 w32[5];
    htfft::lane_twiddles(lane, tw32, w32);
    unsigned parity = 0;
    bool ok = true;
    for (; task < ntasks; task += gridDim.x) {
        const int zr = task / NKB, kx0 = (task - zr * NKB) * COLS;
        const int ncol = min(COLS, NK - kx0);
        ok = tid == 0 ? htasync::bar_wait(&bar, parity, wait_ns) : true;
        if (__syncthreads_or(!ok)) {
            ok = false;
            break;
        }
        parity ^= 1;
        htfft::C2 v[T];
        if (w < ncol) {
            const float2* col = in + w * N;
#pragma unroll
            for (int t = 0; t < T; ++t) v[t] = htfft::to_c2(col[lane + 32 * t]);
        }
        __syncthreads();                      // the columns are in registers
        if (Sh::sep && tid == 0 && task + (int)gridDim.x < ntasks) {
            htasync::fence_async_smem();
            issue(task + (int)gridDim.x);
        }
        if (w < ncol) {   // warp-uniform
            htfft::warp_ifft_inner<T>(v, twL, lane);
            htfft::cross32<T, pencil_rows<T>()>(v, lane, w32);
        }
        pencil_finish<T, S, COLS>(ob, v, C + (long long)zr * Ry * NKP + kx0, NKP, ylo, Ry,
                                  ncol, tid);
        if (!Sh::sep) {
            __syncthreads();
            if (tid == 0 && task + (int)gridDim.x < ntasks) {
                htasync::fence_async_smem();
                issue(task + (int)gridDim.x);
            }
        }
    }
    if (!ok && tid == 0) {
        atomicExch(status, kStatusWaitTimeout);
        htasync::bar_wait(&bar, parity, wait_ns);
    }
}

// TH = n / 64: the packed rows have M = n / 2 = 32 TH points.  Every warp streams rows
// r = global warp, + total warps, ... through two slots: row r + stride is copied into the
// other slot while row r is packed, transformed and stored.  C rows start NKP values apart;
// a copy takes the first n/2 + 1 values rounded up to even (16 bytes).  At TH = 18 the
// 32-point DFTs of the TH rows of the four-step transform are finished after a transpose
// through the row's slot, one row per lane (lanes TH..31 idle): a 32-point DFT in
// registers costs about half the instructions of five shuffle stages over 18 rows.  At
// TH = 9 the shuffle stages stay (measured faster: 9 busy lanes save little there).
template <int TH>
__global__ void __launch_bounds__(256) px_kernel(const float2* __restrict__ C,
                                                 float2* __restrict__ out, int NKP, int zlo,
                                                 int ylo, int Ry, long long rows,
                                                 const float2* __restrict__ twp,
                                                 const float2* __restrict__ twM,
                                                 const float2* __restrict__ tw32,
                                                 int32_t* __restrict__ status,
                                                 long long wait_ns) {
    constexpr int M = 32 * TH, N = 2 * M, S = pencil_slot_x<TH>();
    constexpr bool kRowDft = TH >= 16;
    static_assert(S >= pencil_row_pitch(N) && S >= 33 * TH, "a padded C row must fit a slot");
    extern __shared__ __align__(128) float2 sm[];
    __shared__ __align__(8) unsigned long long bars[8][2];
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    float2* slots = sm + w * 2 * S;
    unsigned long long* bar = bars[w];
    const long long stride = (long long)gridDim.x * 8;
    const unsigned row_bytes = (unsigned)((M + 2) & ~1) * (unsigned)sizeof(float2);
    long long r = (long long)blockIdx.x * 8 + w;
    if (lane == 0) {
        htasync::bar_init(&bar[0], 1);
        htasync::bar_init(&bar[1], 1);
        htasync::bar_init_fence();
        if (r < rows) {
            htasync::bar_expect(&bar[0], row_bytes);
            htasync::bulk_load(slots, C + r * NKP, row_bytes, &bar[0]);
        }
    }
    __syncwarp();
    htfft::C2 w32[5];
    if (!kRowDft) htfft::lane_twiddles(lane, tw32, w32);
    bool ok = true;
    int i = 0;
    for (; r < rows; ++i, r += stride) {
        const int s = i & 1;
        if (lane == 0 && r + stride < rows) {   // the other slot was released at the end of i - 1
            htasync::fence_async_smem();
            htasync::bar_expect(&bar[s ^ 1], row_bytes);
            htasync::bulk_load(slots + (s ^ 1) * S, C + (r + stride) * NKP, row_bytes,
                               &bar[s ^ 1]);
        }
        ok = lane == 0 ? htasync::bar_wait(&bar[s], (unsigned)((i >> 1) & 1), wait_ns) : true;
        __syncwarp();
        if (__any_sync(0xffffffffu, !ok)) {
            ok = false;
            break;
        }
        float2* col = slots + s * S;
        // half-length packing on the way into registers: lane's point k = lane + 32 t is
        // z_k = (X[k] + conj X[M-k]) + i e^{2 pi i k/N} (X[k] - conj X[M-k]), from the raw
        // row (no packed copy is written back to shared memory)
        htfft::C2 v[TH];
#pragma unroll
        for (int t = 0; t < TH; ++t) {
            const int k = lane + 32 * t;
            const float2 a = col[k], bb = col[M - k];
            const float2 b = make_float2(bb.x, -bb.y);          // conj X[M - k]
            const float2 e = make_float2(a.x + b.x, a.y + b.y);
            const float2 d = make_float2(a.x - b.x, a.y - b.y);
            const float2 wv = __ldg(twp + k);                   // e^{2 pi i k / N}
            const float2 o = make_float2(d.x * wv.x - d.y * wv.y, d.x * wv.y + d.y * wv.x);
            v[t] = htfft::to_c2(make_float2(e.x - o.y, e.y + o.x));
        }
        const int zr = (int)(r / Ry), yr = (int)(r - (long long)zr * Ry);
        float2* dst = out + ((long long)(zlo + zr) * N + (ylo + yr)) * M;
        if constexpr (!kRowDft) {
            htfft::warp_ifft_regs<TH>(v, twM, lane, w32);
            __syncwarp();
            htfft::warp_ifft_store<TH>(col, v, lane);
            __syncwarp();
#pragma unroll
            for (int t = 0; t < TH; ++t)
                dst[lane + 32 * t] = col[htfft::lm_slot<TH>(lane + 32 * t)];
        } else {
            htfft::warp_ifft_inner<TH>(v, twM, lane);
            __syncwarp();                      // every lane has read its points of the row
#pragma unroll
            for (int k2 = 0; k2 < TH; ++k2)
                col[k2 * 33 + lane] = make_float2(v[k2].x, v[k2].y);
            __syncwarp();
            if (lane < TH) htfft::dft32_row(col + lane * 33);
            __syncwarp();
            // output i = lane + 32 t sits at km_slot(i) = (i mod TH) * 33 + i / TH
            constexpr int Q = 32 / TH, MR = 32 % TH;
            int k1 = lane / TH, rem = lane - k1 * TH;
#pragma unroll
            for (int t = 0; t < TH; ++t) {
                dst[lane + 32 * t] = col[rem * 33 + k1];
                k1 += Q;
                rem += MR;
                if (rem >= TH) {
                    rem -= TH;
                    ++k1;
                }
            }
        }
        __syncwarp();
    }
    if (!ok && lane == 0) {
        // record the timeout, then wait (bounded) for this warp's copies in flight
        atomicExch(status, kStatusWaitTimeout);
        htasync::bar_wait(&bar[i & 1], (unsigned)((i >> 1) & 1), wait_ns);
        if (r + stride < rows)
            htasync::bar_wait(&bar[(i & 1) ^ 1], (unsigned)(((i + 1) >> 1) & 1), wait_ns);
    }
}

}  // namespace

// Tile sides the pencil path handles: n = 32 T with T in {18, 36}.
static bool pencil_side(int n) { return n == 576 || n == 1152; }

// Row pitch of the window rows U: n/2 + 1 values rounded up to a multiple of 4.
static int window_row_pitch(int n) { return (n / 2 + 1 + 3) & ~3; }

// Once per side n: the distinct b = kx^2 + sy^2 over the rfft modes (kx <= n/2, sy the
// signed ky), ascending, then for every (kx, ky) the index of its b among them, in one
// buffer: [distinct values][row index, kx-major].  103,797 values at n = 1152.
static int window_rows_index(ht_ctx* ctx, int n, cudaStream_t st) {
    if (ctx->wb_n == n) return HT_OK;
    const int h = n / 2, nk = h + 1;
    const int bmax = 2 * h * h;
    std::vector<int32_t> at((size_t)bmax + 1, -1);
    for (int kx = 0; kx < nk; ++kx)
        for (int sy = 0; sy <= h; ++sy) at[(size_t)kx * kx + (size_t)sy * sy] = 0;
    std::vector<int32_t> buf;
    for (int b = 0; b <= bmax; ++b)
        if (at[b] == 0) {
            at[b] = (int32_t)buf.size();
            buf.push_back(b);
        }
    const int count = (int)buf.size();
    buf.resize((size_t)count + (size_t)nk * n);
    for (int kx = 0; kx < nk; ++kx)
        for (int ky = 0; ky < n; ++ky) {
            const int sy = ky <= h ? ky : ky - n;
            buf[(size_t)count + (size_t)kx * n + ky] = at[(size_t)kx * kx + (size_t)sy * sy];
        }
    // the buffer may still be read by a Z pass of the previous side queued on st
    HT_CUDA_TRY(cudaStreamSynchronize(st), "window row index: stream sync");
    int rc = ht_grow(&ctx->d_wb, &ctx->wb_bytes, buf.size() * sizeof(int32_t),
                     "window row index");
    if (rc != HT_OK) return rc;
    HT_CUDA_TRY(cudaMemcpy(ctx->d_wb, buf.data(), buf.size() * sizeof(int32_t),
                           cudaMemcpyHostToDevice), "window row index upload");
    ctx->wb_n = n;
    ctx->wb_count = count;
    return HT_OK;
}

// Per filter, after the window table: the rows U of every distinct b.
static int window_rows(ht_ctx* ctx, int n, cudaStream_t st) {
    int rc = window_rows_index(ctx, n, st);
    if (rc != HT_OK) return rc;
    const int UP = window_row_pitch(n);
    rc = ht_grow(&ctx->d_wu, &ctx->wu_bytes, (size_t)ctx->wb_count * UP * sizeof(float),
                 "window rows");
    if (rc != HT_OK) return rc;
    window_rows_kernel<<<(unsigned)((ctx->wb_count + 31) / 32), dim3(32, 8), 0, st>>>(
        (const float*)ctx->d_win, (const int32_t*)ctx->d_wb, ctx->wb_count, n / 2, UP,
        (float*)ctx->d_wu);
    HT_CUDA_TRY(cudaGetLastError(), "window_rows_kernel launch");
    return HT_OK;
}

// Z, Y and X passes from pencils P, through B and C (C may reuse P's buffer: P is read
// only by the first pass).  Persistent grids: as many CTAs as fit on the device, capped by
// the work items.
template <int T>
static int launch_pencil(ht_ctx* ctx, const float2* P, float2* B, float2* C, float2* d_out,
                         int zlo, int zhi, int ylo, int yhi, cudaStream_t st) {
    constexpr int n = 32 * T, TH = T / 2;
    const int nk = n / 2 + 1, nkp = pencil_row_pitch(n), Rz = zhi - zlo, Ry = yhi - ylo;
    const size_t smz = pencil_smem_yz<T, PencilZ>(), smy = pencil_smem_yz<T, PencilY>(),
                 smx = pencil_smem_x<TH>();
    HT_CUDA_TRY(cudaFuncSetAttribute(pz_kernel<T, PencilZ>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smz), "pz smem");
    HT_CUDA_TRY(cudaFuncSetAttribute(py_kernel<T, PencilY>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smy), "py smem");
    HT_CUDA_TRY(cudaFuncSetAttribute(px_kernel<TH>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smx), "px smem");
    int bz = 0, by = 0, bx = 0;
    HT_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bz, pz_kernel<T, PencilZ>, PencilZ::threads, smz), "pz occupancy");
    HT_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&by, py_kernel<T, PencilY>, PencilY::threads, smy), "py occupancy");
    HT_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bx, px_kernel<TH>, 256, smx), "px occupancy");
    if (bz < 1 || by < 1 || bx < 1) return ht_fail(HT_ERR_CUDA, "pencil kernels do not fit an SM");
    const FusedTw tw = fused_tw(ctx, n);
    int32_t* status = ht_status_word(ctx);
    const long long sms = ctx->num_sms;
    const long long zt = (long long)nk * (n / PencilZ::cols);
    const long long yt = (long long)Rz * ((nk + PencilY::cols - 1) / PencilY::cols);
    const long long rows = (long long)Rz * Ry;
    const unsigned gz = (unsigned)std::min(zt, sms * bz);
    const unsigned gy = (unsigned)std::min(yt, sms * by);
    const unsigned gx = (unsigned)std::min((rows + 7) / 8, sms * bx);
    const int32_t* urow = (const int32_t*)ctx->d_wb + ctx->wb_count;
    pz_kernel<T, PencilZ><<<gz, PencilZ::threads, smz, st>>>(
        P, B, nk, zlo, Rz, (const float*)ctx->d_wu, urow, window_row_pitch(n), tw.lmL, tw.w32,
        status, ctx->wait_ns);
    HT_CUDA_TRY(cudaGetLastError(), "pz_kernel launch");
    py_kernel<T, PencilY><<<gy, PencilY::threads, smy, st>>>(B, C, nk, nkp, Rz, ylo, Ry,
                                                             tw.lmL, tw.w32, status,
                                                             ctx->wait_ns);
    HT_CUDA_TRY(cudaGetLastError(), "py_kernel launch");
    px_kernel<TH><<<gx, 256, smx, st>>>(C, d_out, nkp, zlo, ylo, Ry, rows, tw.nat, tw.lmM,
                                        tw.w32, status, ctx->wait_ns);
    HT_CUDA_TRY(cudaGetLastError(), "px_kernel launch");
    return HT_OK;
}

// Window table W / n^3 per distinct integer |k|^2 (the 1/n^3 of the inverse FFT folded in).
static int scaled_window_table(ht_ctx* ctx, int n, double boxsize, double Rf, int wsmooth,
                               cudaStream_t st) {
    const int h = n / 2;
    const int nvals = 3 * h * h + 1;
    int rc = ht_grow(&ctx->d_win, &ctx->win_bytes, (size_t)nvals * sizeof(float), "window table");
    if (rc != HT_OK) return rc;
    const double dk = 2.0 * 3.14159265358979323846 / boxsize;
    window_table_kernel<<<(nvals + 255) / 256, 256, 0, st>>>((float*)ctx->d_win, nvals, dk, Rf,
                                                             wsmooth, 1.0 / ((double)n * n * n));
    HT_CUDA_TRY(cudaGetLastError(), "window_table_kernel launch");
    return HT_OK;
}

// Spectrum (kz, ky, kx) -> pencils (ky, kx, kz) on stream st (the t1 transpose, no window).
static int launch_pencil_transpose(const float2* in, float2* P, int n, cudaStream_t st) {
    const int nk = n / 2 + 1;
    t1_window_kernel<<<dim3((unsigned)((nk + 31) / 32), (unsigned)((n + 31) / 32), (unsigned)n),
                       dim3(32, 8), 0, st>>>(in, P, n, nk, nullptr);
    HT_CUDA_TRY(cudaGetLastError(), "pencil transpose launch");
    return HT_OK;
}

// One filter from pencils P: output rows (z, y) in [zlo, zhi) x [ylo, yhi).  P may be the
// context's first smoothing buffer (it is consumed by the first pass, which is why C can
// take the same buffer).
static int smooth_pencil_run(ht_ctx* ctx, const float2* P, float* d_out, int n, double boxsize,
                             double Rf, int wsmooth, int zlo, int zhi, int ylo, int yhi,
                             cudaStream_t st) {
    const size_t nk = (size_t)n / 2 + 1;
    const size_t cbytes = (size_t)pencil_row_pitch(n) * (size_t)(zhi - zlo) * (yhi - ylo) *
                          sizeof(float2);
    // C takes the first buffer; when P lives there too it must already be large enough
    // (a reallocation here would free P before the first pass reads it)
    if ((const void*)P == ctx->d_cwork && ctx->cwork_bytes < cbytes)
        return ht_fail(HT_ERR_STATE, "smooth_pencil_run: pencil buffer smaller than C");
    int rc = ht_grow(&ctx->d_cwork2, &ctx->cwork2_bytes,
                     nk * (size_t)(zhi - zlo) * n * sizeof(float2), "smoothing buffer 2");
    if (rc == HT_OK)   // C rows are padded to 128 bytes
        rc = ht_grow(&ctx->d_cwork, &ctx->cwork_bytes, cbytes, "smoothing buffer");
    if (rc == HT_OK) rc = fused_tables(ctx, n);
    if (rc == HT_OK) rc = scaled_window_table(ctx, n, boxsize, Rf, wsmooth, st);
    if (rc == HT_OK) rc = window_rows(ctx, n, st);
    if (rc != HT_OK) return rc;
    float2* B = (float2*)ctx->d_cwork2;
    float2* C = (float2*)ctx->d_cwork;
    float2* out = (float2*)d_out;
    rc = n == 1152 ? launch_pencil<36>(ctx, P, B, C, out, zlo, zhi, ylo, yhi, st)
                   : launch_pencil<18>(ctx, P, B, C, out, zlo, zhi, ylo, yhi, st);
    if (rc != HT_OK) return rc;
    ctx->last_kernels = 5;
    return HT_OK;
}

// ht_smooth_tile path 4: the pencil passes behind a per-call transpose of the spectrum into
// the context's first buffer (four HBM passes per filter instead of the transposed path's
// six).
static int smooth_tile_pencil(ht_ctx* ctx, const void* d_delta_k, float* d_out, int n,
                              double boxsize, double Rf, int wsmooth, int zlo, int zhi,
                              cudaStream_t st) {
    const size_t nk = (size_t)n / 2 + 1;
    // the buffer holds P, then C (padded rows for z in [zlo, zhi), all y): size it for
    // both before P is written
    const size_t need = std::max(nk * n * n, (size_t)pencil_row_pitch(n) * (zhi - zlo) * n) *
                        sizeof(float2);
    int rc = ht_grow(&ctx->d_cwork, &ctx->cwork_bytes, need, "smoothing buffer");
    if (rc != HT_OK) return rc;
    float2* P = (float2*)ctx->d_cwork;
    rc = launch_pencil_transpose((const float2*)d_delta_k, P, n, st);
    if (rc != HT_OK) return rc;
    rc = smooth_pencil_run(ctx, P, d_out, n, boxsize, Rf, wsmooth, zlo, zhi, 0, n, st);
    if (rc == HT_OK) ctx->last_kernels = 6;
    return rc;
}

extern "C" HT_API int ht_smooth_pencil_supported(int n) { return pencil_side(n) ? 1 : 0; }

extern "C" HT_API int ht_spectrum_pencil(ht_ctx* ctx, const void* d_delta_k, void* d_pencil,
                                         int n, void* stream) {
    HT_RANGE("ht_spectrum_pencil");
    if (!ctx || !d_delta_k || !d_pencil) return ht_fail(HT_ERR_INVALID, "ht_spectrum_pencil: NULL argument");
    if (n < 2 || n > 4096 || (n & 1))
        return ht_fail(HT_ERR_INVALID, "ht_spectrum_pencil: need an even n, 2 <= n <= 4096");
    if (d_pencil == d_delta_k)
        return ht_fail(HT_ERR_INVALID, "ht_spectrum_pencil: the transpose is out of place");
    if (ht_fault_injected("launch")) return ht_fail(HT_ERR_FAULT, "injected launch fault: ht_spectrum_pencil");
    HT_CUDA_TRY(cudaSetDevice(ctx->device), "cudaSetDevice");
    int rc = launch_pencil_transpose((const float2*)d_delta_k, (float2*)d_pencil, n,
                                     (cudaStream_t)stream);
    if (rc != HT_OK) return rc;
    ctx->last_kernels = 1;
    return HT_OK;
}

extern "C" HT_API int ht_smooth_pencil(ht_ctx* ctx, const void* d_pencil, float* d_out, int n,
                                       double boxsize, double Rf, int wsmooth, int lo, int hi,
                                       void* stream) {
    HT_RANGE("ht_smooth_pencil");
    if (!ctx || !d_pencil || !d_out) return ht_fail(HT_ERR_INVALID, "ht_smooth_pencil: NULL argument");
    if (!pencil_side(n))
        return ht_fail(HT_ERR_INVALID, "ht_smooth_pencil: tile side " + std::to_string(n) +
                                           " not supported (576 or 1152)");
    if (lo < 0 || hi > n || lo >= hi)
        return ht_fail(HT_ERR_INVALID, "ht_smooth_pencil: need 0 <= lo < hi <= n");
    int rc = check_window_args("ht_smooth_pencil", boxsize, Rf);
    if (rc != HT_OK) return rc;
    if (ht_fault_injected("launch")) return ht_fail(HT_ERR_FAULT, "injected launch fault: ht_smooth_pencil");
    HT_CUDA_TRY(cudaSetDevice(ctx->device), "cudaSetDevice");
    return smooth_pencil_run(ctx, (const float2*)d_pencil, d_out, n, boxsize, Rf, wsmooth, lo, hi,
                             lo, hi, (cudaStream_t)stream);
}


// ------------------------------------------------------ window + inverse FFT (tile) ----

static int smooth_tile_impl(ht_ctx* ctx, const void* d_delta_k, float* d_out, int n,
                            double boxsize, double Rf, int wsmooth, int zlo, int zhi,
                            void* stream) {
    if (!ctx || !d_delta_k || !d_out) return ht_fail(HT_ERR_INVALID, "ht_smooth_tile: NULL argument");
    if (n < 2 || n > 4096) return ht_fail(HT_ERR_INVALID, "ht_smooth_tile: need 2 <= n <= 4096");
    if (zlo < 0 || zhi > n || zlo >= zhi)
        return ht_fail(HT_ERR_INVALID, "ht_smooth_tile: need 0 <= z_lo < z_hi <= n");
    int rc = check_window_args("ht_smooth_tile", boxsize, Rf);
    if (rc != HT_OK) return rc;
    if (ht_fault_injected("launch")) return ht_fail(HT_ERR_FAULT, "injected launch fault: ht_smooth_tile");
    HT_CUDA_TRY(cudaSetDevice(ctx->device), "cudaSetDevice");
    // path: the pencil passes for n = 576 and 1152, the single 3-D plan for power-of-two
    // sides (and odd ones), the transposed 1-D pipeline otherwise; HT_TUNE_FFT_PATH
    // overrides (1 = 3-D plan, 2 = transposed, 3 = fused, 4 = pencil).  The fused kernels
    // read 64-byte pieces of HBM rows (20.1 ms at 1152 against 16.3 ms transposed); the
    // pencil passes read whole columns.
    const bool pow2 = (n & (n - 1)) == 0;
    const bool fused_ok = n == 576 || n == 1152;
    const int path = ctx->tune_fft_path ? ctx->tune_fft_path
                                        : (pencil_side(n) ? 4 : (pow2 || (n & 1) ? 1 : 2));
    if (path == 4 && pencil_side(n))
        return smooth_tile_pencil(ctx, d_delta_k, d_out, n, boxsize, Rf, wsmooth, zlo, zhi,
                                  (cudaStream_t)stream);
    if (path == 3 && fused_ok)
        return smooth_tile_fused(ctx, d_delta_k, d_out, n, boxsize, Rf, wsmooth,
                                 (cudaStream_t)stream);
    if (path == 2 && (n & 1) == 0 && (long long)n * (n / 2 + 1) < 0x7fffffffLL)
        return smooth_tile_transposed(ctx, d_delta_k, d_out, n, boxsize, Rf, wsmooth, zlo, zhi,
                                      (cudaStream_t)stream);
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

extern "C" HT_API int ht_smooth_tile(ht_ctx* ctx, const void* d_delta_k, float* d_out, int n,
                                     double boxsize, double Rf, int wsmooth, void* stream) {
    HT_RANGE("ht_smooth_tile");
    return smooth_tile_impl(ctx, d_delta_k, d_out, n, boxsize, Rf, wsmooth, 0, n, stream);
}

extern "C" HT_API int ht_smooth_tile_planes(ht_ctx* ctx, const void* d_delta_k, float* d_out,
                                            int n, double boxsize, double Rf, int wsmooth,
                                            int z_lo, int z_hi, void* stream) {
    HT_RANGE("ht_smooth_tile_planes");
    return smooth_tile_impl(ctx, d_delta_k, d_out, n, boxsize, Rf, wsmooth, z_lo, z_hi, stream);
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
    HT_RANGE("ht_smooth_filter");
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
