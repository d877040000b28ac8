/*
 * huntian_b200 -- B200 (sm_100a) kernels for Huntian.jl's halo-finding hot path:
 * peak finding on the filtered linear density field and the radial-shell
 * homogeneous-ellipsoid collapse.
 *
 * C ABI only: plain pointers, sizes and status codes.  Device pointers are raw CUDA
 * device addresses (e.g. Julia's pointer(::CuArray), torch's Tensor.data_ptr());
 * `stream` is a cudaStream_t passed as void* (NULL = legacy default stream).
 *
 * Every entry point returns HT_OK (0) or an error code; ht_last_error() gives the
 * message of the calling thread's last failure.  Nothing exits or traps.
 *
 * Array conventions (the reference's): 3-D fields are Float32, column-major
 * (i fastest), 1-based (i, j, k) in all index outputs.
 *
 * Reference interfaces replaced (guanyilun/Huntian.jl):
 *   ht_peakfind_filter  -> ext/CUDAExt.jl:2876-2936 `_find_peaks_kernel!` (one filter of
 *                          the loop at ext/CUDAExt.jl:2985-3012 behind
 *                          `peak_find_tile_gpu`, stub src/Huntian.jl:387-412)
 *   ht_fields_pack +
 *   ht_shell_analyse    -> ext/CUDAExt.jl:2085-2344 `analyse_peaks_gpu_cuda_multirf`
 *                          (stub src/Huntian.jl:259-281): the gather kernel
 *                          ext/CUDAExt.jl:752-924 and post-process kernel
 *                          ext/CUDAExt.jl:1213-1912
 *   ht_ctx_create       -> per-call uploads of ShellTablesGPU (ext/CUDAExt.jl:16-41), the
 *                          collapse table and the SPH table (ext/CUDAExt.jl:45-52)
 *   ht_smooth_window    -> ext/CUDAExt.jl:2831-2871 `_smooth_window_kernel!`
 *   ht_smooth_tile      -> one filter of ext/CUDAExt.jl:2985-2989 (copy + window +
 *                          irfft of the tile's own rfft, as peak_find_tile_gpu does)
 *   ht_smooth_filter    -> the same for a periodic box delivered as a wrapped tile
 *   ht_spectrum_pencil +
 *   ht_smooth_pencil    -> the loop over filters of ext/CUDAExt.jl:2951-2989 with the
 *                          tile's spectrum kept (transposed once) across filters
 *   ht_peak_lightcone   -> the per-peak host loop of src/MultiResolution.jl:1097-1130
 *                          (peak_redshift, fsc_of_z, the z_max cut)
 *   ht_pack_halos       -> the record loop of src/MultiResolution.jl:1159-1219
 *                          (HaloRecord / ExtHaloRecord, src/IO/Catalog.jl:4-48)
 *   ht_merge_halos      -> src/Merger/Merger.jl:38-104 `merge_catalog` (exclusion and
 *                          volume reduction, src/Merger/Exclusion.jl)
 *   ht_finalize_eulerian -> src/Merger/Merger.jl:114-146 `finalize_eulerian`
 *   ht_fsc_of_z         -> src/HaloFinder/RadialShell.jl:181-195 `fsc_of_z` (host)
 *   ht_ctx_shell_r2     -> the shell_r2 array of src/ShellAnalysisGPU.jl:44-71
 *   ht_evolve_ellipses  -> src/EllipsoidalCollapse/EllipsoidalCollapse.jl:492-590
 *                          `evolve_ellipse_full` (solver = :rk4, or :diffeq through
 *                          `_evolve_diffeq` :440-485), many ellipsoids at once
 *   ht_collapse_table   -> src/EllipsoidalCollapse/CollapseTable.jl:29-76 `make_table` /
 *                          `make_table_threaded` (bin/generate_table.jl --solver rk4|diffeq)
 */
#ifndef HUNTIAN_B200_H
#define HUNTIAN_B200_H

#include <stdint.h>

#if defined(__GNUC__)
#define HT_API __attribute__((visibility("default")))
#else
#define HT_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define HT_OK 0
#define HT_ERR_INVALID 1   /* bad argument (null pointer, size, shape) */
#define HT_ERR_CUDA 2      /* a CUDA runtime call failed */
#define HT_ERR_NOMEM 3     /* device allocation failed */
#define HT_ERR_STATE 4     /* call order (e.g. shell analysis before packing fields) */
#define HT_ERR_CAPACITY 5  /* a size exceeds a documented maximum */
#define HT_ERR_FAULT 6     /* injected host-side fault (HT_FAULT_INJECT, tests only) */

/* shell-walk conventions (which reference routine the results reproduce) */
#define HT_CONV_GPU 0      /* analyse_peaks_gpu_cuda_multirf / ShellAnalysisGPU.analyse_peak_gpu
                              + zvir_half (ext/CUDAExt.jl:1213-1912) */
#define HT_CONV_CPU 1      /* RadialShell.analyse_peak (src/HaloFinder/RadialShell.jl:281-865):
                              lagged mrf counter, d2F without the centre cell that stops at the
                              first out-of-tile cell; requires rmax2rs == 0 */

/* shell-walk execution modes (all return identical results) */
#define HT_MODE_PLAIN 0    /* per-field gathers, static peak-to-warp schedule */
#define HT_MODE_BATCHED 1  /* interleaved cell records, persistent kernel, dynamic queue */
#define HT_MODE_LEARNED 2  /* BATCHED, peaks ordered by a predicted walk length (batch cost) */

typedef struct ht_ctx ht_ctx;

/* Context on one CUDA device: shell tables for hunt radius `nhunt` (cells with
 * r^2 <= nhunt^2, ShellAnalysisGPU.jl:44-71), the collapse table (host Float32,
 * column-major nx*ny*nz, axes X1..Z2 as in the HomelTab header, out_val outside the
 * table: CollapseTable.jl:119-138) and the SPH table atab4 (RadialShell.jl:125-147).
 * Replaces the per-call uploads at ext/CUDAExt.jl:2128-2141.  nhunt must be 1..127. */
HT_API int ht_ctx_create(int device, int nhunt, const float* ct_table_host, int nx, int ny, int nz,
                  double X1, double X2, double Y1, double Y2, double Z1, double Z2,
                  double out_val, ht_ctx** out);
HT_API int ht_ctx_destroy(ht_ctx* ctx);

/* Message of this thread's last failed call ("" if none). */
HT_API const char* ht_last_error(void);

/* Number of shells (distinct r^2, incl. r^2 = 0) and cells of the context's table. */
HT_API int ht_ctx_shell_info(const ht_ctx* ctx, int32_t* nshells, int64_t* ncells);
/* Copy the shell r^2 values (nshells entries) to host memory. */
HT_API int ht_ctx_shell_r2(const ht_ctx* ctx, int32_t* r2_host, int32_t cap);

/* fcrit = 10^x where zvir(x, 0, 0) = 1 + z, by 50 bisection steps on the context's
 * collapse table (RadialShell.jl:181-195).  Host computation. */
HT_API int ht_fsc_of_z(const ht_ctx* ctx, double z, double* fcrit_out);

/* ------------------------------------------------------------- peak finding ---- */

/* Output arrays of the peak finder (device memory, capacity max_peaks each).
 * `count` points to ONE device int64: the running number of stored peaks; it must be
 * zeroed by the caller before the first filter and is advanced by each call.
 * `found` (optional, device int64) accumulates all local maxima including those
 * dropped beyond max_peaks.  lapd may be NULL when no Laplacian field is given. */
typedef struct {
    int32_t* i;
    int32_t* j;
    int32_t* k;
    float* delta;       /* delta_s at the peak (FcRf) */
    float* lapd;        /* lapd_s at the peak (d2Rf), nullable */
    int32_t* filter_idx;
    int64_t* count;
    int64_t* found;     /* nullable */
} ht_peaks;

/* One filter of the peak scan (PeakFind.jl:15-78 semantics): cells of the inner cube
 * (nbuff+1 : n-nbuff)^3 with mask != 1, delta_s >= fcrit and no 26-neighbour strictly
 * above (ties accepted) become peaks, are appended in k/j/i scan order after the
 * peaks already counted, and get mask = 1.  Peaks beyond max_peaks are neither stored
 * nor masked.  Unlike the reference GPU kernel the order is deterministic (scan order),
 * so indices are bit-identical to the CPU peak finder.  d_mask is n^3 Int8 (in/out). */
HT_API int ht_peakfind_filter(ht_ctx* ctx, const float* d_delta_s, const float* d_lapd_s,
                       int8_t* d_mask, int n, int nbuff, float fcrit, int32_t filter_idx,
                       int64_t max_peaks, const ht_peaks* out, void* stream);

/* Smoothing window for the per-filter peak scan: d_out = d_delta_k * Float32(W(|k| Rf))
 * on the rfft grid of an n^3 periodic field of side `boxsize` (complex64, layout
 * (n/2+1, n, n) column-major, i.e. what cuFFT's R2C of the column-major field gives),
 * k = 0 unchanged; wsmooth 0 = Gaussian exp(-(kR/2)^2/2), 3 = that times k^2, otherwise
 * the top-hat 3(sin x - x cos x)/x^3, W evaluated in FP64.  In place is allowed.
 * Replaces ext/CUDAExt.jl:2831-2871 `_smooth_window_kernel!` (Filters.jl:72-99). */
HT_API int ht_smooth_window(ht_ctx* ctx, const void* d_delta_k, void* d_out, int n,
                            double boxsize, double Rf, int wsmooth, void* stream);

/* The per-filter smoothing of a periodic n^3 box as the tile the peak scan reads:
 * window (as ht_smooth_window) into a context buffer, cuFFT inverse real FFT normalised by
 * 1/n^3 (Julia's irfft), and d_tile (n + 2 nbuff)^3 Float32 column-major = the box with
 * nbuff cells of periodic wrap on every side.  Replaces, for one filter, the copy +
 * window + irfft of ext/CUDAExt.jl:2985-2999 (Filters.smooth_field, Filters.jl:72-99). */
HT_API int ht_smooth_filter(ht_ctx* ctx, const void* d_delta_k, float* d_tile, int n,
                            int nbuff, double boxsize, double Rf, int wsmooth, void* stream);

/* The per-filter smoothing exactly as peak_find_tile_gpu performs it on a tile
 * (ext/CUDAExt.jl:2951-2989): d_delta_k is the rfft of the n^3 tile itself (the tile is
 * treated as periodic with side boxsize = n * alatt), d_out (n^3 Float32 column-major)
 * receives irfft(W . delta_k) normalised by 1/n^3.  The window (W/n^3, FP64, rounded to
 * FP32 once) is applied on the way into a context buffer; the inverse transform is one
 * out-of-place cuFFT C2R plan for power-of-two sides, and for other even sides three
 * batched 1-D cuFFT transforms along axes made contiguous by transposes (cuFFT's 3-D plan
 * is 3x slower there); n = 576 and 1152 transpose into pencils and run the pencil passes
 * (ht_smooth_pencil).  Plans cached per n; HT_TUNE_FFT_PATH overrides the choice. */
HT_API int ht_smooth_tile(ht_ctx* ctx, const void* d_delta_k, float* d_out, int n,
                          double boxsize, double Rf, int wsmooth, void* stream);

/* ht_smooth_tile that needs to deliver only the planes z_lo <= k < z_hi (0-based) of the
 * tile: the peak scan of one filter reads planes nbuff - 1 .. n - nbuff only.  The
 * transposed path skips the other planes in its y and x passes; other planes of d_out
 * may be left unwritten. */
HT_API int ht_smooth_tile_planes(ht_ctx* ctx, const void* d_delta_k, float* d_out, int n,
                                 double boxsize, double Rf, int wsmooth, int z_lo, int z_hi,
                                 void* stream);

/* Pencil form of the per-filter tile smoothing, for tile sides n = 576 and 1152
 * (ht_smooth_pencil_supported(n) != 0).  The rfft of the tile is the same for every
 * filter, so it is transposed once into pencils:
 *   ht_spectrum_pencil: d_pencil (complex64, (n, n/2+1, n) column-major) receives
 *     P[kz, kx, ky] = d_delta_k[kx, ky, kz] (d_delta_k as for ht_smooth_tile; out of
 *     place, any even n).
 *   ht_smooth_pencil: for one filter, the same irfft(W . delta_k) / n^3 as ht_smooth_tile,
 *     computed in three passes (window + FFT along kz, FFT along ky, half-length real FFT
 *     along kx), each reading whole contiguous columns; only the rows d_out[:, j, k] with
 *     lo <= j - 1, k - 1 < hi (1-based j, k) are written: the rows that the peak scan of the
 *     inner region [lo + 1, hi - 1) reads (lo = nbuff - 1, hi = n - nbuff + 1).
 * These replace the per-filter copy + window + irfft of ext/CUDAExt.jl:2951-2989 when the
 * spectrum is kept across filters (peak_find_tile_gpu's loop over filters). */
HT_API int ht_smooth_pencil_supported(int n);
HT_API int ht_spectrum_pencil(ht_ctx* ctx, const void* d_delta_k, void* d_pencil, int n,
                              void* stream);
HT_API int ht_smooth_pencil(ht_ctx* ctx, const void* d_pencil, float* d_out, int n,
                            double boxsize, double Rf, int wsmooth, int lo, int hi,
                            void* stream);

/* ------------------------------------------------------------ shell collapse ---- */

/* Tile fields (device, Float32 column-major n1*n2*n3).  eta2* may all be NULL (1LPT:
 * zeros), lapd may be NULL (ioutshear = 0: d2F = 0).  The transposed read
 * delta[k, i, j] of the reference gather requires a cubic tile. */
typedef struct {
    const float* delta;
    const float* etax;
    const float* etay;
    const float* etaz;
    const float* eta2x;
    const float* eta2y;
    const float* eta2z;
    const float* lapd;
    int32_t n1, n2, n3;
} ht_fields;

/* Bind a tile to the context and build its interleaved cell-record copy
 * (32 B per cell: delta, delta[k,i,j], eta xyz, eta2 xyz) in context-owned device
 * memory.  The caller's fields must stay valid until the next ht_fields_pack or
 * ht_ctx_destroy (PLAIN mode and lapd read them directly). */
HT_API int ht_fields_pack(ht_ctx* ctx, const ht_fields* fields, void* stream);

/* Peaks to analyse (device arrays of npeaks): 1-based i, j, k; filter radius Rf
 * (Mpc/h, Float64 as the reference's batch tuples carry it); ir2min = min(floor((1.75 Rf/alatt)^2), floor((40/alatt - 1)^2))
 * (MultiResolution.jl:575-576); ZZon = 1 + z and fcrit per peak (the broadcast or
 * lightcone values of ext/CUDAExt.jl:2215-2218). */
typedef struct {
    const int32_t* pi;
    const int32_t* pj;
    const int32_t* pk;
    const double* Rf;
    const int32_t* ir2min;
    const float* ZZon;
    const float* fcrit;
    int64_t npeaks;
    /* Nullable: the order in which to process the peaks, a permutation of 0..npeaks-1
     * (entries outside that range are skipped).  Results stay indexed by peak, so any
     * order gives identical results.  NULL: batch order (PLAIN), or a spatial order
     * computed by the library (BATCHED: Morton order of (i, j, k) within each lane-group
     * class, so that concurrently walked peaks share cells in L2). */
    const int32_t* order;
    /* Nullable: predicted cost per peak (the learned bracket's high quantile of the walk's
     * stop radius, ht_bracket_predict).  HT_MODE_LEARNED without a caller order processes
     * the peaks by descending cost within each lane-group class, so that the peaks sharing
     * a warp walk similar distances and the longest walks start first.  Ignored otherwise. */
    const float* cost;
} ht_peak_batch;

/* Per-peak outputs (device, Float32; vectors are (3, npeaks) and strain (3, 3, npeaks)
 * column-major), the 14 arrays of ext/CUDAExt.jl:2003-2016.  No-collapse peaks get
 * RTHL = zvir_half = -1 and zeros elsewhere. */
typedef struct {
    float* RTHL;
    float* Fbarx;
    float* e_v;
    float* p_v;
    float* strain;
    float* eigs;
    float* Srb;
    float* Sbar;
    float* Sbar2;
    float* gradpk;
    float* gradpkf;
    float* gradpkrf;
    float* d2F;
    float* zvir_half;
    /* Nullable diagnostics (no reference counterpart), Int32 per peak: the number of
     * shells the gather walked (the exact early-exit point), and the shell mp* whose
     * barrier crossing set RTHL (0 for no collapse). */
    int32_t* walk_shells;
    int32_t* collapse_shell;
} ht_results;

/* Radial-shell collapse of every peak of `batch` on the bound tile.  alatt in Mpc/h;
 * rmax2rs > 0 limits shells to r <= rmax2rs*Rf/alatt (ext/CUDAExt.jl:2192-2200);
 * d_mask (nullable, n^3 Int8) gets 1 on core cells within RTHL.  conv: HT_CONV_*;
 * mode: HT_MODE_*.  Results are identical for every mode. */
HT_API int ht_shell_analyse(ht_ctx* ctx, const ht_peak_batch* batch, double alatt,
                     double rmax2rs, int32_t nbuff, int8_t* d_mask, int32_t conv,
                     int32_t mode, const ht_results* out, void* stream);

/* Allocation-free variant of ht_shell_analyse.  No counterpart in the reference.
 *
 * For callers that cannot call cudaMalloc while they run this step: code issuing work
 * into a stream that is being captured into a CUDA graph (allocation is not a capturable
 * operation), or hosts whose device memory belongs to a pool they manage themselves.
 * The call allocates nothing: the shell walk's per-warp scratch is a 32 MiB file-scope
 * __device__ array inside the library (held by every GPU that loads the library until
 * the process exits), and the fields are read in place (no interleaved-record copy, no
 * ht_fields_pack needed).  The caller passes the tile, the peaks and the result arrays;
 * `ctx` (created beforehand) supplies the shell and collapse tables.  Results equal
 * ht_shell_analyse's.
 *
 * - The first call on a device resolves the array's device address
 *   (cudaGetSymbolAddress) with that device current and keeps it for the life of the
 *   process; make that first call before any stream capture begins, and do not use the
 *   library across a cudaDeviceReset of that device (the kept address would be stale).
 * - All calls share the one array: calls whose kernels overlap on the GPU (e.g. on two
 *   streams, or from two threads) race on it and give wrong results.  Serialize them.
 * - Limit: one 8-warp block's scratch, 8 warps * 4 peak slots * (nshells + 2) * 128 bytes,
 *   must fit within 32 MiB, i.e. nshells <= 8190 (nhunt up to about 98); larger hunt
 *   radii return HT_ERR_CAPACITY.  Larger hunt radii run fewer concurrent warps. */
HT_API int ht_shell_analyse_static(ht_ctx* ctx, const ht_fields* fields,
                                   const ht_peak_batch* batch, double alatt, double rmax2rs,
                                   int32_t nbuff, int8_t* d_mask, int32_t conv,
                                   const ht_results* out, void* stream);

/* Result-neutral tunables of a context, for an autotuner (no counterpart in the
 * reference).  None of them changes any output: they only change launch shapes and the
 * processing order.
 *   HT_TUNE_BLOCK_BITS  HT_MODE_LEARNED order: peaks are grouped into spatial blocks of
 *                       2^value cells (Morton prefix) and ordered by descending predicted
 *                       cost inside a block (default 17);
 *   HT_TUNE_PF_KZ       peak scan: k-planes per CTA (0 = chosen from the grid size);
 *   HT_TUNE_WALK_BPSM   shell walk: resident blocks per SM (0 = the occupancy maximum);
 *   HT_TUNE_FFT_PATH    ht_smooth_tile's inverse FFT: 0 = by tile side (the pencil passes
 *                       at 576 and 1152, one 3-D cuFFT plan for powers of two, otherwise
 *                       transposes + batched 1-D transforms), 1 = 3-D plan, 2 = transposed
 *                       1-D (even sides), 3 = fused (sides 576 and 1152), 4 = pencil (sides
 *                       576 and 1152).  They differ by FP32 round-off, so keep one choice per
 *                       run for reproducible peaks. */
#define HT_TUNE_BLOCK_BITS 1
#define HT_TUNE_PF_KZ 2
#define HT_TUNE_WALK_BPSM 3
#define HT_TUNE_FFT_PATH 4
/* Two more keys set the bounded in-kernel waits (the TMA pipelines of the peak scan and of
 * the pencil smoothing), which give up instead of hanging and report through
 * ht_device_status:
 *   HT_TUNE_WAIT_NS     the limit of every wait, in ns of %globaltimer (1e3 .. 6e10;
 *                       default 2e9);
 *   HT_TUNE_INJECT_TX   test hook (default 0): every peak-scan CTA announces this many bytes
 *                       (a multiple of 16, at most 4096) beyond its first copy, so its first
 *                       wait runs out although the copy itself completes; the scan then
 *                       records status 1, drains its copies and returns, and its peaks are
 *                       invalid.  Nothing faults or hangs; set it back to 0 to scan again. */
#define HT_TUNE_WAIT_NS 5
#define HT_TUNE_INJECT_TX 6
HT_API int ht_ctx_tune(ht_ctx* ctx, int32_t key, int64_t value);

/* ------------------------------------------------ lightcone and halo records ---- */

/* Cosmology tables of a run, built once on the host and copied into the context:
 * the chi -> z table of build_chi_to_z (src/Cosmology/Cosmology.jl:334-347; chi ascending,
 * Mpc/h) and the linear-growth tables of Dlinear_tables (Cosmology.jl:159-283). */
typedef struct {
    const double* chi;        /* comoving distance [n_chi], ascending */
    const double* zchi;       /* redshift of each entry [n_chi] */
    int32_t n_chi;
    double z_max;             /* chi_to_z's clamp (the table's z_max) */
    const double* atab;       /* scale factors [ntab], ascending */
    const double* D_atab;     /* D(a)/a [ntab] */
    const double* dlnD_dlna;  /* [ntab] */
    int32_t ntab;
    double amintab, amaxtab, D_ainfty, D_a0, HD_Hainfty, HD_Ha0;
    double Om, OL;            /* omega_m_a of the 2LPT coefficient (MultiResolution.jl:734) */
} ht_cosmo;

/* Copy the tables (host arrays) into the context; required before the two calls below. */
HT_API int ht_ctx_set_cosmo(ht_ctx* ctx, const ht_cosmo* cosmo);

/* Geometry of a tile: side n (cells, buffer included), centre (Mpc/h), cell size. */
typedef struct {
    int32_t n;
    double xbx, ybx, zbx;
    double alatt;
} ht_tile_geom;

/* Per-peak lightcone state before the shell collapse (MultiResolution.jl:1097-1130):
 * position x = xbx + alatt (i - (n+1)/2) (ext/CUDAExt.jl:3039-3046, FP64), z = chi_to_z(
 * |x - obs|) (Cosmology.jl:354-385), ZZon = Float32(1 + z), fcrit = Float32(fsc_of_z(z))
 * (RadialShell.jl:181-195).  Peaks with z <= z_max are kept: their 0-based indices, in
 * order, go to d_keep and their number to *d_nkeep (device Int64).  d_i/d_j/d_k are the
 * peak scan's 1-based cells; d_z may be NULL. */
HT_API int ht_peak_lightcone(ht_ctx* ctx, const int32_t* d_i, const int32_t* d_j,
                             const int32_t* d_k, int64_t npeaks, const ht_tile_geom* geom,
                             const double* obs, double z_max, double* d_z, float* d_ZZon,
                             float* d_fcrit, int32_t* d_keep, int64_t* d_nkeep,
                             void* stream);

/* The peaks of one collapse call, as packing reads them (device arrays). */
typedef struct {
    const int32_t* i;
    const int32_t* j;
    const int32_t* k;
    const double* Rf;         /* filter radius (Mpc/h) */
    const float* FcRf;        /* delta_s at the peak (PeakCandidate.delta) */
    const float* d2Rf;        /* lapd_s at the peak; NULL: zeros */
    const double* z;          /* per-peak redshift (lightcone); NULL: one ZZon for all */
    int64_t npeaks;
} ht_catalog_peaks;

/* Halo records of the collapsed peaks (RTHL > 0, and z <= z_max on a lightcone), in peak
 * order (MultiResolution.jl:1159-1219): HaloRecord rows of 11 Float32 when ioutshear == 0,
 * ExtHaloRecord rows of 33 otherwise (src/IO/Catalog.jl:4-48): position, Sbar D(a),
 * RTHL alatt, Sbar2 (-3/7) Om(a)^(-1/143) D(a)^2 (ilpt >= 2, else 0), Fbarx, and for the
 * extended rows e_v, p_v, strain (11,22,33,23,13,12), d2F, zvir_half, gradpk, gradpkf, Rf,
 * FcRf, d2Rf, gradpkrf.  D(a) = Dlinear_ab(1 / (1 + z)) (Cosmology.jl:286-306).  At most
 * `cap` rows are written; *d_nhalo (device Int64) receives the number of halos. */
HT_API int ht_pack_halos(ht_ctx* ctx, const ht_catalog_peaks* peaks, const ht_results* res,
                         const ht_tile_geom* geom, double ZZon, double z_max, int32_t ilpt,
                         int32_t ioutshear, float* d_records, int64_t cap, int64_t* d_nhalo,
                         void* stream);

/* Lagrangian exclusion of a halo catalog (src/Merger/Merger.jl:38-104 merge_catalog,
 * src/Merger/Exclusion.jl:99-140): halos in decreasing radius (ties by x, y, z, then input
 * order); a surviving halo removes every later halo whose centre lies inside its radius.
 * With volume_reduction, overlapping survivors then shrink by their cap volumes
 * (Exclusion.jl:152-206; fortran_ties counts an equal-radius pair twice), and halos left
 * with no volume are removed.  d_records: nhalo rows of `width` (11 or 33) Float32 in the
 * Catalog layout (x, y, z at 0-2, RTHL at 6).  d_out receives the survivors in input order
 * with their (possibly reduced) RTHL, at most nhalo rows; *d_nout (device Int64) their
 * number.  Deterministic except the last bits of reduced radii (the cap volumes are summed
 * with atomics). */
HT_API int ht_merge_halos(ht_ctx* ctx, const float* d_records, int64_t nhalo, int32_t width,
                          int32_t volume_reduction, int32_t fortran_ties, float* d_out,
                          int64_t* d_nout, void* stream);

/* Eulerian positions and peculiar velocities of a merged raw catalog, in place
 * (Merger.jl:114-146 finalize_eulerian): x = q + d1 + d2, v = a 100 E(a) f(a) (d1 + 2 d2)
 * km/s with f = dlnD/dlna from the context's growth tables, the 2LPT fields zeroed; a from
 * the chi -> z table at the Eulerian distance to obs (ievol = 1) or 1 / (1 + z_out).
 * Requires ht_ctx_set_cosmo. */
HT_API int ht_finalize_eulerian(ht_ctx* ctx, float* d_records, int64_t nhalo, int32_t width,
                                const double* obs, int32_t ievol, double z_out, void* stream);

/* ------------------------------------------------------ learned walk bracket ---- */

/* A 12 -> 64 -> 64 -> 64 -> 2 MLP predicting the 10 % and 90 % quantiles of the radius at
 * which a peak's shell walk stops, used only to order the collapse work (HT_MODE_LEARNED);
 * results never depend on it.  No counterpart in the reference.  Device arrays: BF16
 * weights (raw 16-bit), row-major [out][in]: W1 64x16 (inputs 12..15 are padding), W2 and
 * W3 64x64, W4 8x64 (rows 2..7 zero); FP32 biases b1..b3 [64], b4 [8]; FP32 feature
 * standardisation mean / istd [16]. */
typedef struct {
    uint16_t* W1;
    uint16_t* W2;
    uint16_t* W3;
    uint16_t* W4;
    float* b1;
    float* b2;
    float* b3;
    float* b4;
    float* mean;
    float* istd;
} ht_bracket_model;

/* Number of FP32 parameters in the packed layout of ht_bracket_grad / ht_bracket_adam:
 * W1 [64x16] W2 [64x64] W3 [64x64] W4 [8x64] b1 b2 b3 [64] b4 [8]. */
#define HT_BRACKET_NPARAMS 9928

/* Features [npeaks x 16] FP32 of the batch on the bound tile (ht_fields_pack first):
 * Rf/alatt, sqrt(ir2min), delta_s at the peak (d_peak_delta, nullable), fcrit, ZZon,
 * delta at the peak cell, mean delta on shells 2..5, rad[m0_init], Rf/alatt + 2, zeros. */
HT_API int ht_bracket_features(ht_ctx* ctx, const ht_peak_batch* batch,
                               const float* d_peak_delta, double alatt, float* d_feat,
                               void* stream);

/* Inference: d_pred [n x 2] FP32 (low, high quantile of the stop radius, lattice units)
 * from d_feat [n x 16] (16-byte aligned).  5th-generation tensor cores (tcgen05.mma, BF16
 * operands in shared memory, FP32 accumulators in tensor memory); a bounded wait that gives
 * up sets ht_device_status to 1. */
HT_API int ht_bracket_predict(ht_ctx* ctx, const ht_bracket_model* model, const float* d_feat,
                              int64_t n, float* d_pred, void* stream);

/* Training: pinball-loss gradient (quantiles 0.1 and 0.9 of d_target) over n rows,
 * written to d_grads [HT_BRACKET_NPARAMS] in the packed layout; the mean loss to *d_loss. */
HT_API int ht_bracket_grad(ht_ctx* ctx, const ht_bracket_model* model, const float* d_feat,
                           const float* d_target, int64_t n, float* d_grads, float* d_loss,
                           void* stream);

/* One Adam step (beta 0.9 / 0.999, eps 1e-8) on packed FP32 master parameters, then the
 * BF16 weights and FP32 biases of `model` are rewritten from them. */
HT_API int ht_bracket_adam(ht_ctx* ctx, float* d_params, const float* d_grads, float* d_m,
                           float* d_v, int32_t step, float lr, const ht_bracket_model* model,
                           void* stream);

/* Launch statistics of the last ht_shell_analyse on this context: kernels launched and
 * the total number of shells walked (for the roofline's algorithmic bytes). */
HT_API int ht_last_launch_stats(const ht_ctx* ctx, int64_t* kernels, int64_t* shells_walked,
                         int64_t* cells_walked);

/* Reject-reason counters of the shell collapse: why a peak ended without collapse, the
 * counters of RadialShell.jl:13-32 (bumped at RadialShell.jl:310,517,604,684,698) kept per
 * context on the device.  Every ht_shell_analyse and ht_shell_analyse_static call adds to
 * them (one count per rejected peak) until ht_reset_reject_counts, as the reference's
 * atomics accumulate until reset_dump_counters!.
 *   HT_REJECT_PREMASK      masked by a larger halo before the walk (HT_CONV_CPU with
 *                          rmax2rs > 0 only, which the device path rejects: stays 0)
 *   HT_REJECT_NO_FCRIT     no shell with Fbar >= fcrit inward of the start (:517)
 *   HT_REJECT_M0_ONE       the crossing is the centre shell (:604)
 *   HT_REJECT_NO_COLLAPSE  no shell reaches zvir >= ZZon (:684); also a hunt radius that
 *                          holds fewer than two shells
 *   HT_REJECT_RTHL_NEG     the interpolated radius is not positive (:698)
 *   HT_REJECT_OUTSIDE      the peak's centre lies outside the bound tile (no reference
 *                          counterpart: the reference would index out of bounds) */
#define HT_REJECT_PREMASK 0
#define HT_REJECT_NO_FCRIT 1
#define HT_REJECT_M0_ONE 2
#define HT_REJECT_NO_COLLAPSE 3
#define HT_REJECT_RTHL_NEG 4
#define HT_REJECT_OUTSIDE 5
#define HT_REJECT_COUNT 6

/* counts[HT_REJECT_COUNT]: the counters (get_dump_counts, RadialShell.jl:28-32), after the
 * context's work so far has finished (synchronises the device). */
HT_API int ht_reject_counts(const ht_ctx* ctx, int64_t* counts);
/* Zeroes the counters (reset_dump_counters!, RadialShell.jl:19-26), stream-ordered after
 * the work already issued on `stream` (NULL: the legacy default stream). */
HT_API int ht_reset_reject_counts(ht_ctx* ctx, void* stream);

/* Measurement aid (no reference counterpart): gathers the packed cell records of the bound
 * tile (ht_fields_pack) at n_idx caller-given cell indices (0-based linear, each < n^3),
 * with the 256-bit record load the shell walk uses, and writes the sum of each record's
 * eight values to d_out[i].  With uniformly random indices it measures the rate of
 * scattered 32-byte gathers without any reuse between them: the memory ceiling of a walk
 * that found none of its cells in a cache, to set beside the streaming copy bandwidth.
 * An index outside the tile reads nothing and gives NaN. */
HT_API int ht_record_gather_probe(ht_ctx* ctx, const int64_t* d_idx, int64_t n_idx,
                                  float* d_out, void* stream);

/* Device status of the context since the last call (no reference counterpart: the
 * reference kernels have no waits).  Synchronises the device, then returns 0 in *status
 * when every bounded wait of this context's kernels completed, or 1 when a pipeline wait
 * of the peak scan or of the pencil smoothing gave up (after HT_TUNE_WAIT_NS, 2 s by
 * default: that filter's output is then incomplete), or 2 when a build with -DHT_CHECKED
 * (libhuntian_b200_checked.so) found a data-dependent index outside its array and skipped
 * the access; the word is cleared on read. */
HT_API int ht_device_status(ht_ctx* ctx, int32_t* status);

/* ---------------------------------------------------- collapse-table generation ---- */

/* EllipsoidParams (src/EllipsoidalCollapse/EllipsoidalCollapse.jl:10-45) with its
 * cosmology's Om and OL; the defaults there are iforce_strat 4, ivir_strat 2, fcoll
 * (0.01, 0.171, 0.171), tfac 0.01, nstepmax 10000, zinit_fac 20, solver :diffeq.
 * solver: HT_SOLVER_RK4, the fixed-step RK4 of the Fortran code (tfac, nstepmax; events
 * 1-6), or HT_SOLVER_TSIT5, the :diffeq path (EllipsoidalCollapse.jl:440-485): Tsit5 with
 * abstol 1e-8, reltol 1e-6, at most 100,000 iterations, stopping once axis 1 has
 * virialised (events 1-3; tfac and nstepmax unused). */
#define HT_SOLVER_RK4 0
#define HT_SOLVER_TSIT5 1
typedef struct {
    double Om, OL;
    int32_t iforce_strat;     /* 0, 1, 3, 4, 5 or 6 (2 leaves the velocities constant) */
    int32_t ivir_strat;       /* 1 or 2 */
    double fcoll[3];          /* fcoll_1, fcoll_2, fcoll_3 */
    double tfac;              /* RK4 step factor */
    int32_t nstepmax;         /* step limit, 1 .. 10^8 */
    double zinit_fac;         /* initial 1/a = zinit_fac Frho */
    int32_t solver;           /* HT_SOLVER_RK4 or HT_SOLVER_TSIT5 */
} ht_ellipsoid;

/* DlinearTables (src/Cosmology/Cosmology.jl:68-78), HOST arrays of ntab >= 4 entries, atab
 * ascending (as Dlinear_tables builds it). */
typedef struct {
    const double* atab;
    const double* D_atab;        /* D(a) / a */
    const double* dlnD_dlnatab;
    int32_t ntab;
    double amintab, amaxtab, D_ainfty, D_a0, HD_Hainfty, HD_Ha0;
} ht_growth;

/* evolve_ellipse_full (EllipsoidalCollapse.jl:492-590) with ep->solver for n ellipsoids
 * (DEVICE arrays Frho, e_v, p_v), event idynax (1-3 axis virialisation, 4-6 turnaround,
 * RK4 only): d_zvir = 1/a at the event, d_D = D(a) there, d_fc = Frho D, all -1 when the
 * event does not happen before a = 2 (or nstepmax RK4 steps).  d_D, d_fc and d_steps
 * (steps taken; with Tsit5 accepted and rejected) may be NULL.  One device thread per ellipsoid, FP64.  Asynchronous on `stream`
 * (the growth table is staged to the device in stream order; the host arrays may be
 * released when the call returns). */
HT_API int ht_evolve_ellipses(int device, const ht_ellipsoid* ep, const ht_growth* growth,
                              int64_t n, const double* d_Frho, const double* d_e_v,
                              const double* d_p_v, int32_t idynax, double* d_zvir,
                              double* d_D, double* d_fc, int32_t* d_steps, void* stream);

/* make_table (CollapseTable.jl:29-50): table[i, j, k] = Float32(zvir) of the ellipsoid
 * Frho = 10^x_i, e_v = y_j, p_v = z_k y_j on the regular axes x_i = X1 + (i - 1)(X2 - X1) /
 * (nx - 1) and so on (event 1, axis-1 virialisation), written column-major (i fastest)
 * into the HOST array table[nx ny nz].  Synchronous. */
HT_API int ht_collapse_table(int device, const ht_ellipsoid* ep, const ht_growth* growth,
                             int32_t nx, int32_t ny, int32_t nz, double X1, double X2,
                             double Y1, double Y2, double Z1, double Z2, float* table);

#ifdef __cplusplus
}
#endif
#endif
