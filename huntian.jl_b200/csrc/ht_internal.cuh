// Internal declarations shared by the huntian_b200 CUDA sources.
#pragma once

#ifndef HT_NO_NVTX
#include <nvtx3/nvToolsExt.h>
#endif
#include <cuda_runtime.h>
#include <cufft.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "huntian_b200.h"

// ------------------------------------------------------------------ context ----

struct ht_ctx {
    int device = 0;
    int num_sms = 0;
    int nhunt = 0;

    // Shell table (ShellAnalysisGPU.jl:28-71), 1-based by shell index m = 1..nshells:
    // shell m holds cells [start[m], start[m] + count[m]) of the r^2-sorted cell list.
    int32_t nshells = 0;
    int64_t ncells = 0;
    std::vector<int32_t> h_r2, h_start, h_count;
    std::vector<char4> h_off;
    char4* d_off = nullptr;        // (di, dj, dk, 0) per cell, r^2-sorted
    int32_t* d_start = nullptr;    // [nshells + 2]
    int32_t* d_count = nullptr;    // [nshells + 2]
    int32_t* d_r2 = nullptr;       // [nshells + 2]
    double* d_rad = nullptr;       // sqrt(r2), [nshells + 2]
    double* d_irad = nullptr;      // 1 / rad (0 at the centre), [nshells + 2]
    double* d_irad3 = nullptr;     // 1 / rad^3, [nshells + 2]
    int2* d_cell = nullptr;        // (linear offset in the bound tile, char4 bits) per cell
    int cell_n1 = 0, cell_n2 = 0;  // tile dims d_cell was built for (0: none)
    // SPH window weights of kernel_strain (RadialShell.jl:225-274), which depend only on
    // the two shell radii: row mp holds entries [wrow[mp], wrow[mp+1]) of (m1, weight)
    int64_t nweights = 0;
    int32_t* d_wrow = nullptr;     // [nshells + 2]
    double2* d_wpk = nullptr;      // per entry: (weight, m1 as a double), one 16-byte load
    // result-neutral tunables (ht_ctx_tune)
    int tune_block_bits = 17;      // LEARNED order: spatial block of 2^bits cells
    int tune_pf_kz = 0;            // peak scan: planes per CTA (0: by grid size)
    int tune_walk_bpsm = 0;        // walk: blocks per SM (0: occupancy maximum)
    int tune_fft_path = 0;         // tile smoothing: 0 auto, 1 3-D plan, 2 transposed 1-D,
                                   // 3 fused three-pass, 4 pencil (n = 576, 1152)
    long long wait_ns = 2000000000LL;  // limit of every bounded in-kernel wait
    unsigned inject_tx = 0;        // test hook: bytes announced beyond the first copy of
                                   // every peak-scan CTA (its wait then runs out)

    // collapse table + SPH table
    std::vector<float> h_ct;
    float* d_ct = nullptr;
    int nx = 0, ny = 0, nz = 0;
    double X1 = 0, X2 = 0, Y1 = 0, Y2 = 0, Z1 = 0, Z2 = 0, out_val = -1.0;
    double* d_akk = nullptr;       // 1101 entries

    // bound tile
    bool bound = false;
    ht_fields fields{};
    float4* d_rec = nullptr;       // 2 float4 per cell
    size_t rec_cells = 0;

    // workspaces
    void* d_pf_ws = nullptr;       // peak-find bitmap + segment counts
    size_t pf_ws_bytes = 0;
    double* d_scratch = nullptr;   // shell-walk per-warp profiles
    size_t scratch_bytes = 0;
    void* d_win = nullptr;         // smoothing-window table
    size_t win_bytes = 0;
    void* d_cwork = nullptr;       // complex buffer of the per-filter smoothing
    size_t cwork_bytes = 0;
    cufftHandle fft_plan = 0;      // in-place C2R plan for fft_n^3 (0 = none)
    int fft_n = 0;
    cufftHandle tile_plan = 0;     // out-of-place C2R plan, unpadded output, tile_n^3
    int tile_n = 0;
    void* d_cwork2 = nullptr;      // second complex buffer of the transposed path
    size_t cwork2_bytes = 0;
    cufftHandle tp_plan_n = 0;     // transposed path: 1-D C2C of length tp_n, all rows
    int tp_n = 0;
    cufftHandle tp_plan_y = 0;     // length tp_zc_n along y for tp_zc planes
    cufftHandle tp_plan_x = 0;     // length tp_zc_n / 2 along x for tp_zc planes
    int tp_zc = 0, tp_zc_n = 0;
    void* d_tw = nullptr;          // e^{2 pi i k / n}, k < n / 2
    size_t tw_bytes = 0;
    void* d_ftw = nullptr;         // fused-path twiddles for side fz_n
    size_t ftw_bytes = 0;
    int fz_n = 0;
    // pencil Z pass window rows: the distinct kx^2 + ky^2 of side wb_n (wb_count of them)
    // followed by the row index of every (kx, ky); d_wu holds one row of the window along
    // kz per distinct value, rebuilt for every filter
    void* d_wb = nullptr;
    size_t wb_bytes = 0;
    int wb_n = 0, wb_count = 0;
    void* d_wu = nullptr;
    size_t wu_bytes = 0;
    void* d_order_ws = nullptr;    // BATCHED peak-order keys, indices and sort temp
    size_t order_ws_bytes = 0;
    void* d_mlp_ws = nullptr;      // bracket training activations
    size_t mlp_ws_bytes = 0;
    // lightcone and halo-record tables (ht_ctx_set_cosmo) and their workspace
    bool cosmo_set = false;
    double* d_chi = nullptr;       // chi -> z table
    double* d_zchi = nullptr;
    int n_chi = 0;
    double cosmo_zmax = 0.0;
    double* d_atab = nullptr;      // linear-growth tables
    double* d_Da = nullptr;
    double* d_dlnD = nullptr;
    int ntab = 0;
    double amintab = 0.0, amaxtab = 0.0, D_ainfty = 0.0, D_a0 = 0.0;
    double HD_Hainfty = 0.0, HD_Ha0 = 0.0, cosmo_Om = 0.0, cosmo_OL = 0.0;
    void* d_cat_ws = nullptr;      // flags, indices and CUB temp of the catalog kernels
    size_t cat_ws_bytes = 0;
    void* d_merge_ws = nullptr;    // halo merging: per-halo arrays and CUB temp
    size_t merge_ws_bytes = 0;
    void* d_merge_cells = nullptr; // halo merging: cell counts and starts
    size_t merge_cells_bytes = 0;
    void* d_merge_scan = nullptr;  // halo merging: scan temp of large cell tables
    size_t merge_scan_bytes = 0;
    int32_t* d_queue = nullptr;    // dynamic work counter
    unsigned long long* d_stats = nullptr;  // [0] cells walked, [1] shells walked,
                                            // [8] (int32) device status word,
                                            // [16, 16 + HT_REJECT_COUNT) reject counters

    int64_t last_kernels = 0;
};

// Device status word: kernels with bounded waits store a non-zero code here when a wait
// gives up, instead of trapping; ht_device_status reads and clears it.
inline int32_t* ht_status_word(ht_ctx* ctx) { return (int32_t*)(ctx->d_stats + 8); }

// Status codes in the device status word (ht_device_status).
constexpr int32_t kStatusWaitTimeout = 1;   // a bounded wait gave up
constexpr int32_t kStatusBounds = 2;        // an HT_CHECKED index check failed

// HT_CHECKED builds: an index check before a data-dependent access.  A failed check
// records kStatusBounds in the status word and evaluates to false, so that the caller
// skips the access (no trap); other builds compile the check away.
#ifdef HT_CHECKED
__device__ __forceinline__ bool ht_index_ok(int32_t* status, long long i, long long n) {
    if (i >= 0 && i < n) return true;
    if (status) atomicExch(status, kStatusBounds);
    return false;
}
#define HT_INDEX_OK(status, i, n) ht_index_ok((status), (long long)(i), (long long)(n))
#else
#define HT_INDEX_OK(status, i, n) true
#endif

// Reject-reason counters (HT_REJECT_*), accumulated by the shell walk until reset.
inline unsigned long long* ht_reject_words(ht_ctx* ctx) { return ctx->d_stats + 16; }

// NVTX range around a C-ABI entry point: each call shows as a named range on the host
// timeline of a profiler that records NVTX (Nsight Systems; Nsight Compute with --nvtx).
// nvtx3 is header-only and its calls do nothing unless a profiler has attached.  Built
// with -DHT_NO_NVTX the ranges compile away.
#ifndef HT_NO_NVTX
struct HtRange {
    explicit HtRange(const char* name) { nvtxRangePushA(name); }
    ~HtRange() { nvtxRangePop(); }
    HtRange(const HtRange&) = delete;
    HtRange& operator=(const HtRange&) = delete;
};
#define HT_RANGE(name) HtRange ht_nvtx_range_(name)
#else
#define HT_RANGE(name) ((void)0)
#endif

// ----------------------------------------------------------------- errors ----

int ht_fail(int code, const std::string& msg);
int ht_cuda_fail(cudaError_t e, const char* what);
bool ht_fault_injected(const char* site);   // HT_FAULT_INJECT=<site>[,<site>...]
int ht_alloc(void** p, size_t bytes, const char* what);
int ht_grow(void** p, size_t* have, size_t need, const char* what);

#define HT_CUDA_TRY(call, what)                                   \
    do {                                                          \
        cudaError_t _e = (call);                                  \
        if (_e != cudaSuccess) return ht_cuda_fail(_e, what);     \
    } while (0)

// ------------------------------------------------------- kernel launchers ----

int ht_launch_pack(ht_ctx* ctx, cudaStream_t st);
int ht_launch_peakfind(ht_ctx* ctx, const float* d_delta_s, const float* d_lapd_s,
                       int8_t* d_mask, int n, int nbuff, float fcrit, int32_t filter_idx,
                       int64_t max_peaks, const ht_peaks* out, cudaStream_t st);
int ht_launch_walk(ht_ctx* ctx, const ht_peak_batch* b, double alatt, double rmax2rs,
                   int32_t nbuff, int8_t* d_mask, int32_t conv, int32_t mode,
                   const ht_results* out, cudaStream_t st);
