// Peak finding on one smoothed field (PeakFind.jl:15-78 semantics) on sm_100a.
//
// Four launches per filter, all deterministic:
//   1. flag  : 26-neighbour local-maximum test of every inner cell.  On the main
//              path a CTA owns a 32 (i) x 32 (j) column block and streams kz planes in
//              k: the planes (40 x 34 floats with the one-cell halo, the x origin
//              rounded down to 16 bytes) arrive by TMA (cp.async.bulk.tensor) into an
//              8-slot shared-memory ring tracked by mbarriers, so up to 8 planes per CTA
//              are in flight instead of one DRAM round trip per plane.  Each thread owns
//              4 cells of a column, folds their 3 x 3 maxima of every plane into
//              registers once (separably) and keeps the last three planes' maxima, so a
//              slot is free as soon as all warps have read it.  The int8 mask is read only for cells that pass
//              the height and neighbour tests (the conditions are a plain AND).  Grids
//              whose row pitch is not a multiple of 16 bytes (n % 4 != 0) or that are
//              narrower than the box run the same test from plain loads through a
//              3-plane ring.  Survivors are compacted into a bitmap with one
//              __ballot_sync word per (k, j, 32-cell run of i), laid out in the CPU
//              scan order k -> j -> i.
//   2. count : popcount of each segment of kSegWords bitmap words.
//   3. scan  : one CTA turns the segment counts into absolute output slots after the
//              peaks of earlier filters and advances the running count.
//   4. emit  : each segment re-reads its words, ranks its set bits in scan order and
//              writes (i, j, k, delta_s, lapd_s, filter) plus mask = 1 for every slot
//              below max_peaks.
// Result: the same peak list, in the same order, as the CPU scan, independent of
// thread timing (the reference GPU kernel reserves slots with an atomic counter and is
// order-nondeterministic, ext/CUDAExt.jl:2921).
#include <cuda.h>
#include <cudaTypedefs.h>

#include <mutex>

#include "ht_async.cuh"
#include "ht_internal.cuh"

namespace {

constexpr int kTX = 32, kTY = 8, kKZ = 32;
constexpr int kSegWords = 2048;
constexpr int kEmitThreads = 256;
constexpr int kWordsPerThread = kSegWords / kEmitThreads;

struct PfGeom {
    int n, nbuff, inner, wpr;   // words per row = ceil(inner/32)
    long long nwords;           // inner * inner * wpr
};

__global__ void __launch_bounds__(kTX * kTY) pf_flag_kernel(const float* __restrict__ ds,
                                                            const int8_t* __restrict__ mask,
                                                            PfGeom g, float fcrit,
                                                            uint32_t* __restrict__ bits) {
    __shared__ float plane[3][kTY + 2][kTX + 2];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int ib = g.nbuff + blockIdx.x * kTX;   // 0-based first i of the block
    const int jb = g.nbuff + blockIdx.y * kTY;
    const int kb = g.nbuff + blockIdx.z * kKZ;
    const int hi = g.n - g.nbuff;                // exclusive end of the inner range
    const int i = ib + tx, j = jb + ty;
    const bool active = i < hi && j < hi;
    const long long n = g.n, nn = n * n;
    const int kend = min(kb + kKZ, hi);

    auto load_plane = [&](int slot, int k) {
        // (kTY+2) x (kTX+2) values with a one-cell halo; clamped to the grid (the halo
        // of inner cells is always inside because nbuff >= 1)
        for (int e = ty * kTX + tx; e < (kTY + 2) * (kTX + 2); e += kTX * kTY) {
            const int r = e / (kTX + 2), c = e % (kTX + 2);
            int ii = ib - 1 + c, jj = jb - 1 + r;
            ii = min(max(ii, 0), g.n - 1);
            jj = min(max(jj, 0), g.n - 1);
            plane[slot][r][c] = __ldg(ds + (long long)ii + n * jj + nn * k);
        }
    };
    auto max9 = [&](int slot) {
        float m = plane[slot][ty][tx];
#pragma unroll
        for (int dj = 0; dj < 3; ++dj)
#pragma unroll
            for (int di = 0; di < 3; ++di) m = fmaxf(m, plane[slot][ty + dj][tx + di]);
        return m;
    };

    load_plane(0, kb - 1);
    load_plane(1, kb);
    __syncthreads();
    float mprev = max9(0);
    float mcur = max9(1);
    float ff = plane[1][ty + 1][tx + 1];
    for (int k = kb; k < kend; ++k) {
        const int slot_next = (k - kb + 2) % 3;
        __syncthreads();   // the slot being overwritten was last read two planes ago
        load_plane(slot_next, k + 1);
        __syncthreads();
        const float mnext = max9(slot_next);
        bool peak = false;
        if (active) {
            const long long c = (long long)i + n * j + nn * k;
            // mask == 1 skips; ff < fcrit skips; any neighbour > ff rejects (ties pass).
            // fmaxf ignores NaN neighbours, matching `ff < NaN == false`.
            const float m27 = fmaxf(fmaxf(mprev, mcur), mnext);
            peak = (__ldg(mask + c) != 1) && !(ff < fcrit) && !(ff < m27);
        }
        const unsigned w = __ballot_sync(0xffffffffu, peak);
        if (tx == 0 && j < hi) {
            const long long row = (long long)(k - g.nbuff) * g.inner + (j - g.nbuff);
            bits[row * g.wpr + blockIdx.x] = w;
        }
        mprev = mcur;
        mcur = mnext;
        ff = plane[slot_next][ty + 1][tx + 1];
    }
}


// ------------------------------------------------------------- TMA flag path ----

constexpr int kBoxX = 40;                  // plane box width in floats (160 B)
constexpr int kRowsPT = 4;                 // rows of j per thread
constexpr int kTYB = kTY * kRowsPT;        // 32 rows of j per CTA
constexpr int kBoxY = kTYB + 2;            // 34 rows: j - 1 .. j + 32
constexpr int kPPS = 2;                    // k-planes per TMA stage (box depth)
constexpr int kStages = 4;                 // stages in flight per CTA (8 planes)
constexpr int kPlaneFloats = kBoxX * kBoxY;                // 1360
constexpr int kPlaneBytes = kPlaneFloats * 4 * kPPS;       // bytes of one stage's copy
constexpr int kSlotFloats = 2720;          // 10880 B per stage: 128-byte aligned slots
static_assert(kPlaneFloats * kPPS <= kSlotFloats && (kSlotFloats * 4) % 128 == 0, "slot size");

using htasync::bar_wait;
using htasync::smem_addr;

// `extra` bytes are announced on top of the copy's own (0 except under the test hook
// that makes the stage's bounded wait run out: the copy lands, the phase never completes).
__device__ __forceinline__ void tma_plane(float* dst, const CUtensorMap* tm, int x, int y,
                                          int z, unsigned long long* bar, unsigned extra = 0) {
    const unsigned b = smem_addr(bar);
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
                 :: "r"(b), "r"(kPlaneBytes + extra) : "memory");
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
        "[%0], [%1, {%2, %3, %4}], [%5];"
        :: "r"(smem_addr(dst)), "l"(tm), "r"(x), "r"(y), "r"(z), "r"(b) : "memory");
}

// One CTA: 32 (i) x 32 (j) cells over kz planes; thread (tx, ty) owns column i = ib + tx
// and rows j = jb + 4 ty .. jb + 4 ty + 3.  Planes arrive two per TMA copy (a 40 x 34 x 2
// box); per plane each thread reads 6 rows x 3 columns of the staged box and forms the
// 3 x 3 maxima of its 4 cells separably (vertical 3-maxima sharing the middle pairs, then
// across the 3 columns).  A stage is released once both of its planes are folded.
__global__ void __launch_bounds__(kTX * kTY) pf_flag_tma_kernel(
    const __grid_constant__ CUtensorMap tm, const int8_t* __restrict__ mask,
    PfGeom g, float fcrit, int kz, uint32_t* __restrict__ bits, int32_t* __restrict__ status,
    long long wait_ns, unsigned inject_tx) {
    __shared__ __align__(128) float ring[kStages][kSlotFloats];
    __shared__ __align__(8) unsigned long long full[kStages];
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * kTX + tx;
    const int ib = g.nbuff + blockIdx.x * kTX;   // 0-based first i of the block
    const int jb = g.nbuff + blockIdx.y * kTYB;
    const int kb = g.nbuff + blockIdx.z * kz;
    const int hi = g.n - g.nbuff;                // exclusive end of the inner range
    const int i = ib + tx, j0 = jb + kRowsPT * ty;
    const bool icol = i < hi;
    const int kend = min(kb + kz, hi);
    const int x0 = (ib - 1) & ~3;                // 16-byte aligned box origin
    const int c0 = ib - 1 - x0 + tx;             // column of i - 1 inside the box
    const int r0 = kRowsPT * ty;                 // box row of j0 - 1
    const int nplanes = kend - kb + 2;           // planes kb - 1 .. kend
    const int nstages = (nplanes + kPPS - 1) / kPPS;
    const long long n = g.n, nn = n * n;
    // rows of this thread inside the inner range, and the bitmap word of (k = kb, j0)
    const int nrows = max(0, min(kRowsPT, hi - j0));
    long long word = ((long long)(kb - g.nbuff) * g.inner + (j0 - g.nbuff)) * g.wpr + blockIdx.x;
    const long long word_step_k = (long long)g.inner * g.wpr;

    if (tid == 0) {
        for (int s = 0; s < kStages; ++s) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_addr(&full[s])));
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncthreads();
    int issued = 0;   // stages issued (thread 0 only)
    if (tid == 0) {
        for (; issued < kStages && issued < nstages; ++issued)
            tma_plane(ring[issued], &tm, x0, jb - 1, kb - 1 + kPPS * issued, &full[issued],
                      issued == 0 ? inject_tx : 0u);
    }
    // 3x3 maxima of the thread's 4 cells in plane p, and their centre values
    auto fold = [&](int p, float (&m)[kRowsPT], float (&ctr)[kRowsPT]) {
        const float* pl = ring[(p / kPPS) % kStages] + (p % kPPS) * kPlaneFloats + r0 * kBoxX + c0;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            float r[kRowsPT + 2];
#pragma unroll
            for (int rr = 0; rr < kRowsPT + 2; ++rr) r[rr] = pl[rr * kBoxX + c];
            const float p1 = fmaxf(r[1], r[2]), p3 = fmaxf(r[3], r[4]);
            const float v0 = fmaxf(r[0], p1), v1 = fmaxf(p1, r[3]);
            const float v2 = fmaxf(r[2], p3), v3 = fmaxf(p3, r[5]);
            if (c == 0) {
                m[0] = v0; m[1] = v1; m[2] = v2; m[3] = v3;
            } else {
                m[0] = fmaxf(m[0], v0); m[1] = fmaxf(m[1], v1);
                m[2] = fmaxf(m[2], v2); m[3] = fmaxf(m[3], v3);
            }
            if (c == 1) {
#pragma unroll
                for (int rr = 0; rr < kRowsPT; ++rr) ctr[rr] = r[rr + 1];
            }
        }
    };
    int s_now = 0;
    // wait for stage s; false (uniformly) when the wait timed out
    auto wait_stage = [&](int s) {
        s_now = s;
        const bool ok = bar_wait(&full[s % kStages], (unsigned)((s / kStages) & 1), wait_ns);
        return ok;
    };
    // all warps are done with stage s: hand its slot to stage s + kStages
    auto release_stage = [&](bool ok) {
        if (__syncthreads_or(!ok)) return false;
        if (tid == 0 && issued < nstages) {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            tma_plane(ring[issued % kStages], &tm, x0, jb - 1, kb - 1 + kPPS * issued,
                      &full[issued % kStages]);
            ++issued;
        }
        return true;
    };
    float mprev[kRowsPT], mcur[kRowsPT], mnext[kRowsPT];
    float ff[kRowsPT], fnext[kRowsPT];
    // the peak test of plane k (centre values ff, maxima of planes k-1, k, k+1)
    auto test_plane = [&](int k) {
        unsigned w[kRowsPT];
#pragma unroll
        for (int rr = 0; rr < kRowsPT; ++rr) {
            // ff < fcrit skips; any neighbour > ff rejects (ties pass); mask == 1 skips.
            // fmaxf ignores NaN neighbours, matching `ff < NaN == false`.
            const float m27 = fmaxf(fmaxf(mprev[rr], mcur[rr]), mnext[rr]);
            bool peak = icol && rr < nrows && !(ff[rr] < fcrit) && !(ff[rr] < m27);
            if (peak) peak = __ldg(mask + (long long)i + n * (j0 + rr) + nn * k) != 1;
            w[rr] = __ballot_sync(0xffffffffu, peak);
        }
        // lane rr stores row rr's word
        if (tx < nrows) {
            unsigned v = w[0];
#pragma unroll
            for (int rr = 1; rr < kRowsPT; ++rr) v = tx == rr ? w[rr] : v;
            bits[word + (long long)tx * g.wpr] = v;
        }
        word += word_step_k;
#pragma unroll
        for (int rr = 0; rr < kRowsPT; ++rr) {
            mprev[rr] = mcur[rr];
            mcur[rr] = mnext[rr];
            ff[rr] = fnext[rr];
        }
    };

    // stage 0 holds planes kb - 1 and kb
    bool ok = wait_stage(0);
    fold(0, mprev, ff);
    fold(1, mcur, ff);
    ok = release_stage(ok);
    // each later stage s holds planes 2s, 2s + 1 (relative), i.e. k + 1 for k = kb + 2s - 2
    for (int s = 1; ok && s < nstages; ++s) {
        ok = wait_stage(s);
        const int k = kb + kPPS * s - 2;      // the plane whose test needs plane 2s
        if (k < kend) {
            fold(kPPS * s, mnext, fnext);
            test_plane(k);
        }
        if (k + 1 < kend) {
            fold(kPPS * s + 1, mnext, fnext);
            test_plane(k + 1);
        }
        ok = release_stage(ok);
    }
    if (!ok && tid == 0) {
        // record the timeout, then wait (bounded) for the copies still in flight
        atomicExch(status, kStatusWaitTimeout);
        for (int q = s_now; q < issued; ++q)
            bar_wait(&full[q % kStages], (unsigned)((q / kStages) & 1), wait_ns);
    }
}

__global__ void pf_count_kernel(const uint32_t* __restrict__ bits, long long nwords,
                                int32_t* __restrict__ segcount) {
    __shared__ int red[kEmitThreads / 32];
    const long long w0 = (long long)blockIdx.x * kSegWords;
    int c = 0;
    for (int t = threadIdx.x; t < kSegWords; t += blockDim.x) {
        const long long w = w0 + t;
        if (w < nwords) c += __popc(bits[w]);
    }
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        int s = 0;
        for (int i = 0; i < (int)(blockDim.x / 32); ++i) s += red[i];
        segcount[blockIdx.x] = s;
    }
}

// Single CTA: exclusive scan of segment counts into absolute slots.
__global__ void __launch_bounds__(1024) pf_scan_kernel(const int32_t* __restrict__ segcount,
                                                       int nseg, int64_t* __restrict__ segbase,
                                                       int64_t* count, int64_t* found,
                                                       int64_t max_peaks) {
    __shared__ long long warp_tot[32];
    __shared__ long long carry;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    if (tid == 0) carry = *count;
    __syncthreads();
    for (int base = 0; base < nseg; base += 1024) {
        const int s = base + tid;
        long long v = s < nseg ? segcount[s] : 0;
        long long x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            long long y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) warp_tot[wid] = x;
        __syncthreads();
        if (wid == 0) {
            long long t = warp_tot[lane];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                long long y = __shfl_up_sync(0xffffffffu, t, o);
                if (lane >= o) t += y;
            }
            warp_tot[lane] = t;
        }
        __syncthreads();
        const long long before = (wid > 0 ? warp_tot[wid - 1] : 0) + x - v;
        if (s < nseg) segbase[s] = carry + before;
        __syncthreads();
        if (tid == 1023) carry += warp_tot[31];
        __syncthreads();
    }
    if (tid == 0) {
        const long long total_new = carry - *count;
        if (found) *found += total_new;
        *count = carry < max_peaks ? carry : max_peaks;
    }
}

__global__ void __launch_bounds__(kEmitThreads) pf_emit_kernel(
    const uint32_t* __restrict__ bits, PfGeom g, const int64_t* __restrict__ segbase,
    const float* __restrict__ ds, const float* __restrict__ lapd_s, int8_t* __restrict__ mask,
    int32_t filter_idx, int64_t max_peaks, ht_peaks out, int32_t* status) {
    __shared__ int warp_tot[kEmitThreads / 32];
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const long long w0 = (long long)blockIdx.x * kSegWords + (long long)tid * kWordsPerThread;
    const long long seg0 = __ldg(segbase + blockIdx.x);   // in flight with the words
    uint32_t words[kWordsPerThread];
    static_assert(kWordsPerThread == 8, "two 16-byte loads per thread");
    if (w0 + kWordsPerThread <= g.nwords) {
        // 32-byte aligned: the workspace is, and w0 is a multiple of 8 words
        const uint4 a = __ldg(reinterpret_cast<const uint4*>(bits + w0));
        const uint4 b = __ldg(reinterpret_cast<const uint4*>(bits + w0 + 4));
        words[0] = a.x; words[1] = a.y; words[2] = a.z; words[3] = a.w;
        words[4] = b.x; words[5] = b.y; words[6] = b.z; words[7] = b.w;
    } else {
#pragma unroll
        for (int t = 0; t < kWordsPerThread; ++t)
            words[t] = w0 + t < g.nwords ? bits[w0 + t] : 0u;
    }
    int c = 0;
#pragma unroll
    for (int t = 0; t < kWordsPerThread; ++t) c += __popc(words[t]);
    // block exclusive scan of c
    int x = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_tot[wid] = x;
    __syncthreads();
    int wbase = 0;
    for (int i = 0; i < wid; ++i) wbase += warp_tot[i];
    long long slot = seg0 + wbase + x - c;
    if (c == 0 || slot >= max_peaks) return;
    const long long n = g.n, nn = n * n;
#pragma unroll
    for (int t = 0; t < kWordsPerThread; ++t) {
        uint32_t wd = words[t];
        if (!wd) continue;
        const long long w = w0 + t;
        const long long row = w / g.wpr;
        const int ib = (int)(w - row * g.wpr) * 32;
        const int kk = (int)(row / g.inner), jj = (int)(row - (long long)kk * g.inner);
        while (wd) {
            const int b = __ffs(wd) - 1;
            wd &= wd - 1;
            if (slot >= max_peaks) return;
            const int i = g.nbuff + ib + b, j = g.nbuff + jj, k = g.nbuff + kk;   // 0-based
            const long long cidx = (long long)i + n * j + nn * k;
            if (!HT_INDEX_OK(status, cidx, nn * n)) continue;
            out.i[slot] = i + 1;
            out.j[slot] = j + 1;
            out.k[slot] = k + 1;
            out.delta[slot] = ds[cidx];
            if (out.lapd) out.lapd[slot] = lapd_s ? lapd_s[cidx] : 0.f;
            out.filter_idx[slot] = filter_idx;
            mask[cidx] = 1;
            ++slot;
        }
    }
}


// cuTensorMapEncodeTiled from the driver, looked up once per process.
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static std::once_flag once;
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
                cudaSuccess && q == cudaDriverEntryPointSuccess)
            fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
    });
    return fn;
}

// 3-D tensor map of an n^3 FP32 field with a (40, 10, 1) box; false when the field does
// not meet TMA's rules (row pitch a multiple of 16 bytes, 16-byte aligned base) or is
// narrower than the box, and the plain-load kernel is used instead.
bool pf_tensor_map(CUtensorMap* tm, const float* d, int n) {
    if (n % 4 != 0 || n < kBoxX || ((uintptr_t)d & 15u) != 0) return false;
    PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
    if (!enc) return false;
    const cuuint64_t dims[3] = {(cuuint64_t)n, (cuuint64_t)n, (cuuint64_t)n};
    const cuuint64_t strides[2] = {(cuuint64_t)n * 4, (cuuint64_t)n * n * 4};
    const cuuint32_t box[3] = {kBoxX, kBoxY, kPPS};
    const cuuint32_t estr[3] = {1, 1, 1};
    return enc(tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, (void*)d, dims, strides, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
               CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

}  // namespace

int ht_launch_peakfind(ht_ctx* ctx, const float* d_delta_s, const float* d_lapd_s,
                       int8_t* d_mask, int n, int nbuff, float fcrit, int32_t filter_idx,
                       int64_t max_peaks, const ht_peaks* out, cudaStream_t st) {
    PfGeom g;
    g.n = n;
    g.nbuff = nbuff;
    g.inner = n - 2 * nbuff;
    g.wpr = (g.inner + 31) / 32;
    g.nwords = (long long)g.inner * g.inner * g.wpr;
    ctx->last_kernels = 0;
    if (g.inner <= 0) return HT_OK;
    const long long nseg = (g.nwords + kSegWords - 1) / kSegWords;
    const size_t bits_bytes = ((size_t)g.nwords * 4 + 255) / 256 * 256;
    const size_t need = bits_bytes + (size_t)nseg * (4 + 8) + 256;
    int rc = ht_grow(&ctx->d_pf_ws, &ctx->pf_ws_bytes, need, "peak-find workspace");
    if (rc != HT_OK) return rc;
    uint32_t* bits = (uint32_t*)ctx->d_pf_ws;
    int64_t* segbase = (int64_t*)((char*)ctx->d_pf_ws + bits_bytes);
    int32_t* segcount = (int32_t*)(segbase + nseg);

    const unsigned gx = (unsigned)((g.inner + kTX - 1) / kTX);
    const unsigned gy = (unsigned)((g.inner + kTY - 1) / kTY);
    CUtensorMap tm;
    if (pf_tensor_map(&tm, d_delta_s, n)) {
        // planes per CTA: 64, halved while the grid would give fewer than 16 CTAs per SM
        int kz = 64;
        const long long want = 16LL * ctx->num_sms;
        const unsigned gyb = (unsigned)((g.inner + kTYB - 1) / kTYB);
        while (kz > 8 && (long long)gx * gyb * ((g.inner + kz - 1) / kz) < want) kz >>= 1;
        if (ctx->tune_pf_kz > 0) kz = ctx->tune_pf_kz;   // autotuned (ht_ctx_tune)
        dim3 grid1(gx, gyb, (unsigned)((g.inner + kz - 1) / kz));
        pf_flag_tma_kernel<<<grid1, dim3(kTX, kTY), 0, st>>>(tm, d_mask, g, fcrit, kz, bits,
                                                             ht_status_word(ctx), ctx->wait_ns,
                                                             ctx->inject_tx);
        HT_CUDA_TRY(cudaGetLastError(), "pf_flag_tma_kernel launch");
    } else {
        dim3 grid1(gx, gy, (unsigned)((g.inner + kKZ - 1) / kKZ));
        pf_flag_kernel<<<grid1, dim3(kTX, kTY), 0, st>>>(d_delta_s, d_mask, g, fcrit, bits);
        HT_CUDA_TRY(cudaGetLastError(), "pf_flag_kernel launch");
    }
    pf_count_kernel<<<(unsigned)nseg, kEmitThreads, 0, st>>>(bits, g.nwords, segcount);
    HT_CUDA_TRY(cudaGetLastError(), "pf_count_kernel launch");
    pf_scan_kernel<<<1, 1024, 0, st>>>(segcount, (int)nseg, segbase, out->count, out->found,
                                       max_peaks);
    HT_CUDA_TRY(cudaGetLastError(), "pf_scan_kernel launch");
    pf_emit_kernel<<<(unsigned)nseg, kEmitThreads, 0, st>>>(bits, g, segbase, d_delta_s,
                                                             d_lapd_s, d_mask, filter_idx,
                                                             max_peaks, *out,
                                                             ht_status_word(ctx));
    HT_CUDA_TRY(cudaGetLastError(), "pf_emit_kernel launch");
    ctx->last_kernels = 4;
    return HT_OK;
}
