// Peak finding on one smoothed field (PeakFind.jl:15-78 semantics) on sm_100a.
//
// Four launches per filter, all deterministic:
//   1. flag  : 26-neighbour local-maximum test of every inner cell.  A CTA owns a
//              32 (i) x 8 (j) column block and streams KZ planes in k through a
//              3-plane shared-memory ring with a one-cell halo; every delta_s value is
//              read from HBM once per CTA.  Survivors are compacted into a bitmap with
//              one __ballot_sync word per (k, j, 32-cell run of i), laid out in the
//              CPU scan order k -> j -> i.
//   2. count : popcount of each segment of kSegWords bitmap words.
//   3. scan  : one CTA turns the segment counts into absolute output slots after the
//              peaks of earlier filters and advances the running count.
//   4. emit  : each segment re-reads its words, ranks its set bits in scan order and
//              writes (i, j, k, delta_s, lapd_s, filter) plus mask = 1 for every slot
//              below max_peaks.
// Result: the same peak list, in the same order, as the CPU scan, independent of
// thread timing (the reference GPU kernel reserves slots with an atomic counter and is
// order-nondeterministic, ext/CUDAExt.jl:2921).
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
    int32_t filter_idx, int64_t max_peaks, ht_peaks out) {
    __shared__ int warp_tot[kEmitThreads / 32];
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const long long w0 = (long long)blockIdx.x * kSegWords + (long long)tid * kWordsPerThread;
    uint32_t words[kWordsPerThread];
    int c = 0;
#pragma unroll
    for (int t = 0; t < kWordsPerThread; ++t) {
        const long long w = w0 + t;
        words[t] = w < g.nwords ? bits[w] : 0u;
        c += __popc(words[t]);
    }
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
    long long slot = segbase[blockIdx.x] + wbase + x - c;
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

    dim3 grid1((g.inner + kTX - 1) / kTX, (g.inner + kTY - 1) / kTY, (g.inner + kKZ - 1) / kKZ);
    pf_flag_kernel<<<grid1, dim3(kTX, kTY), 0, st>>>(d_delta_s, d_mask, g, fcrit, bits);
    HT_CUDA_TRY(cudaGetLastError(), "pf_flag_kernel launch");
    pf_count_kernel<<<(unsigned)nseg, kEmitThreads, 0, st>>>(bits, g.nwords, segcount);
    HT_CUDA_TRY(cudaGetLastError(), "pf_count_kernel launch");
    pf_scan_kernel<<<1, 1024, 0, st>>>(segcount, (int)nseg, segbase, out->count, out->found,
                                       max_peaks);
    HT_CUDA_TRY(cudaGetLastError(), "pf_scan_kernel launch");
    pf_emit_kernel<<<(unsigned)nseg, kEmitThreads, 0, st>>>(bits, g, segbase, d_delta_s,
                                                             d_lapd_s, d_mask, filter_idx,
                                                             max_peaks, *out);
    HT_CUDA_TRY(cudaGetLastError(), "pf_emit_kernel launch");
    ctx->last_kernels = 4;
    return HT_OK;
}
