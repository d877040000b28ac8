// Warp-level inverse complex FFT of one column of L = 32 T points held in shared memory,
// for the fused smoothing passes (ht_smooth.cu).  Convention: y[k] = sum_t x[t] e^{+2 pi i
// t k / L} (unnormalised inverse).
//
// Four-step with L = 32 x T (Bailey 1990): lane l (0..31) owns x[l + 32 t], t = 0..T-1.
//   1. each lane: T-point DFT over t in registers (mixed radix 2/3/4, composed),
//   2. twiddle by e^{2 pi i l k2 / L} (read from a lane-major table: coalesced),
//   3. for every k2: 32-point DFT across the lanes with xor shuffles (radix-2,
//      decimation in frequency: lane l ends with index k1 = bitrev5(l)),
//   4. y[k2 + T k1] goes back to the column.
// Small-DFT twiddles come from __constant__ tables of e^{2 pi i j / N} computed on the host
// in FP64 (fused_tables in ht_smooth.cu); the lane-dependent step-2 twiddles from a per-L
// global table laid out [k2][lane], so that a warp reads 256 contiguous bytes per k2.
#pragma once

#include <cuda_runtime.h>

namespace htfft {

struct C2 {
    float x, y;
};

__device__ __forceinline__ C2 add(C2 a, C2 b) { return {a.x + b.x, a.y + b.y}; }
__device__ __forceinline__ C2 sub(C2 a, C2 b) { return {a.x - b.x, a.y - b.y}; }
__device__ __forceinline__ C2 mul(C2 a, C2 b) {
    return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}
__device__ __forceinline__ C2 muli(C2 a) { return {-a.y, a.x}; }   // i * a
__device__ __forceinline__ C2 scale(C2 a, float s) { return {a.x * s, a.y * s}; }
__device__ __forceinline__ C2 to_c2(float2 e) { return {e.x, e.y}; }

// e^{2 pi i j / N} for the small composite sizes used in registers (N = 8, 9, 18, 32, 36);
// this header belongs to one translation unit (ht_smooth.cu), which fills them at set-up.
__constant__ float2 c_w8[8];
__constant__ float2 c_w9[9];
__constant__ float2 c_w18[18];
__constant__ float2 c_w32[32];
__constant__ float2 c_w36[36];

template <int N>
__device__ __forceinline__ C2 wsmall(int j);   // e^{2 pi i j / N}, j in [0, N)
template <>
__device__ __forceinline__ C2 wsmall<8>(int j) { const float2 w = c_w8[j]; return {w.x, w.y}; }
template <>
__device__ __forceinline__ C2 wsmall<32>(int j) { const float2 w = c_w32[j]; return {w.x, w.y}; }
template <>
__device__ __forceinline__ C2 wsmall<9>(int j) { const float2 w = c_w9[j]; return {w.x, w.y}; }
template <>
__device__ __forceinline__ C2 wsmall<18>(int j) { const float2 w = c_w18[j]; return {w.x, w.y}; }
template <>
__device__ __forceinline__ C2 wsmall<36>(int j) { const float2 w = c_w36[j]; return {w.x, w.y}; }

// In-register inverse DFT of N points; v[] in natural order on input and output.
template <int N>
struct Dft;

template <>
struct Dft<2> {
    __device__ __forceinline__ static void run(C2 (&v)[2]) {
        const C2 a = v[0], b = v[1];
        v[0] = add(a, b);
        v[1] = sub(a, b);
    }
};

template <>
struct Dft<3> {
    __device__ __forceinline__ static void run(C2 (&v)[3]) {
        const float h = 0.8660254037844386f;   // sqrt(3) / 2
        const C2 a = v[0], s = add(v[1], v[2]), d = sub(v[1], v[2]);
        const C2 m = {a.x - 0.5f * s.x, a.y - 0.5f * s.y};
        const C2 id = scale(muli(d), h);
        v[0] = add(a, s);
        v[1] = add(m, id);
        v[2] = sub(m, id);
    }
};

template <>
struct Dft<4> {
    __device__ __forceinline__ static void run(C2 (&v)[4]) {
        const C2 t0 = add(v[0], v[2]), t1 = sub(v[0], v[2]);
        const C2 t2 = add(v[1], v[3]), t3 = muli(sub(v[1], v[3]));
        v[0] = add(t0, t2);
        v[2] = sub(t0, t2);
        v[1] = add(t1, t3);
        v[3] = sub(t1, t3);
    }
};

// a e^{2 pi i j / N}; the quarter turns (j N/4) are sign changes and swaps
template <int N>
__device__ __forceinline__ C2 twiddle(C2 a, int j) {
    if (j == 0) return a;
    if (4 * j == N) return muli(a);
    if (2 * j == N) return {-a.x, -a.y};
    if (4 * j == 3 * N) return {a.y, -a.x};
    return mul(a, wsmall<N>(j));
}

// N = R1 R2: x[t1 + R1 t2] -> y[k2 + R2 k1] = sum_t1 w_R1^{t1 k1} w_N^{t1 k2}
//                                               sum_t2 x[t1 + R1 t2] w_R2^{t2 k2}
template <int R1, int R2>
struct DftComposite {
    static constexpr int N = R1 * R2;
    __device__ __forceinline__ static void run(C2 (&v)[N]) {
        C2 u[N];
#pragma unroll
        for (int t1 = 0; t1 < R1; ++t1) {
            C2 a[R2];
#pragma unroll
            for (int t2 = 0; t2 < R2; ++t2) a[t2] = v[t1 + R1 * t2];
            Dft<R2>::run(a);
#pragma unroll
            for (int k2 = 0; k2 < R2; ++k2)
                u[t1 + R1 * k2] = twiddle<N>(a[k2], (t1 * k2) % N);
        }
#pragma unroll
        for (int k2 = 0; k2 < R2; ++k2) {
            C2 b[R1];
#pragma unroll
            for (int t1 = 0; t1 < R1; ++t1) b[t1] = u[t1 + R1 * k2];
            Dft<R1>::run(b);
#pragma unroll
            for (int k1 = 0; k1 < R1; ++k1) v[k2 + R2 * k1] = b[k1];
        }
    }
};

template <>
struct Dft<8> {
    __device__ __forceinline__ static void run(C2 (&v)[8]) { DftComposite<2, 4>::run(v); }
};
template <>
struct Dft<32> {
    __device__ __forceinline__ static void run(C2 (&v)[32]) { DftComposite<4, 8>::run(v); }
};
template <>
struct Dft<9> {
    __device__ __forceinline__ static void run(C2 (&v)[9]) { DftComposite<3, 3>::run(v); }
};
template <>
struct Dft<18> {
    __device__ __forceinline__ static void run(C2 (&v)[18]) { DftComposite<2, 9>::run(v); }
};
template <>
struct Dft<36> {
    __device__ __forceinline__ static void run(C2 (&v)[36]) { DftComposite<4, 9>::run(v); }
};

__device__ __forceinline__ int bitrev5(int l) { return __brev((unsigned)l) >> 27; }

// Shared-memory slot of y[i] in the "row-major" column layout of the transposed form:
// row k2 = i mod T holds y[k2 + T k1] at k2 * 33 + k1 (32 values and a pad), so that a
// warp writing X[lane][k2] for one k2 covers 32 consecutive slots and a thread reading
// row k2 walks consecutive slots.  A column needs 33 T slots.
template <int T>
__device__ __forceinline__ int km_slot(int i) {
    const int k1 = i / T;
    return (i - T * k1) * 33 + k1;
}

// The 32-point DFT of row k2 of a row-major column (in place): x[l] = X[l][k2] at
// k2 * 33 + l on entry, y[k2 + T k1] at k2 * 33 + k1 on exit.
__device__ __forceinline__ void dft32_row(float2* row) {
    C2 v[32];
#pragma unroll
    for (int l = 0; l < 32; ++l) v[l] = to_c2(row[l]);
    Dft<32>::run(v);
#pragma unroll
    for (int k = 0; k < 32; ++k) row[k] = make_float2(v[k].x, v[k].y);
}

// Steps 1-2 only: on entry lane holds v[t] = x[lane + 32 t]; on exit v[k2] is the twiddled
// inner transform X[lane][k2], whose 32-point DFTs over the lanes (one per k2) give
// y[k2 + T k1].  For kernels that finish those DFTs in registers after a shared-memory
// transpose (dft32_rows) instead of across lanes.
template <int T>
__device__ __forceinline__ void warp_ifft_inner(C2 (&v)[T], const float2* __restrict__ twLM,
                                                int lane) {
    Dft<T>::run(v);
#pragma unroll
    for (int k2 = 1; k2 < T; ++k2) {
        const float2 w = __ldg(twLM + 32 * k2 + lane);
        v[k2] = mul(v[k2], {w.x, w.y});
    }
}

// Step 3 for rows k2 in [K0, T): the 32-point DFT across lanes, decimation in frequency
// (spans 16, 8, 4, 2, 1); lane l ends with y[k2 + T k1], k1 = bitrev5(l).  Lower lane:
// a + b; upper lane: (b - a) w_{2s}^{lane mod s}, written as one signed sum b + sg a and a
// product by we (1 on lower lanes, and on every lane of the last stage, where w_2^0 = 1):
// the same roundings as the two-branch form, a third of the work.
template <int T, int K0>
__device__ __forceinline__ void cross32(C2 (&v)[T], int lane, const C2 (&w32)[5]) {
#pragma unroll
    for (int st = 4; st >= 0; --st) {
        const int s = 1 << st;
        const bool upper = (lane & s) != 0;
        const float sg = upper ? -1.f : 1.f;
        const C2 we = upper ? w32[st] : C2{1.f, 0.f};
#pragma unroll
        for (int k2 = K0; k2 < T; ++k2) {
            const C2 a = v[k2];
            const C2 b = {__shfl_xor_sync(0xffffffffu, a.x, s),
                          __shfl_xor_sync(0xffffffffu, a.y, s)};
            const C2 r = {fmaf(sg, a.x, b.x), fmaf(sg, a.y, b.y)};
            v[k2] = st == 0 ? r : mul(r, we);
        }
    }
}

// Steps 1-3 on registers: on entry lane holds v[t] = x[lane + 32 t]; on exit v[k2] =
// y[k2 + T k1] with k1 = bitrev5(lane).
// twLM[32 k2 + l] = e^{2 pi i l k2 / (32 T)}, k2 < T, l < 32 (global, cached).  w32[s] for
// the cross-lane stages (precomputed by the caller per lane):
// w32[s] = e^{2 pi i (lane mod 2^s) / 2^{s+1}}.
template <int T>
__device__ __forceinline__ void warp_ifft_regs(C2 (&v)[T], const float2* __restrict__ twLM,
                                               int lane, const C2 (&w32)[5]) {
    warp_ifft_inner<T>(v, twLM, lane);
    cross32<T, 0>(v, lane, w32);
}

// Inverse FFT of the column col[0 .. 32 T) (shared memory, float2), in place, natural
// order on input and output.
template <int T>
__device__ __forceinline__ void warp_ifft(float2* col, const float2* __restrict__ twLM, int lane,
                                          const C2 (&w32)[5]) {
    C2 v[T];
#pragma unroll
    for (int t = 0; t < T; ++t) {
        v[t] = to_c2(col[lane + 32 * t]);
    }
    warp_ifft_regs<T>(v, twLM, lane, w32);
    __syncwarp();
    const int k1 = bitrev5(lane);
#pragma unroll
    for (int k2 = 0; k2 < T; ++k2) col[k2 + T * k1] = make_float2(v[k2].x, v[k2].y);
    __syncwarp();
}

// Shared-memory slot of output y[i] (i = k2 + T k1) in the "lane-major" column layout that
// warp_ifft_store writes: slot rot(k1) + 33 k2, rot(k1) = (k1 >> 1) | ((k1 & 1) << 4).  A
// warp's store of one k2 covers 32 consecutive slots, and each half-warp (even k1 in lanes
// 0-15, odd k1 in lanes 16-31, as k1 = bitrev5(lane)) 16 consecutive ones; readers walking i
// in order step 33 slots (one bank pair) apart: both sides are free of bank conflicts for
// 8-byte elements.  A column needs 33 T slots.
__device__ __forceinline__ int lm_rot(int k1) { return (k1 >> 1) | ((k1 & 1) << 4); }

template <int T>
__device__ __forceinline__ int lm_slot(int i) {
    const int k1 = i / T;
    return lm_rot(k1) + 33 * (i - T * k1);
}

// Store the result of warp_ifft_regs into a lane-major column (33 T slots).
template <int T>
__device__ __forceinline__ void warp_ifft_store(float2* col, const C2 (&v)[T], int lane) {
    const int s = lm_rot(bitrev5(lane));
#pragma unroll
    for (int k2 = 0; k2 < T; ++k2) col[s + 33 * k2] = make_float2(v[k2].x, v[k2].y);
}

// Per-lane cross-lane twiddles for warp_ifft: w32[st] = e^{2 pi i (lane mod 2^st) / 2^(st+1)}
__device__ __forceinline__ void lane_twiddles(int lane, const float2* __restrict__ tw32,
                                              C2 (&w32)[5]) {
#pragma unroll
    for (int st = 0; st < 5; ++st) {
        const int s = 1 << st;
        // e^{2 pi i j / (2s)} = e^{2 pi i j (16 / s) / 32}, j = lane mod s
        const float2 w = __ldg(tw32 + ((lane & (s - 1)) * (16 / s)));
        w32[st] = {w.x, w.y};
    }
}

}  // namespace htfft
