// Learned walk-length bracket: a 12 -> 64 -> 64 -> 64 -> 2 MLP (BF16 weights and
// activations, FP32 accumulation on the tensor cores) that predicts,
// for every peak, a low and a high quantile of the radius at which its shell walk stops.
// The shell collapse itself never reads the prediction: it only orders the work (peaks with
// similar predicted walks share a warp, longest first), so every result is identical to the
// unordered path.  No counterpart in the reference.
//
// Features (per peak, all known before the walk):
//   0 Rf / alatt          1 sqrt(ir2min)         2 delta_s at the peak (FcRf)
//   3 fcrit               4 ZZon                 5 delta at the peak cell
//   6..9 mean delta over the in-tile cells of shells 2, 3, 4, 5 (radii 1, sqrt2, sqrt3, 2)
//   10 rad[m0_init]       11 Rf / alatt + 2 (how far the walk must reach at least: the
//                            first shell past ir2min and the gradient window at Rf)
//   12..15 zero padding (K = 16 for the first tensor-core layer)
// Features are standardised with the model's mean / std before the first layer.
//
// Kernels:
//   features_kernel      one thread per peak
//   mlp_infer_tc_kernel  inference, 128 peaks per CTA tile: every layer a tcgen05.mma chain
//                        from shared memory into tensor memory, read back per row
//                        (tcgen05.ld), bias + ReLU + BF16 as the next layer's operand
//   gemm_bf16_kernel     generic C = op(A) op(B) (BF16 in, FP32 out, mma.sync m16n8k16)
//                        for training (offline, not on the step):
//                        forward products, activation gradients and weight gradients
//   small elementwise kernels for bias/ReLU, the pinball-loss gradient, ReLU backward,
//   bias gradients and Adam.
#include <cuda_bf16.h>
#include <math.h>

#include <cub/device/device_radix_sort.cuh>
#include <string>

#include "ht_async.cuh"
#include "ht_internal.cuh"

namespace {

constexpr int kIn = 16, kHid = 64;

__device__ __forceinline__ unsigned pack_bf16(float lo, float hi) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);   // .x = lo (low half)
    unsigned u;
    memcpy(&u, &v, 4);
    return u;
}

__device__ __forceinline__ void mma_bf16(float (&c)[4], const unsigned (&a)[4], unsigned b0,
                                         unsigned b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
        "{%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, {%0, %1, %2, %3};"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// ---------------------------------------------------------------- features ----

struct FeatArgs {
    const float4* rec;        // packed records of the bound tile (nullable)
    const float* delta;       // or the delta field
    int n1, n2, n3;
    long long s2;
    const char4* off;
    const int32_t* start;
    const int32_t* count;
    const int32_t* r2;
    const double* rad;
    int nshells;
    const int32_t* pi;
    const int32_t* pj;
    const int32_t* pk;
    const double* Rf;
    const int32_t* ir2min;
    const float* ZZon;
    const float* fcrit;
    const float* peak_delta;  // delta_s at each peak (nullable: 0)
    long long npeaks;
    double alatt;
};

__global__ void __launch_bounds__(256) features_kernel(const FeatArgs a, float* __restrict__ F) {
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= a.npeaks) return;
    const int ci = a.pi[p], cj = a.pj[p], ck = a.pk[p];
    float f[kIn];
#pragma unroll
    for (int i = 0; i < kIn; ++i) f[i] = 0.f;
    const double Rf = a.Rf[p];
    const int ir2 = a.ir2min[p];
    f[0] = (float)(Rf / a.alatt);
    f[1] = sqrtf((float)max(ir2, 0));
    f[2] = a.peak_delta ? a.peak_delta[p] : 0.f;
    f[3] = a.fcrit[p];
    f[4] = a.ZZon[p];
    auto value = [&](int i, int j, int k, float& v) {
        if (i < 1 || i > a.n1 || j < 1 || j > a.n2 || k < 1 || k > a.n3) return false;
        const long long idx = (long long)(i - 1) + (long long)a.n1 * (j - 1) + a.s2 * (k - 1);
        v = a.rec ? __ldg(a.rec + 2 * idx).x : __ldg(a.delta + idx);
        return true;
    };
    float v;
    if (value(ci, cj, ck, v)) f[5] = v;
    // shells 2-5 (r^2 = 1, 2, 3, 4) hold 6, 12, 8 and 6 cells, the table's first 32 after the
    // centre: a peak at least two cells inside the tile has every one of them, so all 32
    // loads go out before any is summed (same sums, same order as the loop below)
    const bool inner2 = a.nshells >= 5 && ci > 2 && ci + 2 <= a.n1 && cj > 2 &&
                        cj + 2 <= a.n2 && ck > 2 && ck + 2 <= a.n3;
    if (inner2) {
        const long long c0 = (long long)(ci - 1) + (long long)a.n1 * (cj - 1) + a.s2 * (ck - 1);
        const int st2 = __ldg(a.start + 2);
        float w[32];
#pragma unroll
        for (int c = 0; c < 32; ++c) {
            const char4 o = __ldg(a.off + st2 + c);
            const long long idx = c0 + o.x + (long long)a.n1 * o.y + a.s2 * o.z;
            w[c] = a.rec ? __ldg(reinterpret_cast<const float*>(a.rec + 2 * idx))
                         : __ldg(a.delta + idx);
        }
        constexpr int kFirst[5] = {0, 6, 18, 26, 32};
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            float sum = 0.f;
#pragma unroll
            for (int c = kFirst[s]; c < kFirst[s + 1]; ++c) sum += w[c];
            const int nin = kFirst[s + 1] - kFirst[s];
            f[6 + s] = sum / nin;
        }
    }
    for (int s = 2; !inner2 && s <= 5 && s <= a.nshells; ++s) {
        const int st = __ldg(a.start + s), cnt = __ldg(a.count + s);
        float sum = 0.f;
        int nin = 0;
        for (int c = st; c < st + cnt; ++c) {
            const char4 o = __ldg(a.off + c);
            if (value(ci + o.x, cj + o.y, ck + o.z, v)) { sum += v; ++nin; }
        }
        f[4 + s] = nin ? sum / nin : 0.f;
    }
    // data-independent walk bounds: first shell with r2 > ir2min, and where the gradient
    // window at the filter radius ends
    int lo = 1, hi = a.nshells - 1, m0 = a.nshells - 1;
    while (lo <= hi) {
        const int mid = (lo + hi) >> 1;
        if (a.r2[mid] > ir2) { m0 = mid; hi = mid - 1; } else { lo = mid + 1; }
    }
    f[10] = (float)a.rad[m0];
    const double RR = Rf / a.alatt;
    f[11] = (float)(RR + 2.0);
    float* out = F + p * kIn;
#pragma unroll
    for (int i = 0; i < kIn; i += 4) *reinterpret_cast<float4*>(out + i) = make_float4(f[i], f[i + 1], f[i + 2], f[i + 3]);
}

// --------------------------------------------------------- fused inference ----

struct MlpW {
    const __nv_bfloat16* W1;   // [64][16]
    const __nv_bfloat16* W2;   // [64][64]
    const __nv_bfloat16* W3;   // [64][64]
    const __nv_bfloat16* W4;   // [8][64] (rows 2..7 zero)
    const float* b1;           // [64]
    const float* b2;
    const float* b3;
    const float* b4;           // [8]
    const float* mean;         // [16] feature standardisation
    const float* istd;         // [16]
};

// ------------------------------------------------- fused inference, tcgen05 ----
//
// The same four layers on the 5th-generation tensor cores.  A CTA of 128 threads takes
// tiles of 128 peaks (M = 128), persistent over the tiles.  Every layer is a chain of
// tcgen05.mma (kind::f16, BF16 x BF16 -> FP32, one elected thread issues them) from shared
// memory into a 64-column accumulator in tensor memory: the activations A [128 x K] and the
// layer's weights W [N x K] (the row-major weights are K-major already) sit in the
// no-swizzle K-major layout of 8-row x 16-byte core matrices.  The MMAs of a layer are
// committed to an mbarrier; every thread then reads its own row back (tcgen05.ld 32x32b:
// warp w owns lanes 32w .. 32w + 31, and row r of an M = 128 accumulator is lane r), adds
// the bias, applies ReLU, rounds to BF16 and writes the row as the next layer's A.  The
// output layer is padded to N = 16 (weight rows 2 .. 15 zero).  Waits are bounded; a wait
// that gives up records the status, and the CTA still frees its tensor memory.

constexpr int kTcRows = 128;    // peaks per tile (the MMA's M)
constexpr int kTcN4 = 16;       // the output layer's N (2 used)
constexpr int kTcCols = 64;     // tensor-memory columns per CTA (FP32 accumulator, N <= 64)

// Byte offset of element (r, k) in a K-major operand of R rows: core matrices of 8 rows x
// 8 K-values (16 bytes a row, 128 bytes each), row groups 128 bytes apart (the descriptor's
// stride offset), the two K halves of a 16-wide K step R x 16 bytes apart (its leading
// offset), K steps R x 32 bytes apart.
__host__ __device__ constexpr int umma_off(int R, int r, int k) {
    return (k >> 4) * (R * 32) + ((k >> 3) & 1) * (R * 16) + (r >> 3) * 128 + (r & 7) * 16 +
           (k & 7) * 2;
}

// Shared-memory matrix descriptor of such an operand (R rows) starting at shared address
// saddr: start >> 4 in bits [0, 14), leading offset >> 4 in [16, 30), stride offset >> 4
// in [32, 46), version 1 in [46, 48), no swizzle, base offset 0.
__device__ __forceinline__ unsigned long long umma_desc(unsigned saddr, int R) {
    const unsigned long long lbo = (unsigned long long)(R * 16) >> 4, sbo = 128ull >> 4;
    return (unsigned long long)((saddr >> 4) & 0x3FFFu) | (lbo << 16) | (sbo << 32) |
           (1ull << 46);
}

// Instruction descriptor: FP32 accumulator, BF16 A and B, both K-major, N >> 3 in bits
// [17, 23), M >> 4 in bits [24, 29).
__host__ __device__ constexpr unsigned umma_idesc(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((unsigned)(N >> 3) << 17) |
           ((unsigned)(M >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(unsigned tmem_d, unsigned long long da,
                                          unsigned long long db, unsigned idesc,
                                          unsigned accumulate) {
    const unsigned z = 0u;
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
        :: "r"(tmem_d), "l"(da), "l"(db), "r"(idesc), "r"(accumulate), "r"(z), "r"(z), "r"(z),
           "r"(z));
}

__device__ __forceinline__ void umma_commit(unsigned long long* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 :: "r"(htasync::smem_addr(bar)) : "memory");
}

__device__ __forceinline__ void tc_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// 16 consecutive accumulator columns of this thread's lane.
__device__ __forceinline__ void tmem_ld16(unsigned taddr, float (&v)[16]) {
    unsigned u[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
        : "=r"(u[0]), "=r"(u[1]), "=r"(u[2]), "=r"(u[3]), "=r"(u[4]), "=r"(u[5]), "=r"(u[6]),
          "=r"(u[7]), "=r"(u[8]), "=r"(u[9]), "=r"(u[10]), "=r"(u[11]), "=r"(u[12]),
          "=r"(u[13]), "=r"(u[14]), "=r"(u[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(u[i]);
}

// Shared-memory layout of the tcgen05 inference kernel (bytes from the dynamic base).
constexpr int kTcOffA = 0;                                  // A [128 x 64] BF16
constexpr int kTcOffW1 = kTcOffA + kTcRows * kHid * 2;      // W1 [64 x 16]
constexpr int kTcOffW2 = kTcOffW1 + kHid * kIn * 2;         // W2 [64 x 64]
constexpr int kTcOffW3 = kTcOffW2 + kHid * kHid * 2;        // W3 [64 x 64]
constexpr int kTcOffW4 = kTcOffW3 + kHid * kHid * 2;        // W4 [16 x 64]
constexpr int kTcOffB = kTcOffW4 + kTcN4 * kHid * 2;        // b1 b2 b3 [64] b4 [8], FP32
constexpr int kTcSmem = kTcOffB + (3 * kHid + 8) * 4;

// Copy the row-major weights W [rows x K] (global, BF16) into the K-major layout with Rpad
// rows (rows >= rows zero).
__device__ __forceinline__ void stage_weights(unsigned char* dst, const __nv_bfloat16* W,
                                              int rows, int Rpad, int K, int tid, int nthr) {
    for (int e = tid; e < Rpad * (K / 2); e += nthr) {
        const int r = e / (K / 2), k = 2 * (e % (K / 2));
        const unsigned v = r < rows ? __ldg(reinterpret_cast<const unsigned*>(W + (size_t)r * K + k))
                                    : 0u;
        *reinterpret_cast<unsigned*>(dst + umma_off(Rpad, r, k)) = v;
    }
}

// Bias, ReLU and BF16 rounding of the 64 columns of this thread's row, written as row r of
// the next layer's A.
__device__ __forceinline__ void hidden_out(unsigned tmem_row, const float* bias,
                                           unsigned char* A, int r) {
#pragma unroll
    for (int q = 0; q < kHid / 16; ++q) {
        float v[16];
        tmem_ld16(tmem_row + 16 * q, v);
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            uint4 u;
            unsigned* pu = reinterpret_cast<unsigned*>(&u);
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int c = 8 * h + 2 * j;
                pu[j] = pack_bf16(fmaxf(v[c] + bias[16 * q + c], 0.f),
                                  fmaxf(v[c + 1] + bias[16 * q + c + 1], 0.f));
            }
            *reinterpret_cast<uint4*>(A + umma_off(kTcRows, r, 16 * q + 8 * h)) = u;
        }
    }
}

__global__ void __launch_bounds__(kTcRows) mlp_infer_tc_kernel(const MlpW w,
                                                               const float* __restrict__ F,
                                                               long long n,
                                                               float* __restrict__ Y,
                                                               int32_t* status,
                                                               long long wait_ns) {
    extern __shared__ __align__(128) unsigned char tsm[];
    __shared__ __align__(8) unsigned long long bar;
    __shared__ unsigned tmem_slot;
    const int tid = threadIdx.x, warp = tid >> 5;
    unsigned char* A = tsm + kTcOffA;
    float* bias = reinterpret_cast<float*>(tsm + kTcOffB);
    stage_weights(tsm + kTcOffW1, w.W1, kHid, kHid, kIn, tid, kTcRows);
    stage_weights(tsm + kTcOffW2, w.W2, kHid, kHid, kHid, tid, kTcRows);
    stage_weights(tsm + kTcOffW3, w.W3, kHid, kHid, kHid, tid, kTcRows);
    stage_weights(tsm + kTcOffW4, w.W4, 2, kTcN4, kHid, tid, kTcRows);
    for (int i = tid; i < kHid; i += kTcRows) {
        bias[i] = __ldg(w.b1 + i);
        bias[kHid + i] = __ldg(w.b2 + i);
        bias[2 * kHid + i] = __ldg(w.b3 + i);
    }
    if (tid < 8) bias[3 * kHid + tid] = __ldg(w.b4 + tid);
    if (tid == 0) {
        htasync::bar_init(&bar, 1);
        htasync::bar_init_fence();
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     :: "r"(htasync::smem_addr(&tmem_slot)), "r"(kTcCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    htasync::fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const unsigned tmem = tmem_slot;
    const unsigned tmem_row = tmem + ((unsigned)(32 * warp) << 16);   // this warp's lanes
    const unsigned sA = htasync::smem_addr(A);
    const unsigned sW1 = htasync::smem_addr(tsm + kTcOffW1), sW2 = htasync::smem_addr(tsm + kTcOffW2),
                   sW3 = htasync::smem_addr(tsm + kTcOffW3), sW4 = htasync::smem_addr(tsm + kTcOffW4);
    const float* mean = w.mean;
    const float* istd = w.istd;
    const long long ntiles = (n + kTcRows - 1) / kTcRows;
    unsigned parity = 0;
    bool ok = true;
    // one layer: the MMAs over nk K steps, committed; every thread waits for them
    auto layer = [&](unsigned sB, int RB, int nk, int N) -> bool {
        htasync::fence_async_smem();   // this thread's A writes, seen by the tensor cores
        tc_fence_before();
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
            const unsigned idesc = umma_idesc(kTcRows, N);
            for (int s = 0; s < nk; ++s)
                umma_bf16(tmem, umma_desc(sA + s * (kTcRows * 32), kTcRows),
                          umma_desc(sB + s * (RB * 32), RB), idesc, s > 0 ? 1u : 0u);
            umma_commit(&bar);
        }
        const bool done = htasync::bar_wait(&bar, parity, wait_ns);
        parity ^= 1u;
        tc_fence_after();
        return !__syncthreads_or(!done);
    };
    for (long long tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
        const long long row = tile * kTcRows + tid;
        {   // layer-1 input: the standardised features of this thread's peak, BF16
            float x[kIn];
#pragma unroll
            for (int c = 0; c < kIn; c += 4) {
                const float4 f4 = row < n ? __ldg(reinterpret_cast<const float4*>(F + row * kIn + c))
                                          : make_float4(0.f, 0.f, 0.f, 0.f);
                x[c] = f4.x; x[c + 1] = f4.y; x[c + 2] = f4.z; x[c + 3] = f4.w;
            }
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                uint4 u;
                unsigned* pu = reinterpret_cast<unsigned*>(&u);
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const int c = 8 * h + 2 * j;
                    const float a0 = row < n ? (x[c] - __ldg(mean + c)) * __ldg(istd + c) : 0.f;
                    const float a1 = row < n ? (x[c + 1] - __ldg(mean + c + 1)) * __ldg(istd + c + 1)
                                             : 0.f;
                    pu[j] = pack_bf16(a0, a1);
                }
                *reinterpret_cast<uint4*>(A + umma_off(kTcRows, tid, 8 * h)) = u;
            }
        }
        if (!(ok = layer(sW1, kHid, 1, kHid))) break;
        hidden_out(tmem_row, bias, A, tid);
        if (!(ok = layer(sW2, kHid, kHid / 16, kHid))) break;
        hidden_out(tmem_row, bias + kHid, A, tid);
        if (!(ok = layer(sW3, kHid, kHid / 16, kHid))) break;
        hidden_out(tmem_row, bias + 2 * kHid, A, tid);
        if (!(ok = layer(sW4, kTcN4, kHid / 16, kTcN4))) break;
        {
            unsigned u0, u1;
            asm volatile("tcgen05.ld.sync.aligned.32x32b.x2.b32 {%0, %1}, [%2];"
                         : "=r"(u0), "=r"(u1) : "r"(tmem_row));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (row < n) {
                Y[row * 2] = __uint_as_float(u0) + bias[3 * kHid];
                Y[row * 2 + 1] = __uint_as_float(u1) + bias[3 * kHid + 1];
            }
        }
    }
    if (!ok && tid == 0) {
        // record the timeout, then give the MMAs in flight a bounded time to finish
        atomicExch(status, kStatusWaitTimeout);
        htasync::bar_wait(&bar, parity ^ 1u, wait_ns);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;"
                     :: "r"(tmem), "r"(kTcCols));
    }
}

// --------------------------------------------------------------- training ----
//
// C[M x N] (FP32, row stride N) = op(A) op(B): A element (m, k) at A[m sam + k sak], B
// element (k, n) at B[k sbk + n sbn], both BF16.  A CTA computes a 64 x 64 tile with four
// warps of 32 x 32 (2 x 4 mma tiles); K advances in slices of 16 staged in shared memory
// (zero-filled outside the matrices).  The same kernel serves the forward products
// (X W^T), the activation gradients (dZ W) and the weight gradients (dZ^T H, K = batch).

constexpr int kTM = 64, kTN = 64, kTK = 16, kPadK = 24;

__global__ void __launch_bounds__(128) gemm_bf16_kernel(
    const __nv_bfloat16* __restrict__ A, long long sam, long long sak,
    const __nv_bfloat16* __restrict__ B, long long sbk, long long sbn, float* __restrict__ C,
    int M, int N, int K) {
    __shared__ __align__(16) __nv_bfloat16 As[kTM][kPadK];
    __shared__ __align__(16) __nv_bfloat16 Bs[kTN][kPadK];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, t = lane & 3;
    const int m0 = blockIdx.y * kTM, n0 = blockIdx.x * kTN;
    const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
    float acc[2][4][4];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int e = 0; e < 4; ++e) acc[i][j][e] = 0.f;
    const __nv_bfloat16 zero = __float2bfloat16(0.f);
    for (int k0 = 0; k0 < K; k0 += kTK) {
        for (int e = tid; e < kTM * kTK; e += blockDim.x) {
            const int r = e / kTK, c = e % kTK;
            const int m = m0 + r, k = k0 + c;
            As[r][c] = (m < M && k < K) ? A[(long long)m * sam + (long long)k * sak] : zero;
            const int n = n0 + r;
            Bs[r][c] = (n < N && k < K) ? B[(long long)k * sbk + (long long)n * sbn] : zero;
        }
        __syncthreads();
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            unsigned a[4];
            const int r = wm + 16 * i + g;
            a[0] = *reinterpret_cast<const unsigned*>(&As[r][2 * t]);
            a[1] = *reinterpret_cast<const unsigned*>(&As[r + 8][2 * t]);
            a[2] = *reinterpret_cast<const unsigned*>(&As[r][2 * t + 8]);
            a[3] = *reinterpret_cast<const unsigned*>(&As[r + 8][2 * t + 8]);
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int nn = wn + 8 * j + g;
                const unsigned b0 = *reinterpret_cast<const unsigned*>(&Bs[nn][2 * t]);
                const unsigned b1 = *reinterpret_cast<const unsigned*>(&Bs[nn][2 * t + 8]);
                mma_bf16(acc[i][j], a, b0, b1);
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int r = m0 + wm + 16 * i + g, c = n0 + wn + 8 * j + 2 * t;
            if (r < M && c < N) C[(long long)r * N + c] = acc[i][j][0];
            if (r < M && c + 1 < N) C[(long long)r * N + c + 1] = acc[i][j][1];
            if (r + 8 < M && c < N) C[(long long)(r + 8) * N + c] = acc[i][j][2];
            if (r + 8 < M && c + 1 < N) C[(long long)(r + 8) * N + c + 1] = acc[i][j][3];
        }
}

// X = bf16((F - mean) * istd), [M x 16]
__global__ void standardise_kernel(const float* __restrict__ F, const float* __restrict__ mean,
                                   const float* __restrict__ istd, long long M,
                                   __nv_bfloat16* __restrict__ X) {
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= M * kIn) return;
    const int c = (int)(e % kIn);
    X[e] = __float2bfloat16((F[e] - mean[c]) * istd[c]);
}

// Z += b (in place); H = bf16(relu(Z)) when H is given
__global__ void bias_act_kernel(float* __restrict__ Z, const float* __restrict__ b, long long M,
                                int N, __nv_bfloat16* __restrict__ H) {
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= M * N) return;
    const float z = Z[e] + b[e % N];
    Z[e] = z;
    if (H) H[e] = __float2bfloat16(fmaxf(z, 0.f));
}

// Pinball loss of the two quantile outputs (tau 0.1 and 0.9) against the target; dY / M
// as BF16 [M x 16] (columns 2..15 zero) and FP32 [M x 2]; loss summed into *loss.
__global__ void pinball_kernel(const float* __restrict__ Y, const float* __restrict__ tgt,
                               long long M, __nv_bfloat16* __restrict__ dYb,
                               float* __restrict__ dYf, float* __restrict__ loss) {
    const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    float l = 0.f;
    if (r < M) {
        const float tau[2] = {0.1f, 0.9f};
        const float inv = 1.0f / (float)M;
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            const float d = tgt[r] - Y[r * 2 + q];
            l += d > 0.f ? tau[q] * d : (tau[q] - 1.f) * d;
            const float gq = (d > 0.f ? -tau[q] : 1.f - tau[q]) * inv;
            dYf[r * 2 + q] = gq;
            dYb[r * kIn + q] = __float2bfloat16(gq);
        }
#pragma unroll
        for (int c = 2; c < kIn; ++c) dYb[r * kIn + c] = __float2bfloat16(0.f);
    }
    for (int o = 16; o >= 1; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(loss, l / (float)M);
}

// dZ = dH * (Z > 0): FP32 in place and a BF16 copy
__global__ void relu_back_kernel(float* __restrict__ dH, const float* __restrict__ Z, long long M,
                                 int N, __nv_bfloat16* __restrict__ dZb) {
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= M * N) return;
    const float d = Z[e] > 0.f ? dH[e] : 0.f;
    dH[e] = d;
    dZb[e] = __float2bfloat16(d);
}

// db[n] = sum_m dZ[m][n] (one block per column, fixed reduction order)
__global__ void colsum_kernel(const float* __restrict__ dZ, long long M, int N,
                              float* __restrict__ db) {
    __shared__ float red[256];
    const int n = blockIdx.x;
    float s = 0.f;
    for (long long m = threadIdx.x; m < M; m += blockDim.x) s += dZ[m * N + n];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = blockDim.x / 2; o >= 1; o >>= 1) {
        if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) db[n] = red[0];
}

// Adam on the packed FP32 parameters; writes the BF16 weights and FP32 biases of `out`.
struct PackedModel {
    __nv_bfloat16* W[4];
    float* b[4];
};

__global__ void adam_kernel(float* __restrict__ p, const float* __restrict__ gr,
                            float* __restrict__ m, float* __restrict__ v, int n, float lr,
                            float b1t, float b2t, PackedModel out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float g = gr[i];
    const float mi = 0.9f * m[i] + 0.1f * g;
    const float vi = 0.999f * v[i] + 0.001f * g * g;
    m[i] = mi;
    v[i] = vi;
    const float mh = mi / (1.f - b1t), vh = vi / (1.f - b2t);
    const float pi = p[i] - lr * mh / (sqrtf(vh) + 1e-8f);
    p[i] = pi;
    // packed layout: W1 [64x16] W2 [64x64] W3 [64x64] W4 [8x64] b1 b2 b3 [64] b4 [8]
    const int off[9] = {0, 1024, 5120, 9216, 9728, 9792, 9856, 9920, 9928};
    for (int s = 0; s < 8; ++s) {
        if (i >= off[s] && i < off[s + 1]) {
            if (s < 4) out.W[s][i - off[s]] = __float2bfloat16(pi);
            else out.b[s - 4][i - off[s]] = pi;
        }
    }
}

}  // namespace

// ------------------------------------------------------------------ C ABI ----

namespace {

int check_model(const ht_bracket_model* m, const char* who) {
    if (!m || !m->W1 || !m->W2 || !m->W3 || !m->W4 || !m->b1 || !m->b2 || !m->b3 || !m->b4 ||
        !m->mean || !m->istd)
        return ht_fail(HT_ERR_INVALID, std::string(who) + ": NULL model array");
    return HT_OK;
}

MlpW mlp_of(const ht_bracket_model* m) {
    MlpW w;
    w.W1 = (const __nv_bfloat16*)m->W1; w.W2 = (const __nv_bfloat16*)m->W2;
    w.W3 = (const __nv_bfloat16*)m->W3; w.W4 = (const __nv_bfloat16*)m->W4;
    w.b1 = m->b1; w.b2 = m->b2; w.b3 = m->b3; w.b4 = m->b4;
    w.mean = m->mean; w.istd = m->istd;
    return w;
}

int launch_gemm(const __nv_bfloat16* A, long long sam, long long sak, const __nv_bfloat16* B,
                long long sbk, long long sbn, float* C, long long M, int N, long long K,
                cudaStream_t st) {
    if (M > 0x7fffffffLL || K > 0x7fffffffLL)
        return ht_fail(HT_ERR_CAPACITY, "bracket GEMM: dimension too large");
    dim3 grid((unsigned)((N + kTN - 1) / kTN), (unsigned)((M + kTM - 1) / kTM));
    gemm_bf16_kernel<<<grid, 128, 0, st>>>(A, sam, sak, B, sbk, sbn, C, (int)M, N, (int)K);
    HT_CUDA_TRY(cudaGetLastError(), "gemm_bf16_kernel launch");
    return HT_OK;
}

unsigned blocks_for(long long n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

extern "C" HT_API int ht_bracket_features(ht_ctx* ctx, const ht_peak_batch* b,
                                          const float* d_peak_delta, double alatt,
                                          float* d_feat, void* stream) {
    HT_RANGE("ht_bracket_features");
    if (!ctx || !b || !d_feat) return ht_fail(HT_ERR_INVALID, "ht_bracket_features: NULL argument");
    if (!ctx->bound) return ht_fail(HT_ERR_STATE, "ht_bracket_features: no tile bound (ht_fields_pack)");
    if (b->npeaks < 0) return ht_fail(HT_ERR_INVALID, "ht_bracket_features: npeaks < 0");
    if (!(alatt > 0.0)) return ht_fail(HT_ERR_INVALID, "ht_bracket_features: alatt must be > 0");
    if (b->npeaks == 0) return HT_OK;
    if (!b->pi || !b->pj || !b->pk || !b->Rf || !b->ir2min || !b->ZZon || !b->fcrit)
        return ht_fail(HT_ERR_INVALID, "ht_bracket_features: NULL peak array");
    HT_CUDA_TRY(cudaSetDevice(ctx->device), "cudaSetDevice");
    FeatArgs a;
    const ht_fields& f = ctx->fields;
    a.rec = ctx->d_rec; a.delta = f.delta;
    a.n1 = f.n1; a.n2 = f.n2; a.n3 = f.n3; a.s2 = (long long)f.n1 * f.n2;
    a.off = ctx->d_off; a.start = ctx->d_start; a.count = ctx->d_count; a.r2 = ctx->d_r2;
    a.rad = ctx->d_rad; a.nshells = ctx->nshells;
    a.pi = b->pi; a.pj = b->pj; a.pk = b->pk; a.Rf = b->Rf; a.ir2min = b->ir2min;
    a.ZZon = b->ZZon; a.fcrit = b->fcrit; a.peak_delta = d_peak_delta;
    a.npeaks = b->npeaks; a.alatt = alatt;
    features_kernel<<<blocks_for(b->npeaks, 256), 256, 0, (cudaStream_t)stream>>>(a, d_feat);
    HT_CUDA_TRY(cudaGetLastError(), "features_kernel launch");
    ctx->last_kernels = 1;
    return HT_OK;
}

extern "C" HT_API int ht_bracket_predict(ht_ctx* ctx, const ht_bracket_model* m,
                                         const float* d_feat, int64_t n, float* d_pred,
                                         void* stream) {
    HT_RANGE("ht_bracket_predict");
    if (!ctx || !d_feat || !d_pred) return ht_fail(HT_ERR_INVALID, "ht_bracket_predict: NULL argument");
    int rc = check_model(m, "ht_bracket_predict");
    if (rc != HT_OK) return rc;
    if (n < 0) return ht_fail(HT_ERR_INVALID, "ht_bracket_predict: n < 0");
    if (n == 0) return HT_OK;
    if (((uintptr_t)d_feat & 15u) != 0)
        return ht_fail(HT_ERR_INVALID, "ht_bracket_predict: d_feat must be 16-byte aligned");
    HT_CUDA_TRY(cudaSetDevice(ctx->device), "cudaSetDevice");
    // persistent CTAs of 128 peaks, four per SM (each holds 64 tensor-memory columns)
    const long long tiles = (n + kTcRows - 1) / kTcRows;
    const unsigned grid = (unsigned)std::min<long long>(tiles, 4LL * ctx->num_sms);
    mlp_infer_tc_kernel<<<grid, kTcRows, kTcSmem, (cudaStream_t)stream>>>(
        mlp_of(m), d_feat, n, d_pred, ht_status_word(ctx), ctx->wait_ns);
    HT_CUDA_TRY(cudaGetLastError(), "mlp_infer_tc_kernel launch");
    ctx->last_kernels = 1;
    return HT_OK;
}

extern "C" HT_API int ht_bracket_grad(ht_ctx* ctx, const ht_bracket_model* m,
                                      const float* d_feat, const float* d_target, int64_t n,
                                      float* d_grads, float* d_loss, void* stream) {
    HT_RANGE("ht_bracket_grad");
    if (!ctx || !d_feat || !d_target || !d_grads || !d_loss)
        return ht_fail(HT_ERR_INVALID, "ht_bracket_grad: NULL argument");
    int rc = check_model(m, "ht_bracket_grad");
    if (rc != HT_OK) return rc;
    if (n < 1 || n > (1LL << 24)) return ht_fail(HT_ERR_INVALID, "ht_bracket_grad: need 1 <= n <= 2^24");
    HT_CUDA_TRY(cudaSetDevice(ctx->device), "cudaSetDevice");
    cudaStream_t st = (cudaStream_t)stream;
    // workspace per row: X (16 bf16), Z1..Z3 (64 f32), H1..H3 (64 bf16), Y (2 f32),
    // dYb (16 bf16), dYf (2 f32), dH (64 f32), dZb (64 bf16)
    const size_t row = 16 * 2 + 3 * 64 * 4 + 3 * 64 * 2 + 8 + 16 * 2 + 8 + 64 * 4 + 64 * 2;
    rc = ht_grow(&ctx->d_mlp_ws, &ctx->mlp_ws_bytes, row * (size_t)n + 4096, "bracket training workspace");
    if (rc != HT_OK) return rc;
    char* w = (char*)ctx->d_mlp_ws;
    auto take = [&](size_t bytes) { char* p = w; w += (bytes + 255) / 256 * 256; return p; };
    __nv_bfloat16* X = (__nv_bfloat16*)take((size_t)n * 16 * 2);
    float* Z[3]; __nv_bfloat16* H[3];
    for (int l = 0; l < 3; ++l) { Z[l] = (float*)take((size_t)n * 64 * 4); H[l] = (__nv_bfloat16*)take((size_t)n * 64 * 2); }
    float* Y = (float*)take((size_t)n * 2 * 4);
    __nv_bfloat16* dYb = (__nv_bfloat16*)take((size_t)n * 16 * 2);
    float* dYf = (float*)take((size_t)n * 2 * 4);
    float* dH = (float*)take((size_t)n * 64 * 4);
    __nv_bfloat16* dZb = (__nv_bfloat16*)take((size_t)n * 64 * 2);
    const __nv_bfloat16* W[4] = {(const __nv_bfloat16*)m->W1, (const __nv_bfloat16*)m->W2,
                                 (const __nv_bfloat16*)m->W3, (const __nv_bfloat16*)m->W4};
    const float* bias[4] = {m->b1, m->b2, m->b3, m->b4};
    // gradient layout (FP32): dW1 [64x16] dW2 dW3 [64x64] dW4 [8x64] db1 db2 db3 [64] db4 [8]
    float* gW[4] = {d_grads, d_grads + 1024, d_grads + 5120, d_grads + 9216};
    float* gb[4] = {d_grads + 9728, d_grads + 9792, d_grads + 9856, d_grads + 9920};
    HT_CUDA_TRY(cudaMemsetAsync(d_grads, 0, 9928 * sizeof(float), st), "grad reset");
    HT_CUDA_TRY(cudaMemsetAsync(d_loss, 0, sizeof(float), st), "loss reset");
    const int T = 256;
    standardise_kernel<<<blocks_for(n * kIn, T), T, 0, st>>>(d_feat, m->mean, m->istd, n, X);
    HT_CUDA_TRY(cudaGetLastError(), "standardise_kernel launch");
    // forward: Z_l = H_{l-1} W_l^T + b_l, H_l = relu(Z_l)
    const __nv_bfloat16* in = X;
    int K = kIn;
    for (int l = 0; l < 3; ++l) {
        if ((rc = launch_gemm(in, K, 1, W[l], 1, K, Z[l], n, kHid, K, st)) != HT_OK) return rc;
        bias_act_kernel<<<blocks_for(n * kHid, T), T, 0, st>>>(Z[l], bias[l], n, kHid, H[l]);
        HT_CUDA_TRY(cudaGetLastError(), "bias_act_kernel launch");
        in = H[l];
        K = kHid;
    }
    if ((rc = launch_gemm(H[2], kHid, 1, W[3], 1, kHid, Y, n, 2, kHid, st)) != HT_OK) return rc;
    bias_act_kernel<<<blocks_for(n * 2, T), T, 0, st>>>(Y, bias[3], n, 2, nullptr);
    HT_CUDA_TRY(cudaGetLastError(), "bias_act_kernel launch");
    pinball_kernel<<<blocks_for(n, T), T, 0, st>>>(Y, d_target, n, dYb, dYf, d_loss);
    HT_CUDA_TRY(cudaGetLastError(), "pinball_kernel launch");
    // output layer: dW4 = dY^T H3 (rows 0..1), db4, dH3 = dY W4
    if ((rc = launch_gemm(dYb, 1, kIn, H[2], kHid, 1, gW[3], 2, kHid, n, st)) != HT_OK) return rc;
    colsum_kernel<<<2, 256, 0, st>>>(dYf, n, 2, gb[3]);
    HT_CUDA_TRY(cudaGetLastError(), "colsum_kernel launch");
    if ((rc = launch_gemm(dYb, kIn, 1, W[3], kHid, 1, dH, n, kHid, 2, st)) != HT_OK) return rc;
    for (int l = 2; l >= 0; --l) {
        relu_back_kernel<<<blocks_for(n * kHid, T), T, 0, st>>>(dH, Z[l], n, kHid, dZb);
        HT_CUDA_TRY(cudaGetLastError(), "relu_back_kernel launch");
        colsum_kernel<<<kHid, 256, 0, st>>>(dH, n, kHid, gb[l]);
        HT_CUDA_TRY(cudaGetLastError(), "colsum_kernel launch");
        const __nv_bfloat16* prev = l > 0 ? H[l - 1] : X;
        const int Kp = l > 0 ? kHid : kIn;
        // dW_l = dZ_l^T prev : (64 x Kp), K = n
        if ((rc = launch_gemm(dZb, 1, kHid, prev, Kp, 1, gW[l], kHid, Kp, n, st)) != HT_OK) return rc;
        if (l > 0) {
            // dH_{l-1} = dZ_l W_l : (n x 64), K = 64
            if ((rc = launch_gemm(dZb, kHid, 1, W[l], kHid, 1, dH, n, kHid, kHid, st)) != HT_OK)
                return rc;
        }
    }
    ctx->last_kernels = 0;
    return HT_OK;
}

extern "C" HT_API int ht_bracket_adam(ht_ctx* ctx, float* d_params, const float* d_grads,
                                      float* d_m, float* d_v, int32_t step, float lr,
                                      const ht_bracket_model* out, void* stream) {
    HT_RANGE("ht_bracket_adam");
    if (!ctx || !d_params || !d_grads || !d_m || !d_v)
        return ht_fail(HT_ERR_INVALID, "ht_bracket_adam: NULL argument");
    int rc = check_model(out, "ht_bracket_adam");
    if (rc != HT_OK) return rc;
    if (step < 1) return ht_fail(HT_ERR_INVALID, "ht_bracket_adam: step counts from 1");
    HT_CUDA_TRY(cudaSetDevice(ctx->device), "cudaSetDevice");
    PackedModel pm;
    pm.W[0] = (__nv_bfloat16*)out->W1; pm.W[1] = (__nv_bfloat16*)out->W2;
    pm.W[2] = (__nv_bfloat16*)out->W3; pm.W[3] = (__nv_bfloat16*)out->W4;
    pm.b[0] = out->b1; pm.b[1] = out->b2; pm.b[2] = out->b3; pm.b[3] = out->b4;
    const float b1t = powf(0.9f, (float)step), b2t = powf(0.999f, (float)step);
    adam_kernel<<<blocks_for(HT_BRACKET_NPARAMS, 256), 256, 0, (cudaStream_t)stream>>>(
        d_params, d_grads, d_m, d_v, HT_BRACKET_NPARAMS, lr, b1t, b2t, pm);
    HT_CUDA_TRY(cudaGetLastError(), "adam_kernel launch");
    ctx->last_kernels = 1;
    return HT_OK;
}
