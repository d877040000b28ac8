// Small-case driver for the pencil smoothing kernels of the 1152^3 tile (pz_kernel<36>,
// py_kernel<36>, px_kernel<18>): the same kernels and launch shapes as ht_smooth_pencil, on
// a reduced number of kx planes (Z, Y passes) and rows (X pass), so that an ncu capture with
// many passes stays at ~2 GB of device memory.  Built by `python huntian.jl_b200/build.py
// --smallcase`; usage: pencil_smallcase [kx_planes = 64] [reps = 3] [rows = 64]: the Y pass
// writes `rows` y rows of every z plane and the X pass transforms `rows` z planes (rows =
// 1026 gives the full-size Y and X passes, ~12 GB).  Prints the CUDA-event time of each
// kernel; inputs are zeros (the timing does not depend on the values).
#include <cstdio>
#include <cstdlib>

#include "csrc/ht_smooth.cu"   // the kernels live in that translation unit

#define CK(call)                                                                          \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess) {                                                          \
            printf("CUDA error %s at %s:%d\n", cudaGetErrorString(e_), __FILE__, __LINE__); \
            return 2;                                                                     \
        }                                                                                 \
    } while (0)

int main(int argc, char** argv) {
    const int nks = argc > 1 ? atoi(argv[1]) : 64;   // kx planes of the Z / Y passes
    const int reps = argc > 2 ? atoi(argv[2]) : 3;
    const int nrow = argc > 3 ? atoi(argv[3]) : 64;
    constexpr int T = 36, n = 32 * T, TH = T / 2;
    if (nks < 8 || nks > n / 2 + 1) { printf("kx_planes must be in [8, %d]\n", n / 2 + 1); return 1; }
    if (nrow < 1 || nrow > n - 126) { printf("rows must be in [1, %d]\n", n - 126); return 1; }
    ht_ctx ctx;
    ctx.device = 0;
    CK(cudaDeviceGetAttribute(&ctx.num_sms, cudaDevAttrMultiProcessorCount, 0));
    CK(cudaMalloc(&ctx.d_stats, 256));
    CK(cudaMemset(ctx.d_stats, 0, 256));
    if (fused_tables(&ctx, n) != HT_OK || scaled_window_table(&ctx, n, n * 1.46, 5.0, 1, 0) != HT_OK) {
        printf("set-up failed: %s\n", ht_last_error());
        return 1;
    }
    // the bench's region: rows (z, y) in [63, 1089); the Y pass writes nrow y rows, the X
    // pass transforms nrow z planes of R rows
    const int lo = 63, R = n - 2 * lo, ry = nrow, zx = nrow;
    const int nkp = pencil_row_pitch(n);              // padded C row
    const long long rows = (long long)zx * R;
    const size_t pb = (size_t)n * nks * n * sizeof(float2);
    const size_t bb = (size_t)nks * R * n * sizeof(float2);
    const size_t cb = (size_t)rows * nkp * sizeof(float2);
    const size_t ob = (size_t)zx * n * n * sizeof(float);
    float2 *P, *B, *C, *out;
    CK(cudaMalloc(&P, pb));
    CK(cudaMalloc(&B, bb));
    CK(cudaMalloc(&C, cb));
    CK(cudaMalloc(&out, ob));
    CK(cudaMemset(P, 0, pb));
    CK(cudaMemset(C, 0, cb));
    const size_t smz = pencil_smem_yz<T, PencilZ>(), smy = pencil_smem_yz<T, PencilY>(),
                 smx = pencil_smem_x<TH>();
    CK(cudaFuncSetAttribute(pz_kernel<T, PencilZ>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smz));
    CK(cudaFuncSetAttribute(py_kernel<T, PencilY>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smy));
    CK(cudaFuncSetAttribute(px_kernel<TH>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smx));
    int bz = 0, by = 0, bx = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bz, pz_kernel<T, PencilZ>, PencilZ::threads, smz));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&by, py_kernel<T, PencilY>, PencilY::threads, smy));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bx, px_kernel<TH>, 256, smx));
    const FusedTw tw = fused_tw(&ctx, n);
    int32_t* status = ht_status_word(&ctx);
    const long long sms = ctx.num_sms;
    const unsigned gz = (unsigned)std::min((long long)nks * (n / PencilZ::cols), sms * bz);
    const unsigned gy = (unsigned)std::min((long long)R * ((nks + PencilY::cols - 1) / PencilY::cols), sms * by);
    const unsigned gx = (unsigned)std::min((rows + 7) / 8, sms * bx);
    printf("kx planes %d: blocks per SM z %d y %d x %d, grids %u %u %u\n", nks, bz, by, bx, gz, gy, gx);
    cudaEvent_t e[4];
    for (auto& x : e) CK(cudaEventCreate(&x));
    for (int r = 0; r < reps; ++r) {
        CK(cudaEventRecord(e[0]));
        pz_kernel<T, PencilZ><<<gz, PencilZ::threads, smz>>>(P, B, nks, lo, R, (const float*)ctx.d_win, tw.lmL, tw.w32, status);
        CK(cudaEventRecord(e[1]));
        py_kernel<T, PencilY><<<gy, PencilY::threads, smy>>>(B, C, nks, nkp, R, lo, ry, tw.lmL, tw.w32, status);
        CK(cudaEventRecord(e[2]));
        px_kernel<TH><<<gx, 256, smx>>>(C, out, nkp, 0, 0, R, rows, tw.nat, tw.lmM, tw.w32, status);
        CK(cudaEventRecord(e[3]));
        CK(cudaDeviceSynchronize());
        float a, b, c;
        CK(cudaEventElapsedTime(&a, e[0], e[1]));
        CK(cudaEventElapsedTime(&b, e[1], e[2]));
        CK(cudaEventElapsedTime(&c, e[2], e[3]));
        printf("rep %d: pz %.3f ms  py %.3f ms  px %.3f ms (%lld rows)\n", r, a, b, c, rows);
    }
    int st = 0;
    CK(cudaMemcpy(&st, status, sizeof st, cudaMemcpyDeviceToHost));
    printf("status %d\n", st);
    return st == 0 ? 0 : 3;
}
