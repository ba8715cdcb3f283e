// FP64 mode product on the FP64 tensor cores (DMMA, mma.sync m16n8k4 .f64),
// used only by the adjoint to form G = W ×₁ φᵀ ×₂ φᵀ ×₃ φᵀ in double
// precision (FCB_ADJOINT_FP64), so that the gradient is limited by the FP64
// pair contraction and not by the rounding of G.
//
//     D[r,p] = Σ_a A[a + lda*r] * B[a + ldb*p],  D at (r % F) + F_pad*(r / F) + ldd*p
//
// 128×128 output tile per 256-thread CTA; 8 warps as 4 (rows) × 2 (columns),
// a warp tile of 32 rows × 64 columns = 2 × 8 m16n8 accumulators (64 doubles
// per thread).  16-deep K slices are fetched into registers while the
// previous slice is multiplied, and stored transposed in (dynamic, 68 KB)
// shared memory ([k][row], rows padded by 8 doubles so that the four k rows of
// a fragment load fall in different bank halves).  Fragment layout of m16n8k4 .f64
// (g = lane / 4, t = lane % 4): A a0 (row g, k t), a1 (row g+8, k t);
// B b0 (k t, column g); C c0,c1 (row g, columns 2t, 2t+1), c2,c3 (row g+8).
#include "fcb200_internal.cuh"

namespace fcb {
namespace {

constexpr int TM = 128, TN = 128, TK = 16, PAD = 8;

__device__ __forceinline__ void dmma(double (&c)[4], double a0, double a1, double b0) {
    asm volatile("mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0, %1, %2, %3}, {%4, %5}, {%6}, "
                 "{%0, %1, %2, %3};"
                 : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
                 : "d"(a0), "d"(a1), "d"(b0));
}

__global__ void __launch_bounds__(256) mode_product_f64_kernel(const double* __restrict__ A,
                                                               const double* __restrict__ B,
                                                               double* __restrict__ D, ModeProduct mp) {
    extern __shared__ __align__(16) double smem_f64[];
    auto As = reinterpret_cast<double (*)[TK][TM + PAD]>(smem_f64);                     // [2][TK][TM + PAD]
    auto Bs = reinterpret_cast<double (*)[TK][TN + PAD]>(smem_f64 + 2 * TK * (TM + PAD));  // [2][TK][TN + PAD]
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int g = lane >> 2, t = lane & 3;
    const int wr = (warp & 3) * 32, wp = (warp >> 2) * 64;  // warp tile origin in the CTA tile
    const int64_t r0 = (int64_t)blockIdx.x * TM;
    const int64_t p0 = (int64_t)blockIdx.y * TN;

    // Loader: each thread fetches 8 consecutive K values of one row of A and
    // of one column of B per slice (row lr, K offset lk).
    const int lk = (tid & 1) * 8, lr = tid >> 1;
    double ra[8], rb[8];
    auto fetch = [&](int64_t k0) {
        const int64_t r = r0 + lr, p = p0 + lr;
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int64_t k = k0 + lk + u;
            ra[u] = (r < mp.R && k < mp.K) ? A[k + mp.lda * r] : 0.0;
            rb[u] = (p < mp.M && k < mp.K) ? B[k + mp.ldb * p] : 0.0;
        }
    };
    auto stash = [&](int buf) {
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            As[buf][lk + u][lr] = ra[u];
            Bs[buf][lk + u][lr] = rb[u];
        }
    };

    double acc[2][8][4];
#pragma unroll
    for (int mi = 0; mi < 2; ++mi)
#pragma unroll
        for (int ni = 0; ni < 8; ++ni)
#pragma unroll
            for (int e = 0; e < 4; ++e) acc[mi][ni][e] = 0.0;

    const int64_t nk = (mp.K + TK - 1) / TK;
    fetch(0);
    stash(0);
    __syncthreads();
    for (int64_t kt = 0; kt < nk; ++kt) {
        const int buf = (int)(kt & 1);
        if (kt + 1 < nk) fetch((kt + 1) * TK);
#pragma unroll
        for (int k4 = 0; k4 < TK; k4 += 4) {
            double a[2][2], b[8];
#pragma unroll
            for (int mi = 0; mi < 2; ++mi) {
                a[mi][0] = As[buf][k4 + t][wr + 16 * mi + g];
                a[mi][1] = As[buf][k4 + t][wr + 16 * mi + g + 8];
            }
#pragma unroll
            for (int ni = 0; ni < 8; ++ni) b[ni] = Bs[buf][k4 + t][wp + 8 * ni + g];
#pragma unroll
            for (int mi = 0; mi < 2; ++mi)
#pragma unroll
                for (int ni = 0; ni < 8; ++ni) dmma(acc[mi][ni], a[mi][0], a[mi][1], b[ni]);
        }
        if (kt + 1 < nk) stash(buf ^ 1);
        __syncthreads();
    }

#pragma unroll
    for (int mi = 0; mi < 2; ++mi)
#pragma unroll
        for (int ni = 0; ni < 8; ++ni)
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int64_t r = r0 + wr + 16 * mi + g + (e >= 2 ? 8 : 0);
                const int64_t p = p0 + wp + 8 * ni + 2 * t + (e & 1);
                if (r < mp.R && p < mp.M) D[(r % mp.F) + mp.F_pad * (r / mp.F) + mp.ldd * p] = acc[mi][ni][e];
            }
}

__global__ void widen_kernel(const float* __restrict__ src, double* __restrict__ dst, int64_t count) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x)
        dst[i] = (double)src[i];
}

}  // namespace

int mode_product_f64(const double* A, const double* B, double* D, const ModeProduct& mp, cudaStream_t s) {
    if (mp.R <= 0 || mp.M <= 0) return FCB_OK;
    dim3 grid((unsigned)((mp.R + TM - 1) / TM), (unsigned)((mp.M + TN - 1) / TN));
    if (grid.y > 65535) return set_error(FCB_ERR_ARG, "mode product: too many modes");
    constexpr int smem = (int)sizeof(double) * 2 * TK * (TM + PAD + TN + PAD);
    // a per-device attribute of the function: set on every launch, since
    // handles on several devices may share this process
    FCB_CUDA(cudaFuncSetAttribute(mode_product_f64_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    mode_product_f64_kernel<<<grid, 256, smem, s>>>(A, B, D, mp);
    FCB_CUDA(cudaGetLastError());
    return FCB_OK;
}

int widen_f32_to_f64(const float* src, double* dst, int64_t count, cudaStream_t s) {
    if (count <= 0) return FCB_OK;
    const int64_t blocks = (count + 255) / 256;
    widen_kernel<<<(unsigned)(blocks < 4096 ? blocks : 4096), 256, 0, s>>>(src, dst, count);
    FCB_CUDA(cudaGetLastError());
    return FCB_OK;
}

}  // namespace fcb
