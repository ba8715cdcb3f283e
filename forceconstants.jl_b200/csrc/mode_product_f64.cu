// FP64 mode product on the CUDA cores (DFMA), used only by the adjoint to form
// G = W ×₁ φᵀ ×₂ φᵀ ×₃ φᵀ in double precision (FCB_ADJOINT_FP64), so that the
// gradient is limited by the FP64 pair contraction and not by the rounding of G.
//
//     D[r,p] = Σ_a A[a + lda*r] * B[a + ldb*p],  D at (r % F) + F_pad*(r / F) + ldd*p
//
// 128×128 output tile per 256-thread CTA, 8-deep K slices double-buffered in
// shared memory (stored transposed, rows contiguous), an 8×8 register
// micro-tile per thread: thread (tr, tp) owns rows {4tr..4tr+3, 64+4tr..} and
// columns {4tp.., 64+4tp..}.  Per K step a warp reads 16 distinct 32-byte row
// groups of A and 2 of B (the rest are shared-memory broadcasts) for 2048 DFMA.
#include "fcb200_internal.cuh"

namespace fcb {
namespace {

constexpr int TM = 128, TN = 128, TK = 8, PAD = 2;

__global__ void __launch_bounds__(256) mode_product_f64_kernel(const double* __restrict__ A,
                                                               const double* __restrict__ B,
                                                               double* __restrict__ D, ModeProduct mp) {
    __shared__ __align__(16) double As[2][TK][TM + PAD];
    __shared__ __align__(16) double Bs[2][TK][TN + PAD];
    const int tid = threadIdx.x;
    const int tr = tid & 15, tp = tid >> 4;
    const int64_t r0 = (int64_t)blockIdx.x * TM;
    const int64_t p0 = (int64_t)blockIdx.y * TN;

    // Loader: each thread fetches 4 consecutive K values of one row of A and
    // of one column of B per slice (row lr, K offset lk).
    const int lk = (tid & 1) * 4, lr = tid >> 1;
    double ra[4], rb[4];
    auto fetch = [&](int64_t k0) {
        const int64_t r = r0 + lr, p = p0 + lr;
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int64_t k = k0 + lk + u;
            ra[u] = (r < mp.R && k < mp.K) ? A[k + mp.lda * r] : 0.0;
            rb[u] = (p < mp.M && k < mp.K) ? B[k + mp.ldb * p] : 0.0;
        }
    };
    auto stash = [&](int buf) {
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            As[buf][lk + u][lr] = ra[u];
            Bs[buf][lk + u][lr] = rb[u];
        }
    };

    double acc[8][8];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = 0.0;

    const int64_t nk = (mp.K + TK - 1) / TK;
    fetch(0);
    stash(0);
    __syncthreads();
    for (int64_t kt = 0; kt < nk; ++kt) {
        const int buf = (int)(kt & 1);
        if (kt + 1 < nk) fetch((kt + 1) * TK);
#pragma unroll
        for (int k = 0; k < TK; ++k) {
            const double2 a0 = *reinterpret_cast<const double2*>(&As[buf][k][4 * tr]);
            const double2 a1 = *reinterpret_cast<const double2*>(&As[buf][k][4 * tr + 2]);
            const double2 a2 = *reinterpret_cast<const double2*>(&As[buf][k][64 + 4 * tr]);
            const double2 a3 = *reinterpret_cast<const double2*>(&As[buf][k][64 + 4 * tr + 2]);
            const double2 b0 = *reinterpret_cast<const double2*>(&Bs[buf][k][4 * tp]);
            const double2 b1 = *reinterpret_cast<const double2*>(&Bs[buf][k][4 * tp + 2]);
            const double2 b2 = *reinterpret_cast<const double2*>(&Bs[buf][k][64 + 4 * tp]);
            const double2 b3 = *reinterpret_cast<const double2*>(&Bs[buf][k][64 + 4 * tp + 2]);
            const double a[8] = {a0.x, a0.y, a1.x, a1.y, a2.x, a2.y, a3.x, a3.y};
            const double b[8] = {b0.x, b0.y, b1.x, b1.y, b2.x, b2.y, b3.x, b3.y};
#pragma unroll
            for (int i = 0; i < 8; ++i)
#pragma unroll
                for (int j = 0; j < 8; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
        }
        if (kt + 1 < nk) stash(buf ^ 1);
        __syncthreads();
    }

#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const int64_t p = p0 + (j < 4 ? 4 * tp + j : 64 + 4 * tp + (j - 4));
        if (p >= mp.M) continue;
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const int64_t r = r0 + (i < 4 ? 4 * tr + i : 64 + 4 * tr + (i - 4));
            if (r < mp.R) D[(r % mp.F) + mp.F_pad * (r / mp.F) + mp.ldd * p] = acc[i][j];
        }
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
    mode_product_f64_kernel<<<grid, 256, 0, s>>>(A, B, D, mp);
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
