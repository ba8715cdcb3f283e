// Plain FP32 mode product on the CUDA cores (FFMA) — the "FP32 GPU form" of
// mcc3 (src/mcc.jl:29-51 in Float32), used for FCB_MCC3_FP32.
//
//     D[r,p] = Σ_a A[a + lda*r] * B[a + ldb*p]
//
// 128×128 output tile per 256-thread CTA, 16-deep K slices double-buffered in
// shared memory (stored transposed so the inner loop reads broadcast-friendly
// float4 rows), an 8×8 register micro-tile per thread, accumulated as column
// pairs by packed f32x2 FMAs (half the FMA instructions).  Thread (tr, tp) owns
// rows {4tr..4tr+3, 64+4tr..} and columns {4tp.., 64+4tp..}; lanes of a warp
// vary along r, the contiguous output index, so each float4 store of a warp is
// a 256-byte contiguous segment.
#include "fcb200_internal.cuh"

namespace fcb {
namespace {

constexpr int TM = 128, TN = 128, TK = 16, PAD = 4;

__device__ __forceinline__ float2 ffma2(float2 a, float2 b, float2 c) {
    uint64_t d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;"
        : "=l"(d)
        : "l"(*reinterpret_cast<const uint64_t*>(&a)), "l"(*reinterpret_cast<const uint64_t*>(&b)),
          "l"(*reinterpret_cast<const uint64_t*>(&c)));
    return *reinterpret_cast<const float2*>(&d);
}

__device__ __forceinline__ float accv(const float2 (&acc)[8][4], int i, int j) {
    return (j & 1) ? acc[i][j >> 1].y : acc[i][j >> 1].x;
}

template <bool VEC>
__global__ void __launch_bounds__(256, 2) mode_product_f32_kernel(const float* __restrict__ A,
                                                               const float* __restrict__ B,
                                                               float* __restrict__ D, ModeProduct mp) {
    __shared__ __align__(16) float As[2][TK][TM + PAD];
    __shared__ __align__(16) float Bs[2][TK][TN + PAD];
    const int tid = threadIdx.x;
    const int tr = tid & 15, tp = tid >> 4;
    const int64_t r0 = (int64_t)blockIdx.x * TM;
    const int64_t p0 = (int64_t)blockIdx.y * TN;

    // Loader mapping: each thread fetches 2 float4 of A and 2 of B per slice
    // (rows lr and lr+64, K offset lk..lk+3).
    const int lk = (tid & 3) * 4, lr = tid >> 2;
    float4 ra[2], rb[2];

    auto fetch = [&](int64_t k0) {
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int64_t r = r0 + lr + 64 * h, p = p0 + lr + 64 * h, k = k0 + lk;
            if (VEC) {
                ra[h] = (r < mp.R && k < mp.K) ? *reinterpret_cast<const float4*>(A + k + mp.lda * r)
                                               : make_float4(0.f, 0.f, 0.f, 0.f);
                rb[h] = (p < mp.M && k < mp.K) ? *reinterpret_cast<const float4*>(B + k + mp.ldb * p)
                                               : make_float4(0.f, 0.f, 0.f, 0.f);
            } else {
                float a[4], b[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    a[u] = (r < mp.R && k + u < mp.K) ? A[k + u + mp.lda * r] : 0.f;
                    b[u] = (p < mp.M && k + u < mp.K) ? B[k + u + mp.ldb * p] : 0.f;
                }
                ra[h] = make_float4(a[0], a[1], a[2], a[3]);
                rb[h] = make_float4(b[0], b[1], b[2], b[3]);
            }
        }
    };
    auto stash = [&](int buf) {
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            As[buf][lk + 0][lr + 64 * h] = ra[h].x;
            As[buf][lk + 1][lr + 64 * h] = ra[h].y;
            As[buf][lk + 2][lr + 64 * h] = ra[h].z;
            As[buf][lk + 3][lr + 64 * h] = ra[h].w;
            Bs[buf][lk + 0][lr + 64 * h] = rb[h].x;
            Bs[buf][lk + 1][lr + 64 * h] = rb[h].y;
            Bs[buf][lk + 2][lr + 64 * h] = rb[h].z;
            Bs[buf][lk + 3][lr + 64 * h] = rb[h].w;
        }
    };

    // acc[i][jp] holds columns (2jp, 2jp+1) of row i: packed f32x2 FMAs, each
    // half rounded as fmaf rounds it
    float2 acc[8][4];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = make_float2(0.f, 0.f);

    const int64_t nk = (mp.K + TK - 1) / TK;
    fetch(0);
    stash(0);
    __syncthreads();
    for (int64_t kt = 0; kt < nk; ++kt) {
        const int buf = (int)(kt & 1);
        if (kt + 1 < nk) fetch((kt + 1) * TK);
#pragma unroll
        for (int k = 0; k < TK; ++k) {
            const float4 a0 = *reinterpret_cast<const float4*>(&As[buf][k][4 * tr]);
            const float4 a1 = *reinterpret_cast<const float4*>(&As[buf][k][64 + 4 * tr]);
            const float4 b0 = *reinterpret_cast<const float4*>(&Bs[buf][k][4 * tp]);
            const float4 b1 = *reinterpret_cast<const float4*>(&Bs[buf][k][64 + 4 * tp]);
            const float a[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
            const float2 b[4] = {make_float2(b0.x, b0.y), make_float2(b0.z, b0.w), make_float2(b1.x, b1.y),
                                 make_float2(b1.z, b1.w)};
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                const float2 ai = make_float2(a[i], a[i]);
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = ffma2(ai, b[j], acc[i][j]);
            }
        }
        if (kt + 1 < nk) stash(buf ^ 1);
        __syncthreads();
    }

#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const int64_t p = p0 + (j < 4 ? 4 * tp + j : 64 + 4 * tp + (j - 4));
        if (p >= mp.M) continue;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int64_t rb0 = r0 + 64 * h + 4 * tr;
            if (VEC && rb0 + 3 < mp.R) {
                const int64_t off = (rb0 % mp.F) + mp.F_pad * (rb0 / mp.F) + mp.ldd * p;
                *reinterpret_cast<float4*>(D + off) = make_float4(accv(acc, 4 * h + 0, j), accv(acc, 4 * h + 1, j),
                                                                  accv(acc, 4 * h + 2, j), accv(acc, 4 * h + 3, j));
            } else {
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int64_t r = rb0 + u;
                    if (r < mp.R) D[(r % mp.F) + mp.F_pad * (r / mp.F) + mp.ldd * p] = accv(acc, 4 * h + u, j);
                }
            }
        }
    }
}

}  // namespace

int mode_product_f32(const float* A, const float* B, float* D, const ModeProduct& mp, cudaStream_t s) {
    if (mp.R <= 0 || mp.M <= 0) return FCB_OK;
    const bool vec = (mp.lda % 4 == 0) && (mp.ldb % 4 == 0) && (mp.K % 4 == 0) && (mp.F % 4 == 0) &&
                     (mp.F_pad % 4 == 0) && (mp.ldd % 4 == 0) && ((uintptr_t)A % 16 == 0) &&
                     ((uintptr_t)B % 16 == 0) && ((uintptr_t)D % 16 == 0);
    dim3 grid((unsigned)((mp.R + TM - 1) / TM), (unsigned)((mp.M + TN - 1) / TN));
    if (grid.y > 65535) return set_error(FCB_ERR_ARG, "mode product: too many modes");
    if (vec)
        mode_product_f32_kernel<true><<<grid, 256, 0, s>>>(A, B, D, mp);
    else
        mode_product_f32_kernel<false><<<grid, 256, 0, s>>>(A, B, D, mp);
    FCB_CUDA(cudaGetLastError());
    return FCB_OK;
}

}  // namespace fcb
