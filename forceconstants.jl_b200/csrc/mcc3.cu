// mcc3 pipeline: three mode products with rotating index order.
//
//   P1  U1[j,k,p] = Σ_i Ψ[i,j,k]  φ[i,n_lo+p]     rows (j,k),  R = n²
//   P2  U2[k,p,q] = Σ_j U1[j,k,p] φ[j,m_lo+q]     rows (k,p),  R = n·Mn
//   P3  K3[p,q,s] = Σ_k U2[k,p,q] φ[k,l_lo+s]     rows (p,q),  R = Mn·Mm
//
// which is src/mcc.jl:29-51 (K1[n,j,k], K2[n,k,m], K1[n,m,l]) with each
// product's output written in exactly the layout the next product reads as
// its K-major operand.  For the split precisions every intermediate is stored
// as hi/lo planes with the leading dimension padded to 16 bytes (TMA rule), so
// the epilogue of P1/P2 emits the next operand directly and no conversion pass
// runs between products.
#include "fcb200_internal.cuh"

namespace fcb {
namespace {

// FP32 matrix (rows × cols, element (c,r) at src[c + ld_src*r]) → hi/lo planes
// with leading dimension ld_dst.  Padding columns are left untouched (the
// tensor maps never read them).
__global__ void split_kernel(const float* __restrict__ src, int64_t rows, int64_t cols, int64_t ld_src,
                             void* __restrict__ hi, void* __restrict__ lo, int64_t ld_dst, int kind) {
    const int64_t total = rows * cols;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = t / cols, c = t - r * cols;
        const float v = src[c + ld_src * r];
        const int64_t o = c + ld_dst * r;
        if (kind == 1) {
            const __nv_bfloat16 h = __float2bfloat16_rn(v);
            static_cast<__nv_bfloat16*>(hi)[o] = h;
            static_cast<__nv_bfloat16*>(lo)[o] = __float2bfloat16_rn(v - __bfloat162float(h));
        } else {
            uint32_t hb;
            asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(hb) : "f"(v));
            const float h = __uint_as_float(hb);
            static_cast<float*>(hi)[o] = h;
            static_cast<float*>(lo)[o] = v - h;
        }
    }
}

// One CTA per (q, s), q <= s: the run K3[0..q, q, s] (contiguous in the full
// layout) to packed[s(s+1)(s+2)/6 + q(q+1)/2 + p].
__global__ void pack_k3_kernel(const float* __restrict__ full, int64_t M, float* __restrict__ packed) {
    const int64_t q = blockIdx.x, s = blockIdx.y;
    if (q > s) return;
    const int64_t base = s * (s + 1) * (s + 2) / 6 + q * (q + 1) / 2;
    const float* src = full + M * (q + M * s);
    for (int64_t p = threadIdx.x; p <= q; p += blockDim.x) packed[base + p] = src[p];
}

}  // namespace

int pack_k3_launch(const float* full, int64_t M, float* packed, cudaStream_t s) {
    if (M <= 0) return FCB_OK;
    if (M > 65535) return set_error(FCB_ERR_ARG, "packed K3: too many modes");
    pack_k3_kernel<<<dim3((unsigned)M, (unsigned)M), 128, 0, s>>>(full, M, packed);
    FCB_CUDA(cudaGetLastError());
    return FCB_OK;
}

int split_operand(const float* src, int64_t rows, int64_t cols, int64_t ld_src, void* hi, void* lo,
                  int64_t ld_dst, int kind, cudaStream_t s) {
    const int64_t total = rows * cols;
    if (total <= 0) return FCB_OK;
    int64_t blocks = (total + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    split_kernel<<<(unsigned)blocks, 256, 0, s>>>(src, rows, cols, ld_src, hi, lo, ld_dst, kind);
    FCB_CUDA(cudaGetLastError());
    return FCB_OK;
}

}  // namespace fcb
