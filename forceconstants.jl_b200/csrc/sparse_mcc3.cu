// Block-sparse first mode product of the LJ snapshot path.
//
// mcc3 (src/mcc.jl:29-51) contracts Ψ with φ along each index in turn; the
// first product is
//     U1[j,k,p] = Σ_i Ψ[i,j,k] φ[i,p].
// The assembled LJ Ψ is block sparse: for k in atom K every non-zero Ψ[i,j,k]
// has i and j in nbr(K), the atoms within the cutoff of K and K itself (for j
// outside K only i ∈ atom(j) ∪ K contribute; for j inside K all of nbr(K) — the
// acoustic-sum-rule column).  So U1[j,k,p] vanishes unless j ∈ nbr(K) and each
// non-zero is a short sum: 6 terms, or 3·|nbr(K)| for the three self columns.
// This kernel computes them in FP32 on CUDA cores from per-atom coefficient
// tables (the FP32-rounded mass-weighted Ψ entries, lj_sparse_coefs) and writes
// U1 directly as the split operand of the second mode product, in the dense
// layout j + n_pad·(k + n·p): every column is written in full, zeros included,
// with coalesced stores.  The tensor-core products P2 and P3 are unchanged.
// Work: 2·n·M·(3·6|nbr| + 9|nbr|)/3 flops instead of 2n³M, and no split Ψ
// operand to write or read (4n³ bytes each way).
#include "fcb200_internal.cuh"

namespace fcb {
namespace {

constexpr int PC = 64;    // modes per CTA
constexpr int PSUB = 16;  // modes per work item
constexpr int CJ = 8;     // rows j per chunk (16 bytes of a BF16 plane)

struct SparseP1Args {
    int N, n, cap, M, mode_lo;
    int64_t np;
    const int* nb;
    const int* count;
    const int* self_slot;
    const float* coef;
    const float* phi;
    void* u1_hi;
    void* u1_lo;
};

// Split 8 consecutive values into the hi/lo planes at element offset `off`
// (16-byte aligned); TF32 planes are 32 bytes, the second half written only
// when it lies inside the padded column (`tail` false).
template <int KIND>
__device__ __forceinline__ void store_chunk8(void* hi, void* lo, int64_t off, const float (&v)[CJ], bool tail) {
    if constexpr (KIND == 1) {
        uint32_t h[4], l[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const __nv_bfloat162 hb = __floats2bfloat162_rn(v[2 * i], v[2 * i + 1]);
            const __nv_bfloat162 lb =
                __floats2bfloat162_rn(v[2 * i] - __low2float(hb), v[2 * i + 1] - __high2float(hb));
            h[i] = *reinterpret_cast<const uint32_t*>(&hb);
            l[i] = *reinterpret_cast<const uint32_t*>(&lb);
        }
        *reinterpret_cast<uint4*>(static_cast<__nv_bfloat16*>(hi) + off) = make_uint4(h[0], h[1], h[2], h[3]);
        *reinterpret_cast<uint4*>(static_cast<__nv_bfloat16*>(lo) + off) = make_uint4(l[0], l[1], l[2], l[3]);
    } else {
        float h[CJ], l[CJ];
#pragma unroll
        for (int i = 0; i < CJ; ++i) {
            uint32_t b;
            asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(b) : "f"(v[i]));
            h[i] = __uint_as_float(b);
            l[i] = v[i] - h[i];
        }
        float* ph = static_cast<float*>(hi) + off;
        float* pl = static_cast<float*>(lo) + off;
        *reinterpret_cast<float4*>(ph) = make_float4(h[0], h[1], h[2], h[3]);
        *reinterpret_cast<float4*>(pl) = make_float4(l[0], l[1], l[2], l[3]);
        if (!tail) {
            *reinterpret_cast<float4*>(ph + 4) = make_float4(h[4], h[5], h[6], h[7]);
            *reinterpret_cast<float4*>(pl + 4) = make_float4(l[4], l[5], l[6], l[7]);
        }
    }
}

// One work item: rows j0 .. j0+7 of the columns (3K+kc, pp0 .. pp0+npp-1).
// Row j of atom A = j/3 in slot sl of K's list is
//   Σ_t c[t]·φ[3A+t, p] + Σ_t c[3+t]·φ[3K+t, p]      (A ≠ K),
//   the self-column sum                               (A = K),
//   0                                                 (A outside the list).
__device__ __forceinline__ void chunk_setup(const SparseP1Args& a, const float* cp, const int* slot_of, int L, int ss,
                                            int j0, int kc, float (&c)[CJ][6], int (&ro)[CJ]) {
#pragma unroll
    for (int e = 0; e < CJ; ++e) {
        const int j = j0 + e;
        const int A = j / 3, jc = j - 3 * A;
        const int sl = (j < a.n) ? slot_of[A] : -1;
        const bool pair = sl >= 0 && sl != ss;
#pragma unroll
        for (int t = 0; t < 6; ++t) c[e][t] = pair ? cp[(kc * 6 + t) * L + 3 * sl + jc] : 0.f;
        ro[e] = 3 * (sl >= 0 ? sl : 0) * (PC + 1);
    }
}

// One CTA per (atom K, PC modes): the 3·PC columns U1[:, 3K+kc, p].  Shared
// memory: the φ rows of K's neighbour degrees of freedom for the CTA's modes
// (row stride PC+1), the atom's coefficient tables, the 9·PC self-column sums,
// the slot of every atom in K's list (-1 outside) and the column chunks in
// work order (chunks touching K's neighbourhood first, so that warps stay
// uniform).
template <int KIND>
__global__ void __launch_bounds__(256) sparse_p1_kernel(SparseP1Args a) {
    extern __shared__ float sm[];
    __shared__ int n_live;
    const int K = blockIdx.y, p0 = blockIdx.x * PC;
    const int L = 3 * a.cap;
    const int cnt = a.count[K], ss = a.self_slot[K];
    const int nchunks = (a.n + CJ - 1) / CJ;
    float* phis = sm;                       // [L][PC+1]
    float* cp = phis + L * (PC + 1);        // pair part [3][6][L], then self part [3][3][L]
    float* cs = cp + 18 * L;
    float* selfres = cp + 27 * L;           // [9][PC]
    int* slot_of = reinterpret_cast<int*>(selfres + 9 * PC);  // [N]
    int* order = slot_of + a.N;                                // [nchunks]
    const int* nbK = a.nb + (int64_t)K * a.N;
    for (int J = threadIdx.x; J < a.N; J += blockDim.x) slot_of[J] = -1;
    for (int il = threadIdx.x; il < L; il += blockDim.x) {
        const int sl = il / 3;
        const bool live = sl < cnt;
        const int64_t src = live ? (int64_t)(3 * nbK[sl] + il % 3) + (int64_t)a.n * (a.mode_lo + p0) : 0;
#pragma unroll 8
        for (int pp = 0; pp < PC; ++pp)
            phis[il * (PC + 1) + pp] = (live && p0 + pp < a.M) ? a.phi[src + (int64_t)a.n * pp] : 0.f;
    }
    {
        const float4* cg = reinterpret_cast<const float4*>(a.coef + (int64_t)K * 27 * L);
        float4* c4 = reinterpret_cast<float4*>(cp);
        for (int e = threadIdx.x; e < 27 * L / 4; e += blockDim.x) c4[e] = cg[e];
    }
    __syncthreads();
    for (int sl = threadIdx.x; sl < cnt; sl += blockDim.x) slot_of[nbK[sl]] = sl;
    __syncthreads();

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (warp == 0) {
        int base = 0;
        for (int pass = 0; pass < 2; ++pass) {
            for (int c0 = 0; c0 < nchunks; c0 += 32) {
                const int c = c0 + lane;
                bool nz = false;
                if (c < nchunks) {
                    const int Alo = (c * CJ) / 3, Ahi = (c * CJ + CJ - 1) / 3;
                    for (int A = Alo; A <= Ahi && A < a.N; ++A) nz |= slot_of[A] >= 0;
                }
                const bool want = c < nchunks && (pass == 0 ? nz : !nz);
                const unsigned m = __ballot_sync(0xffffffffu, want);
                if (want) order[base + __popc(m & ((1u << lane) - 1u))] = c;
                base += __popc(m);
            }
            if (pass == 0 && lane == 0) n_live = base;
        }
    }
    // Self columns: S[kc·3+jc][pp] = Σ_il cs[kc·3+jc][il]·φ_K[il][pp], one
    // thread per (pp, group of kj) so that each φ value loaded feeds several sums.
    for (int o = threadIdx.x; o < 3 * PC; o += blockDim.x) {
        const int pp = o % PC, g = o / PC;  // kj = g, g+3, g+6
        const float* c0 = cs + g * L;
        const float* c1 = cs + (g + 3) * L;
        const float* c2 = cs + (g + 6) * L;
        float s0 = 0.f, s1 = 0.f, s2 = 0.f;
        for (int il = 0; il < 3 * cnt; ++il) {
            const float ph = phis[il * (PC + 1) + pp];
            s0 = fmaf(c0[il], ph, s0);
            s1 = fmaf(c1[il], ph, s1);
            s2 = fmaf(c2[il], ph, s2);
        }
        selfres[g * PC + pp] = s0;
        selfres[(g + 3) * PC + pp] = s1;
        selfres[(g + 6) * PC + pp] = s2;
    }
    __syncthreads();

    const int items = nchunks * 3 * (PC / PSUB);
    for (int it = threadIdx.x; it < items; it += blockDim.x) {
        const int q = it % nchunks, rest = it / nchunks;
        const int kc = rest % 3, pp0 = p0 + (rest / 3) * PSUB;
        if (pp0 >= a.M) continue;
        const int npp = a.M - pp0 < PSUB ? a.M - pp0 : PSUB;
        const int j0 = order[q] * CJ;
        if (q >= n_live) {  // rows outside K's neighbourhood
            const float z[CJ] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
            int64_t off = (int64_t)j0 + a.np * ((int64_t)(3 * K + kc) + (int64_t)a.n * pp0);
            const int64_t step = a.np * (int64_t)a.n;
            const bool tail = (int64_t)j0 + 4 >= a.np;
            for (int pp = 0; pp < npp; ++pp, off += step) store_chunk8<KIND>(a.u1_hi, a.u1_lo, off, z, tail);
            continue;
        }
        float c[CJ][6];
        int ro[CJ];
        chunk_setup(a, cp, slot_of, L, ss, j0, kc, c, ro);
        const float* phK = phis + 3 * ss * (PC + 1);
        int64_t off = (int64_t)j0 + a.np * ((int64_t)(3 * K + kc) + (int64_t)a.n * pp0);
        const int64_t step = a.np * (int64_t)a.n;
        const bool tail = (int64_t)j0 + 4 >= a.np;
        const int ks = 3 * K - j0;  // position of K's first row in the chunk
        const bool has_self = ks > -3 && ks < CJ;
        for (int pp = 0; pp < npp; ++pp, off += step) {
            const int P = pp0 - p0 + pp;  // mode index within the CTA
            const float k0 = phK[P], k1 = phK[(PC + 1) + P], k2 = phK[2 * (PC + 1) + P];
            float v[CJ];
#pragma unroll
            for (int e = 0; e < CJ; ++e) {
                const float* r = phis + ro[e] + P;
                float acc = c[e][3] * k0;
                acc = fmaf(c[e][4], k1, acc);
                acc = fmaf(c[e][5], k2, acc);
                acc = fmaf(c[e][0], r[0], acc);
                acc = fmaf(c[e][1], r[PC + 1], acc);
                v[e] = fmaf(c[e][2], r[2 * (PC + 1)], acc);
            }
            if (has_self) {
#pragma unroll
                for (int e = 0; e < CJ; ++e) {
                    const int jc = e - ks;
                    if (jc >= 0 && jc < 3) v[e] = selfres[(kc * 3 + jc) * PC + P];
                }
            }
            store_chunk8<KIND>(a.u1_hi, a.u1_lo, off, v, tail);
        }
    }
}

}  // namespace

// cap must be a multiple of 4 (the coefficient tables are copied as float4).
size_t sparse_p1_smem_bytes(int cap, int64_t N) {
    const size_t L = 3 * (size_t)cap;
    const size_t nchunks = (3 * (size_t)N + CJ - 1) / CJ;
    return sizeof(float) * (L * (PC + 1) + 27 * L + 9 * PC) + sizeof(int) * ((size_t)N + nchunks);
}

int sparse_p1_launch(fcb200_context* h, int kind, int64_t N, int cap, const int* d_nb, const int* d_count,
                     const int* d_self, const float* d_coef, const float* d_phi, int64_t np, int64_t mode_lo,
                     int64_t M, void* u1_hi, void* u1_lo, cudaStream_t s) {
    (void)h;
    SparseP1Args a;
    a.N = (int)N;
    a.n = (int)(3 * N);
    a.cap = cap;
    a.M = (int)M;
    a.mode_lo = (int)mode_lo;
    a.np = np;
    a.nb = d_nb;
    a.count = d_count;
    a.self_slot = d_self;
    a.coef = d_coef;
    a.phi = d_phi;
    a.u1_hi = u1_hi;
    a.u1_lo = u1_lo;
    const size_t smem = sparse_p1_smem_bytes(cap, N);
    const dim3 grid((unsigned)((M + PC - 1) / PC), (unsigned)N);
    if (kind == 1) {
        FCB_CUDA(cudaFuncSetAttribute(sparse_p1_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        sparse_p1_kernel<1><<<grid, 256, smem, s>>>(a);
    } else {
        FCB_CUDA(cudaFuncSetAttribute(sparse_p1_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        sparse_p1_kernel<2><<<grid, 256, smem, s>>>(a);
    }
    FCB_CUDA(cudaGetLastError());
    return FCB_OK;
}

}  // namespace fcb
