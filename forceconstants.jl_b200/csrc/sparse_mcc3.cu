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

constexpr int PC = 32;  // modes per CTA
constexpr int PB = 4;   // modes per shared-memory column block
constexpr int CJ = 8;   // rows per 16-byte store of a BF16 plane
constexpr int P1C_THREADS = 384;  // compact form: ≥ 3·Kc/2 tasks for neighbourhoods up to 84 atoms
constexpr int PSC = PC + 2;       // compact form: row stride of the staged φ rows (8-byte aligned mode pairs)

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

template <int KIND>
__device__ __forceinline__ void store_zero8(void* hi, void* lo, int64_t off, bool tail) {
    if constexpr (KIND == 1) {
        *reinterpret_cast<uint4*>(static_cast<__nv_bfloat16*>(hi) + off) = make_uint4(0, 0, 0, 0);
        *reinterpret_cast<uint4*>(static_cast<__nv_bfloat16*>(lo) + off) = make_uint4(0, 0, 0, 0);
    } else {
        float4* ph = reinterpret_cast<float4*>(static_cast<float*>(hi) + off);
        float4* pl = reinterpret_cast<float4*>(static_cast<float*>(lo) + off);
        ph[0] = make_float4(0.f, 0.f, 0.f, 0.f);
        pl[0] = make_float4(0.f, 0.f, 0.f, 0.f);
        if (!tail) {
            ph[1] = make_float4(0.f, 0.f, 0.f, 0.f);
            pl[1] = make_float4(0.f, 0.f, 0.f, 0.f);
        }
    }
}

// One CTA per (atom K, PC modes): the 3·PC columns U1[:, 3K+kc, p].  Shared
// memory holds the φ rows of K's neighbourhood for the CTA's modes (row stride
// PC+1), the atom's coefficient tables, the 9·PC self-column sums, and a block
// of 3·PB whole columns (n_pad FP32 rows each).  For every PB modes the block is
// zeroed, the non-zero rows are scattered into it — one thread per (neighbour
// slot, kc) computes the 3 rows of that atom, 6 terms each — and the block
// leaves as whole column segments, 8 rows (16 bytes per BF16 plane) per lane.
template <int KIND>
__global__ void __launch_bounds__(256) sparse_p1_kernel(SparseP1Args a) {
    extern __shared__ float sm[];
    const int K = blockIdx.y, p0 = blockIdx.x * PC;
    const int L = 3 * a.cap;
    const int cnt = a.count[K], ss = a.self_slot[K];
    if (cnt > a.cap) return;  // reported by the coefficient kernel; the output is invalid
    const int npad = (int)((a.np + CJ - 1) / CJ * CJ);  // block rows: n_pad rounded up to whole chunks
    float* phis = sm;                       // [L][PC+1]
    float* cp = phis + L * (PC + 1);        // pair part [3][6][L], then self part [3][3][L]
    float* cs = cp + 18 * L;
    float* selfres = cp + 27 * L;           // [9][PC]
    float* blk = selfres + 9 * PC;          // [3·PB columns][npad] (rows past n stay zero)
    const int* nbK = a.nb + (int64_t)K * a.N;
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
    // Self columns: S[kc·3+jc][pp] = Σ_il cs[kc·3+jc][il]·φ_K[il][pp].
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
    const int nch = npad / CJ;              // 16-byte chunks per column
    const int64_t step = a.np * (int64_t)a.n;
    {
        float4* b4 = reinterpret_cast<float4*>(blk);
        for (int e = threadIdx.x; e < 3 * PB * npad / 4; e += blockDim.x) b4[e] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    __syncthreads();
    for (int pb0 = 0; pb0 < PC && p0 + pb0 < a.M; pb0 += PB) {
        // scatter: item = (slot, kc), slot fastest across lanes (distinct rows,
        // distinct banks); the block is all zero here
        for (int it = threadIdx.x; it < 3 * cnt; it += blockDim.x) {
            const int kc = it / cnt, sl = it - kc * cnt;
            const int J = nbK[sl];
            if (sl == ss) {
#pragma unroll
                for (int pb = 0; pb < PB; ++pb)
#pragma unroll
                    for (int jc = 0; jc < 3; ++jc)
                        blk[(kc * PB + pb) * npad + 3 * J + jc] = selfres[(kc * 3 + jc) * PC + pb0 + pb];
                continue;
            }
            float c[3][6];
#pragma unroll
            for (int jc = 0; jc < 3; ++jc)
#pragma unroll
                for (int t = 0; t < 6; ++t) c[jc][t] = cp[(kc * 6 + t) * L + 3 * sl + jc];
            const float* rj = phis + 3 * sl * (PC + 1) + pb0;
            const float* rk = phis + 3 * ss * (PC + 1) + pb0;
#pragma unroll
            for (int pb = 0; pb < PB; ++pb) {
                const float x0 = rj[pb], x1 = rj[(PC + 1) + pb], x2 = rj[2 * (PC + 1) + pb];
                const float y0 = rk[pb], y1 = rk[(PC + 1) + pb], y2 = rk[2 * (PC + 1) + pb];
                float* dst = blk + (kc * PB + pb) * npad + 3 * J;
#pragma unroll
                for (int jc = 0; jc < 3; ++jc) {
                    float acc = c[jc][0] * x0;
                    acc = fmaf(c[jc][1], x1, acc);
                    acc = fmaf(c[jc][2], x2, acc);
                    acc = fmaf(c[jc][3], y0, acc);
                    acc = fmaf(c[jc][4], y1, acc);
                    dst[jc] = fmaf(c[jc][5], y2, acc);
                }
            }
        }
        __syncthreads();
        // write the block out (whole column segments, 8 rows per lane) and
        // leave it zero for the next modes
        for (int w = threadIdx.x; w < 3 * PB * nch; w += blockDim.x) {
            const int col = w / nch, c8 = w - col * nch;
            const int kc = col / PB, pb = col - kc * PB;
            float4* src = reinterpret_cast<float4*>(blk + col * npad + CJ * c8);
            const float4 u = src[0];
            const float4 v = src[1];
            src[0] = make_float4(0.f, 0.f, 0.f, 0.f);
            src[1] = make_float4(0.f, 0.f, 0.f, 0.f);
            if (p0 + pb0 + pb >= a.M) continue;
            const int64_t off = (int64_t)CJ * c8 + a.np * ((int64_t)(3 * K + kc)) + step * (p0 + pb0 + pb);
            const bool tail = (int64_t)CJ * c8 + 4 >= a.np;
            const bool zero = u.x == 0.f && u.y == 0.f && u.z == 0.f && u.w == 0.f && v.x == 0.f && v.y == 0.f &&
                              v.z == 0.f && v.w == 0.f;
            if (zero) {
                store_zero8<KIND>(a.u1_hi, a.u1_lo, off, tail);
            } else {
                const float x[CJ] = {u.x, u.y, u.z, u.w, v.x, v.y, v.z, v.w};
                store_chunk8<KIND>(a.u1_hi, a.u1_lo, off, x, tail);
            }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Compact first product.  U1[j,k,p] vanishes unless j ∈ nbr(atom(k)), so the
// compact form keeps, for every column k = 3K + kc and mode p, only the rows
// of K's neighbourhood in slot order:
//     U1c[j' + Kc·(p + Mp·k)],  j' = 3·slot + jc < 3·|nbr(K)|, zero up to Kc,
// and, as the second product's per-atom operand, the same rows of φ:
//     φK[j' + Kc·(q + M·K)] = φ[3·nbr(K)[slot] + jc, q].
// The second product is then a grouped GEMM over the atoms with Kc (about
// 3·|nbr|) instead of n terms.  One CTA per (atom K, PC modes); one thread per
// (kc, pair of rows j') walks the modes with its 12 coefficients in registers;
// a warp stores 128 contiguous bytes per plane.  Rows p ≥ M (up to Mp) are
// written as zeros.
struct SparseP1cArgs {
    int N, n, cap, M, Mp, Kc, mode_lo;
    const int* nb;
    const int* count;
    const int* self_slot;
    const float* coef;
    const float* phi;
    void* u1_hi;
    void* u1_lo;
    void* pk_hi;
    void* pk_lo;
};

template <int KIND>
__device__ __forceinline__ void store_pair(void* hi, void* lo, int64_t off, float v0, float v1) {
    if constexpr (KIND == 1) {
        const __nv_bfloat162 h = __floats2bfloat162_rn(v0, v1);
        const __nv_bfloat162 l = __floats2bfloat162_rn(v0 - __low2float(h), v1 - __high2float(h));
        *reinterpret_cast<__nv_bfloat162*>(static_cast<__nv_bfloat16*>(hi) + off) = h;
        *reinterpret_cast<__nv_bfloat162*>(static_cast<__nv_bfloat16*>(lo) + off) = l;
    } else {
        uint32_t b0, b1;
        asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(b0) : "f"(v0));
        asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(b1) : "f"(v1));
        const float h0 = __uint_as_float(b0), h1 = __uint_as_float(b1);
        *reinterpret_cast<float2*>(static_cast<float*>(hi) + off) = make_float2(h0, h1);
        *reinterpret_cast<float2*>(static_cast<float*>(lo) + off) = make_float2(v0 - h0, v1 - h1);
    }
}

template <int KIND>
__global__ void __launch_bounds__(P1C_THREADS) sparse_p1c_kernel(SparseP1cArgs a) {
    extern __shared__ float sm[];
    const int K = blockIdx.y, p0 = blockIdx.x * PC;
    const int L = 3 * a.cap;
    const int cnt = a.count[K], ss = a.self_slot[K];
    if (cnt > a.cap) return;  // reported by the coefficient kernel; the output is invalid
    float* phis = sm;                       // [L][PSC]
    float* cp = phis + L * PSC;             // pair part [3][6][L], then self part [3][3][L]
    float* cs = cp + 18 * L;
    float* selfres = cp + 27 * L;           // [9][PC]
    const int* nbK = a.nb + (int64_t)K * a.N;
    for (int il = threadIdx.x; il < L; il += blockDim.x) {
        const int sl = il / 3;
        const bool live = sl < cnt;
        const int64_t src = live ? (int64_t)(3 * nbK[sl] + il % 3) + (int64_t)a.n * (a.mode_lo + p0) : 0;
#pragma unroll 8
        for (int pp = 0; pp < PC; ++pp)
            phis[il * PSC + pp] = (live && p0 + pp < a.M) ? a.phi[src + (int64_t)a.n * pp] : 0.f;
    }
    {
        const float4* cg = reinterpret_cast<const float4*>(a.coef + (int64_t)K * 27 * L);
        float4* c4 = reinterpret_cast<float4*>(cp);
        for (int e = threadIdx.x; e < 27 * L / 4; e += blockDim.x) c4[e] = cg[e];
    }
    __syncthreads();
    for (int o = threadIdx.x; o < 3 * PC; o += blockDim.x) {
        const int pp = o % PC, g = o / PC;  // kj = g, g+3, g+6
        const float* c0 = cs + g * L;
        const float* c1 = cs + (g + 3) * L;
        const float* c2 = cs + (g + 6) * L;
        float s0 = 0.f, s1 = 0.f, s2 = 0.f;
        const int n3 = 3 * cnt;
        int il = 0;
        // four rows per step: the coefficient rows as float4 (L is a multiple
        // of 4), the same summation order as one row at a time
        for (; il + 4 <= n3; il += 4) {
            const float4 a0 = *reinterpret_cast<const float4*>(c0 + il);
            const float4 a1 = *reinterpret_cast<const float4*>(c1 + il);
            const float4 a2 = *reinterpret_cast<const float4*>(c2 + il);
            const float* ph = phis + il * PSC + pp;
            const float f0 = ph[0], f1 = ph[PSC], f2 = ph[2 * PSC], f3 = ph[3 * PSC];
            s0 = fmaf(a0.x, f0, s0);
            s1 = fmaf(a1.x, f0, s1);
            s2 = fmaf(a2.x, f0, s2);
            s0 = fmaf(a0.y, f1, s0);
            s1 = fmaf(a1.y, f1, s1);
            s2 = fmaf(a2.y, f1, s2);
            s0 = fmaf(a0.z, f2, s0);
            s1 = fmaf(a1.z, f2, s1);
            s2 = fmaf(a2.z, f2, s2);
            s0 = fmaf(a0.w, f3, s0);
            s1 = fmaf(a1.w, f3, s1);
            s2 = fmaf(a2.w, f3, s2);
        }
        for (; il < n3; ++il) {
            const float ph = phis[il * PSC + pp];
            s0 = fmaf(c0[il], ph, s0);
            s1 = fmaf(c1[il], ph, s1);
            s2 = fmaf(c2[il], ph, s2);
        }
        selfres[g * PC + pp] = s0;
        selfres[(g + 3) * PC + pp] = s1;
        selfres[(g + 6) * PC + pp] = s2;
    }
    // φK rows of this CTA's modes (no dependence on the self sums)
    const int npair = a.Kc / 2;
    for (int it = threadIdx.x; it < PC * npair; it += blockDim.x) {
        const int pp = it / npair, j0 = 2 * (it - pp * npair);
        if (p0 + pp >= a.M) break;
        const float v0 = j0 < 3 * cnt ? phis[j0 * PSC + pp] : 0.f;
        const float v1 = j0 + 1 < 3 * cnt ? phis[(j0 + 1) * PSC + pp] : 0.f;
        store_pair<KIND>(a.pk_hi, a.pk_lo, (int64_t)j0 + (int64_t)a.Kc * ((p0 + pp) + (int64_t)a.M * K), v0, v1);
    }
    __syncthreads();
    for (int task = threadIdx.x; task < 3 * npair; task += blockDim.x) {
        const int kc = task / npair, j0 = 2 * (task - kc * npair);
        float c[2][6];
        int rowj[2];
        bool self[2], valid[2];
        const float* sres[2];
        bool pair[2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int jv = j0 + h, sl = jv / 3, jc = jv - 3 * sl;
            valid[h] = sl < cnt;
            self[h] = sl == ss;
            pair[h] = valid[h] && !self[h];
            rowj[h] = pair[h] ? 3 * sl : 3 * ss;
            sres[h] = selfres + (kc * 3 + jc) * PC;
        }
        // both columns' coefficients by one 8-byte load (j0 even, L a multiple of 4)
#pragma unroll
        for (int t2 = 0; t2 < 6; ++t2) {
            const float2 cc = j0 < L ? *reinterpret_cast<const float2*>(cp + (kc * 6 + t2) * L + j0)
                                     : make_float2(0.f, 0.f);
            c[0][t2] = pair[0] ? cc.x : 0.f;
            c[1][t2] = pair[1] ? cc.y : 0.f;
        }
        const float* yk = phis + 3 * ss * PSC;
        int64_t off = (int64_t)j0 + (int64_t)a.Kc * (p0 + (int64_t)a.Mp * (3 * K + kc));
        // two modes per step: 8-byte shared loads (rows are PSC = PC + 2 floats apart)
        for (int pp = 0; pp < PC; pp += 2, off += 2 * (int64_t)a.Kc) {
            const float2 y0 = *reinterpret_cast<const float2*>(yk + pp);
            const float2 y1 = *reinterpret_cast<const float2*>(yk + PSC + pp);
            const float2 y2 = *reinterpret_cast<const float2*>(yk + 2 * PSC + pp);
            float v0[2], v1[2];
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const float* xj = phis + rowj[h] * PSC + pp;
                const float2 x0 = *reinterpret_cast<const float2*>(xj);
                const float2 x1 = *reinterpret_cast<const float2*>(xj + PSC);
                const float2 x2 = *reinterpret_cast<const float2*>(xj + 2 * PSC);
                float s0 = c[h][0] * x0.x, s1 = c[h][0] * x0.y;
                s0 = fmaf(c[h][1], x1.x, s0);
                s1 = fmaf(c[h][1], x1.y, s1);
                s0 = fmaf(c[h][2], x2.x, s0);
                s1 = fmaf(c[h][2], x2.y, s1);
                s0 = fmaf(c[h][3], y0.x, s0);
                s1 = fmaf(c[h][3], y0.y, s1);
                s0 = fmaf(c[h][4], y1.x, s0);
                s1 = fmaf(c[h][4], y1.y, s1);
                s0 = fmaf(c[h][5], y2.x, s0);
                s1 = fmaf(c[h][5], y2.y, s1);
                if (self[h]) {  // the self table need not be 8-byte aligned (L may be odd)
                    s0 = sres[h][pp];
                    s1 = sres[h][pp + 1];
                }
                v0[h] = valid[h] ? s0 : 0.f;
                v1[h] = valid[h] ? s1 : 0.f;
            }
            store_pair<KIND>(a.u1_hi, a.u1_lo, off, v0[0], v0[1]);
            store_pair<KIND>(a.u1_hi, a.u1_lo, off + a.Kc, v1[0], v1[1]);
        }
    }
}

}  // namespace

// cap must be a multiple of 4 (the coefficient tables are copied as float4).
size_t sparse_p1_smem_bytes(int cap, int64_t N) {
    const size_t L = 3 * (size_t)cap;
    const size_t npad = (3 * (size_t)N + 7) / 8 * 8;  // the column block holds n_pad rows (≥ the BF16 padding)
    return sizeof(float) * (L * (PC + 1) + 27 * L + 9 * PC + 3 * PB * npad);
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

namespace fcb {

size_t sparse_p1c_smem_bytes(int cap) {
    const size_t L = 3 * (size_t)cap;
    return sizeof(float) * (L * PSC + 27 * L + 9 * PC);
}

int sparse_p1c_launch(int kind, int64_t N, int cap, const int* d_nb, const int* d_count, const int* d_self,
                      const float* d_coef, const float* d_phi, int64_t mode_lo, int64_t M, int64_t Mp, int64_t Kc,
                      void* u1_hi, void* u1_lo, void* pk_hi, void* pk_lo, cudaStream_t s) {
    SparseP1cArgs a;
    a.N = (int)N;
    a.n = (int)(3 * N);
    a.cap = cap;
    a.M = (int)M;
    a.Mp = (int)Mp;
    a.Kc = (int)Kc;
    a.mode_lo = (int)mode_lo;
    a.nb = d_nb;
    a.count = d_count;
    a.self_slot = d_self;
    a.coef = d_coef;
    a.phi = d_phi;
    a.u1_hi = u1_hi;
    a.u1_lo = u1_lo;
    a.pk_hi = pk_hi;
    a.pk_lo = pk_lo;
    const size_t smem = sparse_p1c_smem_bytes(cap);
    const dim3 grid((unsigned)(Mp / PC), (unsigned)N);
    if (kind == 1) {
        FCB_CUDA(cudaFuncSetAttribute(sparse_p1c_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        sparse_p1c_kernel<1><<<grid, P1C_THREADS, smem, s>>>(a);
    } else {
        FCB_CUDA(cudaFuncSetAttribute(sparse_p1c_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        sparse_p1c_kernel<2><<<grid, P1C_THREADS, smem, s>>>(a);
    }
    FCB_CUDA(cudaGetLastError());
    return FCB_OK;
}

}  // namespace fcb
