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
constexpr int P1M_MODES = 64;     // compact form: modes per CTA (two per thread of a warp)
constexpr int P1M_THREADS = 256;  // compact form: 8 warps
constexpr int P1M_J = 16;         // compact form: φK rows per store (one 32-byte sector per BF16 plane)
constexpr int P1M_LD = P1M_MODES + 2;  // compact form: row stride of the staged φ rows (8-byte mode pairs)
constexpr int P1M_STAGE = 32;     // compact form: φ loads a thread has in flight while staging
static_assert(P1M_MODES % P1M_STAGE == 0, "the staging batches cover the CTA's modes");

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
//     U1c[p + Mp·(j' + Kc·k)],  j' = 3·slot + jc < 3·|nbr(K)|, zero up to Kc,
// and, as the second product's per-atom operand, the same rows of φ:
//     φK[j' + Kc·(q + M·K)] = φ[3·nbr(K)[slot] + jc, q].
// The second product is then a grouped GEMM over the atoms with Kc (about
// 3·|nbr|) instead of n terms.
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

// Packed FP32 pairs (Blackwell's f32x2 mul / fma: two IEEE operations per
// instruction, each rounded as mulf / fmaf would round it).
__device__ __forceinline__ uint64_t f2u(float2 v) { return *reinterpret_cast<const uint64_t*>(&v); }
__device__ __forceinline__ float2 u2f(uint64_t v) { return *reinterpret_cast<const float2*>(&v); }

__device__ __forceinline__ float2 mul2(float2 a, float2 b) {
    uint64_t d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(f2u(a)), "l"(f2u(b)));
    return u2f(d);
}

__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) {
    uint64_t d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(f2u(a)), "l"(f2u(b)), "l"(f2u(c)));
    return u2f(d);
}

// 32 bytes in one 256-bit store (a whole L2 sector per lane).
__device__ __forceinline__ void st_v8(void* p, const uint32_t (&v)[8]) {
    asm volatile("st.global.v8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"l"(p), "r"(v[0]), "r"(v[1]),
                 "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7])
                 : "memory");
}

// Split 16 consecutive values into the hi/lo planes at element offset `off`
// (a multiple of 16): 32 bytes per BF16 plane, 64 per TF32 plane.
template <int KIND>
__device__ __forceinline__ void store_chunk16(void* hi, void* lo, int64_t off, const float (&v)[P1M_J]) {
    if constexpr (KIND == 1) {
        uint32_t h[8], l[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const __nv_bfloat162 hb = __floats2bfloat162_rn(v[2 * i], v[2 * i + 1]);
            const __nv_bfloat162 lb =
                __floats2bfloat162_rn(v[2 * i] - __low2float(hb), v[2 * i + 1] - __high2float(hb));
            h[i] = *reinterpret_cast<const uint32_t*>(&hb);
            l[i] = *reinterpret_cast<const uint32_t*>(&lb);
        }
        st_v8(static_cast<__nv_bfloat16*>(hi) + off, h);
        st_v8(static_cast<__nv_bfloat16*>(lo) + off, l);
    } else {
#pragma unroll
        for (int half = 0; half < 2; ++half) {
            uint32_t h[8], l[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                uint32_t b;
                asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(b) : "f"(v[8 * half + i]));
                h[i] = b;
                l[i] = __float_as_uint(v[8 * half + i] - __uint_as_float(b));
            }
            st_v8(static_cast<float*>(hi) + off + 8 * half, h);
            st_v8(static_cast<float*>(lo) + off + 8 * half, l);
        }
    }
}

// Split a pair of values (two consecutive modes) into the hi/lo planes at
// element offset `off` (even): 4 bytes per BF16 plane, 8 per TF32 plane.
template <int KIND>
__device__ __forceinline__ void store_mode_pair(void* hi, void* lo, int64_t off, float2 v) {
    if constexpr (KIND == 1) {
        const __nv_bfloat162 h = __floats2bfloat162_rn(v.x, v.y);
        const __nv_bfloat162 l = __floats2bfloat162_rn(v.x - __low2float(h), v.y - __high2float(h));
        *reinterpret_cast<__nv_bfloat162*>(static_cast<__nv_bfloat16*>(hi) + off) = h;
        *reinterpret_cast<__nv_bfloat162*>(static_cast<__nv_bfloat16*>(lo) + off) = l;
    } else {
        uint32_t b0, b1;
        asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(b0) : "f"(v.x));
        asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(b1) : "f"(v.y));
        const float h0 = __uint_as_float(b0), h1 = __uint_as_float(b1);
        *reinterpret_cast<float2*>(static_cast<float*>(hi) + off) = make_float2(h0, h1);
        *reinterpret_cast<float2*>(static_cast<float*>(lo) + off) = make_float2(v.x - h0, v.y - h1);
    }
}

// One CTA per (atom K, P1M_MODES modes); a thread holds two consecutive
// modes, so every store of a warp is 128 contiguous bytes of one BF16 plane:
// U1c is written mode-fastest, U1c[p + Mp·(j' + Kc·k)], and read by the second
// product as an MN-major A operand.  After staging (the φ rows of K's
// neighbourhood, and the pair coefficients rearranged per slot with every
// value doubled for the packed f32x2 arithmetic), warps 0-2 form the ASR self
// sums of column kc = warp (in the reference's term order) and warps 3-7 write
// the φK rows; then the slots go round-robin to the 8 warps, a warp computing
// the 9 rows (kc, jc) of its slot for all 64 modes.  Every entry is c0·x0 then
// five fused multiply-adds, as in the reference contraction's term order.
// Rows j' from 3·|nbr(K)| up to Kc, and modes p ≥ M (up to Mp), are zeros.
// Held to 96 registers: two CTAs (2 × 256 × 96) leave room on every SM for
// one 256-thread block of the FP64 Ψ writer (64 registers), which the
// snapshot path starts beside this kernel on a second stream.
template <int KIND>
__global__ void __maxnreg__(96) sparse_p1m_kernel(SparseP1cArgs a) {
    extern __shared__ float sm[];
    const int K = blockIdx.y, p0 = blockIdx.x * P1M_MODES;
    const int L = 3 * a.cap;
    const int cnt = a.count[K], ss = a.self_slot[K];
    if (cnt > a.cap) return;  // reported by the coefficient kernel; the output is invalid
    const int n3 = 3 * cnt;
    float* phis = sm;                              // [L][P1M_LD], mode fastest
    float* cdup = phis + L * P1M_LD;               // [slot][kc][jc][t][2]: 108 floats per slot
    float* cs = cdup + 108 * a.cap;                // self part [kc][jc][L]
    float* selfres = cs + 9 * L;                   // [kc][jc][P1M_MODES]
    const int* nbK = a.nb + (int64_t)K * a.N;
    const float* coefK = a.coef + (int64_t)K * 27 * L;
    // Staging: the tables sit in L2, so its time is load latency.  Each thread
    // issues a whole batch of loads into registers before its first shared
    // store: 2 round trips for the φ rows, 1 for the pair coefficients and
    // 1 for the self part (where a shared store after every load waited on
    // each load in turn, 29 round trips).
    for (int il = threadIdx.x; il < L; il += blockDim.x) {
        const int sl = il / 3;
        const bool live = sl < cnt;
        const float* src = a.phi + (live ? (int64_t)(3 * nbK[sl] + il % 3) + (int64_t)a.n * (a.mode_lo + p0) : 0);
#pragma unroll
        for (int h = 0; h < P1M_MODES; h += P1M_STAGE) {
            float v[P1M_STAGE];
#pragma unroll
            for (int u = 0; u < P1M_STAGE; ++u)
                v[u] = (live && p0 + h + u < a.M) ? src[(int64_t)a.n * (h + u)] : 0.f;
#pragma unroll
            for (int u = 0; u < P1M_STAGE; ++u) phis[il * P1M_LD + h + u] = v[u];
        }
    }
    for (int j = threadIdx.x; j < L; j += blockDim.x) {   // pair part: row r = kc·6 + t of the table
        const int sl = j / 3, jc = j - 3 * sl;
        float c[18];
#pragma unroll
        for (int r = 0; r < 18; ++r) c[r] = coefK[r * L + j];
#pragma unroll
        for (int r = 0; r < 18; ++r) {
            const int kc = r / 6, t = r - 6 * kc;
            *reinterpret_cast<float2*>(cdup + ((sl * 9 + kc * 3 + jc) * 6 + t) * 2) = make_float2(c[r], c[r]);
        }
    }
    {
        const float4* cg = reinterpret_cast<const float4*>(coefK + 18 * L);
        float4* c4 = reinterpret_cast<float4*>(cs);
        const int E = 9 * L / 4;
        for (int e0 = threadIdx.x; e0 < E; e0 += 4 * blockDim.x) {
            float4 t[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int e = e0 + u * blockDim.x;
                t[u] = e < E ? cg[e] : make_float4(0.f, 0.f, 0.f, 0.f);
            }
#pragma unroll
            for (int u = 0; u < 4; ++u)
                if (e0 + u * (int)blockDim.x < E) c4[e0 + u * blockDim.x] = t[u];
        }
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int pm = 2 * lane;                       // this thread's modes p0 + pm, p0 + pm + 1
    if (warp < 3) {
        // self sums of column kc: Σ_il cs[kc][jc][il] · φ[il, p], il ascending
        const int kc = warp;
        const float* c0 = cs + (kc * 3) * L;
        const float* c1 = c0 + L;
        const float* c2 = c1 + L;
        float2 s0 = make_float2(0.f, 0.f), s1 = s0, s2 = s0;
        int il = 0;
        for (; il + 4 <= n3; il += 4) {
            const float4 a0 = *reinterpret_cast<const float4*>(c0 + il);
            const float4 a1 = *reinterpret_cast<const float4*>(c1 + il);
            const float4 a2 = *reinterpret_cast<const float4*>(c2 + il);
            const float* ph = phis + il * P1M_LD + pm;
            const float2 f0 = *reinterpret_cast<const float2*>(ph);
            const float2 f1 = *reinterpret_cast<const float2*>(ph + P1M_LD);
            const float2 f2 = *reinterpret_cast<const float2*>(ph + 2 * P1M_LD);
            const float2 f3 = *reinterpret_cast<const float2*>(ph + 3 * P1M_LD);
            s0 = fma2(make_float2(a0.x, a0.x), f0, s0);
            s1 = fma2(make_float2(a1.x, a1.x), f0, s1);
            s2 = fma2(make_float2(a2.x, a2.x), f0, s2);
            s0 = fma2(make_float2(a0.y, a0.y), f1, s0);
            s1 = fma2(make_float2(a1.y, a1.y), f1, s1);
            s2 = fma2(make_float2(a2.y, a2.y), f1, s2);
            s0 = fma2(make_float2(a0.z, a0.z), f2, s0);
            s1 = fma2(make_float2(a1.z, a1.z), f2, s1);
            s2 = fma2(make_float2(a2.z, a2.z), f2, s2);
            s0 = fma2(make_float2(a0.w, a0.w), f3, s0);
            s1 = fma2(make_float2(a1.w, a1.w), f3, s1);
            s2 = fma2(make_float2(a2.w, a2.w), f3, s2);
        }
        for (; il < n3; ++il) {
            const float2 ph = *reinterpret_cast<const float2*>(phis + il * P1M_LD + pm);
            s0 = fma2(make_float2(c0[il], c0[il]), ph, s0);
            s1 = fma2(make_float2(c1[il], c1[il]), ph, s1);
            s2 = fma2(make_float2(c2[il], c2[il]), ph, s2);
        }
        *reinterpret_cast<float2*>(selfres + (kc * 3 + 0) * P1M_MODES + pm) = s0;
        *reinterpret_cast<float2*>(selfres + (kc * 3 + 1) * P1M_MODES + pm) = s1;
        *reinterpret_cast<float2*>(selfres + (kc * 3 + 2) * P1M_MODES + pm) = s2;
    } else {
        // φK rows: φK[j' + Kc·(q + M·K)], zero past the neighbourhood, 16 rows
        // of a mode per task (one 32-byte sector per BF16 plane)
        const int npk = a.Kc / P1M_J;
        for (int task = threadIdx.x - 96; task < P1M_MODES * npk; task += P1M_THREADS - 96) {
            const int q = task % P1M_MODES, ck = task / P1M_MODES;
            if (p0 + q >= a.M) continue;
            float v[P1M_J];
#pragma unroll
            for (int jj = 0; jj < P1M_J; ++jj) {
                const int j = ck * P1M_J + jj;
                v[jj] = j < n3 ? phis[j * P1M_LD + q] : 0.f;
            }
            store_chunk16<KIND>(a.pk_hi, a.pk_lo, (int64_t)a.Kc * ((p0 + q) + (int64_t)a.M * K) + ck * P1M_J, v);
        }
    }
    __syncthreads();
    float2 y[3];
#pragma unroll
    for (int t = 0; t < 3; ++t) y[t] = *reinterpret_cast<const float2*>(phis + (3 * ss + t) * P1M_LD + pm);
    // U1c[p + Mp·(j' + Kc·(3K + kc))]
    const int64_t colK = (int64_t)a.Kc * (3 * K);
    const int64_t pbase = p0 + pm;
    for (int sl = warp; sl < cnt; sl += P1M_THREADS / 32) {
        float2 x[3];
#pragma unroll
        for (int t = 0; t < 3; ++t) x[t] = *reinterpret_cast<const float2*>(phis + (3 * sl + t) * P1M_LD + pm);
        const float4* cq = reinterpret_cast<const float4*>(cdup + sl * 108);
        const bool self = sl == ss;
#pragma unroll
        for (int kc = 0; kc < 3; ++kc)
#pragma unroll
            for (int jc = 0; jc < 3; ++jc) {
                const float4 q0 = cq[(kc * 3 + jc) * 3], q1 = cq[(kc * 3 + jc) * 3 + 1],
                             q2 = cq[(kc * 3 + jc) * 3 + 2];
                float2 v = mul2(make_float2(q0.x, q0.y), x[0]);
                v = fma2(make_float2(q0.z, q0.w), x[1], v);
                v = fma2(make_float2(q1.x, q1.y), x[2], v);
                v = fma2(make_float2(q1.z, q1.w), y[0], v);
                v = fma2(make_float2(q2.x, q2.y), y[1], v);
                v = fma2(make_float2(q2.z, q2.w), y[2], v);
                if (self) v = *reinterpret_cast<const float2*>(selfres + (kc * 3 + jc) * P1M_MODES + pm);
                store_mode_pair<KIND>(a.u1_hi, a.u1_lo,
                                      pbase + (int64_t)a.Mp * ((3 * sl + jc) + colK + (int64_t)a.Kc * kc), v);
            }
    }
    // rows past the neighbourhood
    const int nz = a.Kc - n3;
    for (int e = warp; e < 3 * nz; e += P1M_THREADS / 32) {
        const int kc = e / nz, j = n3 + (e - kc * nz);
        store_mode_pair<KIND>(a.u1_hi, a.u1_lo, pbase + (int64_t)a.Mp * (j + colK + (int64_t)a.Kc * kc),
                              make_float2(0.f, 0.f));
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
    return sizeof(float) * (L * P1M_LD + 108 * (size_t)cap + 9 * L + 9 * P1M_MODES);
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
    const dim3 grid((unsigned)(Mp / P1M_MODES), (unsigned)N);
    if (kind == 1) {
        FCB_CUDA(cudaFuncSetAttribute(sparse_p1m_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        sparse_p1m_kernel<1><<<grid, P1M_THREADS, smem, s>>>(a);
    } else {
        FCB_CUDA(cudaFuncSetAttribute(sparse_p1m_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        sparse_p1m_kernel<2><<<grid, P1M_THREADS, smem, s>>>(a);
    }
    FCB_CUDA(cudaGetLastError());
    return FCB_OK;
}

}  // namespace fcb
