// Dense IFC2/IFC3 assembly for pair Lennard-Jones on sm_100a.
//
// Reference semantics (ForceConstants.jl):
//   third_order!  src/analytical/third_order_analytical.jl:4-69  (pair loop, 6-way scatter)
//   ϕ₃            src/analytical/third_order_analytical.jl:216-224
//   LJ Φ′..Φ‴     src/interactions/LennardJones.jl:38-52
//   ASR!(ifc3)    src/asr.jl:19-40
//   apply_tols!   src/helper_funcs.jl:20-27
//   mass_weight_third_order!  src/analytical/third_order_analytical.jl:185-214
//
// The reference builds Ψ by scattering pair blocks into a zeroed n³ array and
// then running a strided ASR pass over it.  Here the final value of every
// element is a closed function of (I,J,K) and a small per-pair table, so Ψ is
// produced in one streaming pass that writes each byte exactly once:
//
//   kernel 1 (pairs): for every ordered pair (A,B) inside the cutoff, the 27
//     values T_AB[a][b][c] = -ϕ₃(mirror(r_A - r_B), a, b, c).
//   kernel 2 (self):  the ASR self block S_A[a][b][c] = -Σ_k X_k over k in
//     ascending order, X_k being the (A,A,k) entry the pair loop left behind.
//   kernel 3 (dense): one warp per column (jj,kk) of the column-major tensor;
//     every element's value is looked up, tol-zeroed, optionally mass
//     weighted, and stored with 16-byte vector stores (FP64), plus the FP32 /
//     split-BF16 / split-TF32 mass-weighted copies the mode products consume.
//
// Which element of T_AB a given Ψ entry takes is fixed by the reference's
// "last writer wins" order of the 6-way scatter (α outer, β, γ inner) and by
// the ASR overwrite of every (i,j,i) block; the table lookups below replay that
// order so the FP64 result is bit-identical to the CPU restatement.  Every
// FP64 operation on that path is an explicitly rounded intrinsic, so no
// multiply-add is contracted.
#include "fcb200_internal.cuh"

namespace fcb {
namespace {

__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double ddiv(double a, double b) { return __ddiv_rn(a, b); }

__device__ __forceinline__ double ipow(double x, int n) {
    double p = x;
    for (int i = 1; i < n; ++i) p = dmul(p, x);
    return p;
}

// helper_funcs.jl:7-17
__device__ __forceinline__ void nearest_mirror(double r[3], const double* box) {
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        double L = box[d];
        if (r[d] > L / 2.0) r[d] = dsub(r[d], L);
        else if (r[d] < -L / 2.0) r[d] = dadd(r[d], L);
    }
}

// LennardJones.jl:38-52 (Φ′, Φ″, Φ‴)
__device__ __forceinline__ void lj_derivs(double sigma, double eps, double r, double d[3]) {
    double s6 = ipow(sigma, 6), s12 = ipow(sigma, 12);
    d[0] = dmul(dmul(-1.0, eps), dsub(dmul(48.0, ddiv(s12, ipow(r, 13))), dmul(24.0, ddiv(s6, ipow(r, 7)))));
    d[1] = dmul(dmul(4.0, eps), dsub(dmul(156.0, ddiv(s12, ipow(r, 14))), dmul(42.0, ddiv(s6, ipow(r, 8)))));
    d[2] = dmul(dmul(-4.0, eps), dsub(dmul(2184.0, ddiv(s12, ipow(r, 15))), dmul(336.0, ddiv(s6, ipow(r, 9)))));
}

// third_order_analytical.jl:216-224
__device__ __forceinline__ double phi3(const double d[3], double rn, const double r[3], int a, int b,
                                       int c) {
    double t1 = ddiv(dmul(dmul(r[a], r[b]), r[c]), ipow(rn, 3));
    double t2 = dadd(dsub(d[2], ddiv(dmul(3.0, d[1]), rn)), ddiv(dmul(3.0, d[0]), ipow(rn, 2)));
    double s = 0.0;
    if (b == c) s = dadd(s, r[a]);
    if (c == a) s = dadd(s, r[b]);
    if (a == b) s = dadd(s, r[c]);
    double t3 = ddiv(s, ipow(rn, 2));
    double t4 = dsub(d[1], ddiv(d[0], rn));
    return dadd(dmul(t1, t2), dmul(t3, t4));
}

// second_order_analytical.jl:44-51
__device__ __forceinline__ double phi2(const double d[3], double rn, const double r[3], int a, int b) {
    double t = dmul(ddiv(dmul(r[a], r[b]), ipow(rn, 2)), dsub(d[1], ddiv(d[0], rn)));
    return (a == b) ? dadd(t, ddiv(d[0], rn)) : t;
}

__device__ __forceinline__ bool pair_vector(const double* pos, const double* box, int64_t A, int64_t B,
                                            double rc2, double r[3], double* rn) {
#pragma unroll
    for (int x = 0; x < 3; ++x) r[x] = dsub(pos[3 * A + x], pos[3 * B + x]);
    nearest_mirror(r, box);
    double d2 = dadd(dadd(dmul(r[0], r[0]), dmul(r[1], r[1])), dmul(r[2], r[2]));
    if (!(d2 < rc2)) return false;
    *rn = __dsqrt_rn(d2);
    return true;
}

// kernel 1: T_AB for every ordered pair inside the cutoff.
__global__ void lj_pair_kernel(const double* __restrict__ pos, const double* __restrict__ box,
                               int64_t N, double sigma, double eps, double rc2,
                               double* __restrict__ T, uint8_t* __restrict__ flag) {
    int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= N * N) return;
    int64_t A = p / N, B = p - A * N;
    double r[3], rn;
    bool in = (A != B) && pair_vector(pos, box, A, B, rc2, r, &rn);
    flag[p] = in ? 1 : 0;
    if (!in) return;
    double d[3];
    lj_derivs(sigma, eps, rn, d);
    double* t = T + p * 27;
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b)
            for (int c = 0; c < 3; ++c) t[9 * a + 3 * b + c] = -phi3(d, rn, r, a, b, c);
}

// kernel 2: ASR self block of every atom (asr.jl:31-32 restricted to k = i).
__global__ void lj_self_kernel(int64_t N, const double* __restrict__ T, const uint8_t* __restrict__ flag,
                               double* __restrict__ S) {
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= N * 27) return;
    int64_t I = t / 27;
    int comp = (int)(t - I * 27);
    int a = comp / 9, b = (comp / 3) % 3, c = comp % 3;
    int hi = a > b ? a : b, lo = a > b ? b : a;
    int up = 9 * a + 3 * b + c;          // k > I: block (i,i,j) written as val(α,β,γ)
    int dn = 9 * c + 3 * hi + lo;        // k < I: block (j,j,i) written as val(α,max,min)
    double s = 0.0;
    for (int64_t k = 0; k < N; ++k) {
        if (!flag[I * N + k]) continue;
        const double* tk = T + (I * N + k) * 27;
        s = dadd(s, k > I ? tk[up] : tk[dn]);
    }
    S[t] = -s;
}

struct DenseArgs {
    int64_t N, n, n_pad;
    double tol;
    const double* T;
    const uint8_t* flag;
    const double* S;
    const double* masses;
    double* psi64;
    bool psi64_weighted;
    float* psi32;
    void* split_hi;
    void* split_lo;
    int split_kind;
};

// Final (pre-tol) value of Ψ[I a, J b, K c]; see the file comment.
__device__ __forceinline__ double element_value(const DenseArgs& g, int64_t I, int a, int64_t J, int b,
                                                int64_t K, int c) {
    const int64_t N = g.N;
    if (J != K) {
        const double* t = g.T + (J * N + K) * 27;
        if (I == J) {
            if (J < K) return t[9 * a + 3 * b + c];
            int hi = a > b ? a : b, lo = a > b ? b : a;
            return t[9 * c + 3 * hi + lo];
        }
        if (I == K) {
            int hi = b > c ? b : c, lo = b > c ? c : b;
            if (K < J) return -t[9 * a + 3 * hi + lo];
            return -t[9 * b + 3 * c + a];
        }
        return 0.0;
    }
    if (I == J) return g.S[J * 27 + 9 * a + 3 * b + c];
    if (!g.flag[J * N + I]) return 0.0;
    const double* t = g.T + (J * N + I) * 27;
    if (I < J) {
        int hi = b > c ? b : c, lo = b > c ? c : b;
        return t[9 * a + 3 * hi + lo];
    }
    return t[9 * b + 3 * c + a];
}

// apply_tols! then the mass weighting of the reference, in its association
// order sqrt((m_i*m_j)*m_k).
__device__ __forceinline__ void finish(const DenseArgs& g, double v, double mJ, double mK, int64_t I,
                                       double* raw, double* mw) {
    if (fabs(v) < g.tol) v = 0.0;
    *raw = v;
    if (g.masses != nullptr && v != 0.0) {
        *mw = ddiv(v, __dsqrt_rn(dmul(dmul(g.masses[I], mJ), mK)));
    } else {
        *mw = v;
    }
}

__device__ __forceinline__ void store_split(const DenseArgs& g, int64_t off, double w0, double w1) {
    if (g.split_kind == 1) {
        __nv_bfloat162 h, l;
        h.x = __double2bfloat16(w0);
        h.y = __double2bfloat16(w1);
        l.x = __double2bfloat16(w0 - (double)__bfloat162float(h.x));
        l.y = __double2bfloat16(w1 - (double)__bfloat162float(h.y));
        *reinterpret_cast<__nv_bfloat162*>(static_cast<__nv_bfloat16*>(g.split_hi) + off) = h;
        *reinterpret_cast<__nv_bfloat162*>(static_cast<__nv_bfloat16*>(g.split_lo) + off) = l;
    } else if (g.split_kind == 2) {
        float f0 = (float)w0, f1 = (float)w1;
        uint32_t h0, h1;
        asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(h0) : "f"(f0));
        asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(h1) : "f"(f1));
        float2 h = make_float2(__uint_as_float(h0), __uint_as_float(h1));
        float2 l = make_float2((float)(w0 - (double)h.x), (float)(w1 - (double)h.y));
        *reinterpret_cast<float2*>(static_cast<float*>(g.split_hi) + off) = h;
        *reinterpret_cast<float2*>(static_cast<float*>(g.split_lo) + off) = l;
    }
}

__device__ __forceinline__ void store_split1(const DenseArgs& g, int64_t off, double w) {
    if (g.split_kind == 1) {
        __nv_bfloat16 h = __double2bfloat16(w);
        static_cast<__nv_bfloat16*>(g.split_hi)[off] = h;
        static_cast<__nv_bfloat16*>(g.split_lo)[off] = __double2bfloat16(w - (double)__bfloat162float(h));
    } else if (g.split_kind == 2) {
        float f = (float)w;
        uint32_t hb;
        asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(hb) : "f"(f));
        float h = __uint_as_float(hb);
        static_cast<float*>(g.split_hi)[off] = h;
        static_cast<float*>(g.split_lo)[off] = (float)(w - (double)h);
    }
}

// kernel 3: the dense streaming writer.  One warp per column (jj,kk).
// VEC2: n is even, so every column starts on a 16-byte boundary and each lane
// writes pairs of elements.
template <bool VEC2>
__global__ void __launch_bounds__(256) ifc3_dense_kernel(DenseArgs g) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int64_t n = g.n, N = g.N;
    const int64_t ncols = n * n;
    for (int64_t col = warp; col < ncols; col += nwarps) {
        const int64_t jj = col % n, kk = col / n;
        const int64_t J = jj / 3, K = kk / 3;
        const int b = (int)(jj - 3 * J), c = (int)(kk - 3 * K);
        const bool zero_col = (J != K) && !g.flag[J * N + K];
        const double mJ = g.masses ? g.masses[J] : 0.0, mK = g.masses ? g.masses[K] : 0.0;
        double* p64 = g.psi64 ? g.psi64 + col * n : nullptr;
        float* p32 = g.psi32 ? g.psi32 + col * n : nullptr;
        const int64_t soff = col * g.n_pad;
        if (VEC2) {
            for (int64_t e = 2 * lane; e < n; e += 64) {
                double r0 = 0.0, r1 = 0.0, w0 = 0.0, w1 = 0.0;
                if (!zero_col) {
                    int64_t I0 = e / 3, I1 = (e + 1) / 3;
                    int a0 = (int)(e - 3 * I0), a1 = (int)(e + 1 - 3 * I1);
                    double v0 = element_value(g, I0, a0, J, b, K, c);
                    double v1 = element_value(g, I1, a1, J, b, K, c);
                    finish(g, v0, mJ, mK, I0, &r0, &w0);
                    finish(g, v1, mJ, mK, I1, &r1, &w1);
                }
                if (p64) {
                    double2 o = g.psi64_weighted ? make_double2(w0, w1) : make_double2(r0, r1);
                    __stcs(reinterpret_cast<double2*>(p64 + e), o);
                }
                if (p32) __stcs(reinterpret_cast<float2*>(p32 + e), make_float2((float)w0, (float)w1));
                if (g.split_kind) store_split(g, soff + e, w0, w1);
            }
        } else {
            for (int64_t e = lane; e < n; e += 32) {
                double r0 = 0.0, w0 = 0.0;
                if (!zero_col) {
                    int64_t I0 = e / 3;
                    int a0 = (int)(e - 3 * I0);
                    finish(g, element_value(g, I0, a0, J, b, K, c), mJ, mK, I0, &r0, &w0);
                }
                if (p64) p64[e] = g.psi64_weighted ? w0 : r0;
                if (p32) p32[e] = (float)w0;
                if (g.split_kind) store_split1(g, soff + e, w0);
            }
        }
        // Padding columns of the split planes are never read by the mode
        // products (the tensor map's K extent is n), so they are left as is.
    }
}

// Split pair (hi, lo) of two consecutive mass-weighted values.  The BF16 hi
// part is rounded through FP32 (cvt.rn.f32.f64 then cvt.rn.bf16x2.f32); the lo
// part captures the exact remainder to BF16 precision either way.
__device__ __forceinline__ void split_pair(const DenseArgs& g, int64_t off, double w0, double w1) {
    if (g.split_kind == 1) {
        const __nv_bfloat162 h = __floats2bfloat162_rn((float)w0, (float)w1);
        const float h0 = __low2float(h), h1 = __high2float(h);
        const __nv_bfloat162 l = __floats2bfloat162_rn((float)(w0 - (double)h0), (float)(w1 - (double)h1));
        *reinterpret_cast<__nv_bfloat162*>(static_cast<__nv_bfloat16*>(g.split_hi) + off) = h;
        *reinterpret_cast<__nv_bfloat162*>(static_cast<__nv_bfloat16*>(g.split_lo) + off) = l;
    } else if (g.split_kind == 2) {
        uint32_t b0, b1;
        const float f0 = (float)w0, f1 = (float)w1;
        asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(b0) : "f"(f0));
        asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(b1) : "f"(f1));
        const float h0 = __uint_as_float(b0), h1 = __uint_as_float(b1);
        *reinterpret_cast<float2*>(static_cast<float*>(g.split_hi) + off) = make_float2(h0, h1);
        *reinterpret_cast<float2*>(static_cast<float*>(g.split_lo) + off) =
            make_float2((float)(w0 - (double)h0), (float)(w1 - (double)h1));
    }
}

__device__ __forceinline__ void split_zero(const DenseArgs& g, int64_t off) {
    if (g.split_kind == 1) {
        *reinterpret_cast<uint32_t*>(static_cast<__nv_bfloat16*>(g.split_hi) + off) = 0u;
        *reinterpret_cast<uint32_t*>(static_cast<__nv_bfloat16*>(g.split_lo) + off) = 0u;
    } else if (g.split_kind == 2) {
        *reinterpret_cast<float2*>(static_cast<float*>(g.split_hi) + off) = make_float2(0.f, 0.f);
        *reinterpret_cast<float2*>(static_cast<float*>(g.split_lo) + off) = make_float2(0.f, 0.f);
    }
}

// The dense writer for even n (every column starts on a 16-byte boundary).
// Lane l writes elements (2l, 2l+1) of each 64-element group, so every warp
// store instruction covers one contiguous segment (512 B of FP64, 128 B per
// BF16 plane).  The column class is decided once per column; element values
// are evaluated only for pairs that touch the rows of the column's atoms
// (pair columns) or in self columns (J == K); everything else stores
// constant zeros.
__global__ void __launch_bounds__(256) ifc3_dense_kernel2(DenseArgs g) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int n = (int)g.n;
    const int64_t N = g.N;
    const int64_t ncols = (int64_t)n * n;
    for (int64_t col = warp; col < ncols; col += nwarps) {
        const int kk = (int)(col / n), jj = (int)(col - (int64_t)kk * n);
        const int J = jj / 3, K = kk / 3;
        const int b = jj - 3 * J, c = kk - 3 * K;
        const bool self_col = (J == K);
        const bool live = self_col || g.flag[(int64_t)J * N + K];
        const int j0 = 3 * J, k0 = 3 * K;
        double* p64 = g.psi64 ? g.psi64 + col * n : nullptr;
        float* p32 = g.psi32 ? g.psi32 + col * n : nullptr;
        const int64_t soff = col * g.n_pad;
        for (int e = 2 * lane; e < n; e += 64) {
            const bool touch = live && (self_col || (e + 2 > j0 && e < j0 + 3) || (e + 2 > k0 && e < k0 + 3));
            if (!touch) {
                if (p64) __stcs(reinterpret_cast<double2*>(p64 + e), make_double2(0.0, 0.0));
                if (p32) __stcs(reinterpret_cast<float2*>(p32 + e), make_float2(0.f, 0.f));
                split_zero(g, soff + e);
                continue;
            }
            const double mJ = g.masses ? g.masses[J] : 0.0, mK = g.masses ? g.masses[K] : 0.0;
            double r0 = 0.0, r1 = 0.0, w0 = 0.0, w1 = 0.0;
            const int I0 = e / 3, I1 = (e + 1) / 3;
            const int a0 = e - 3 * I0, a1 = e + 1 - 3 * I1;
            if (self_col || I0 == J || I0 == K) finish(g, element_value(g, I0, a0, J, b, K, c), mJ, mK, I0, &r0, &w0);
            if (self_col || I1 == J || I1 == K) finish(g, element_value(g, I1, a1, J, b, K, c), mJ, mK, I1, &r1, &w1);
            if (p64) {
                const double2 o = g.psi64_weighted ? make_double2(w0, w1) : make_double2(r0, r1);
                __stcs(reinterpret_cast<double2*>(p64 + e), o);
            }
            if (p32) __stcs(reinterpret_cast<float2*>(p32 + e), make_float2((float)w0, (float)w1));
            if (g.split_kind) split_pair(g, soff + e, w0, w1);
        }
    }
}

// In-place mass weighting (third_order_analytical.jl:185-214).
template <bool VEC2>
__global__ void __launch_bounds__(256) mass_weight3_kernel(double* __restrict__ psi,
                                                           const double* __restrict__ m, int64_t n) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t col = warp; col < n * n; col += nwarps) {
        const int64_t J = (col % n) / 3, K = (col / n) / 3;
        const double mJ = m[J], mK = m[K];
        double* p = psi + col * n;
        if (VEC2) {
            for (int64_t e = 2 * lane; e < n; e += 64) {
                double2 v = *reinterpret_cast<double2*>(p + e);
                if (v.x != 0.0) v.x = ddiv(v.x, __dsqrt_rn(dmul(dmul(m[e / 3], mJ), mK)));
                if (v.y != 0.0) v.y = ddiv(v.y, __dsqrt_rn(dmul(dmul(m[(e + 1) / 3], mJ), mK)));
                *reinterpret_cast<double2*>(p + e) = v;
            }
        } else {
            for (int64_t e = lane; e < n; e += 32) {
                double v = p[e];
                if (v != 0.0) p[e] = ddiv(v, __dsqrt_rn(dmul(dmul(m[e / 3], mJ), mK)));
            }
        }
    }
}

// Second order (second_order_analytical.jl:3-42 + asr.jl:3-17 + apply_tols!),
// optionally divided by sqrt(m_i m_j) (dynmat.jl:5-33).  One thread per entry.
__global__ void lj_ifc2_kernel(const double* __restrict__ pos, const double* __restrict__ box, int64_t N,
                               double sigma, double eps, double rc2, double tol,
                               const double* __restrict__ masses, double* __restrict__ out) {
    const int64_t n = 3 * N;
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n * n) return;
    int64_t ii = t % n, jj = t / n;
    int64_t I = ii / 3, J = jj / 3;
    int a = (int)(ii - 3 * I), b = (int)(jj - 3 * J);
    double v = 0.0, r[3], rn, d[3];
    if (I != J) {
        // Entry written by the pair (min, max): -ϕ₂(r_min - r_max); ϕ₂ is even in r.
        int64_t lo = I < J ? I : J, hi = I < J ? J : I;
        if (pair_vector(pos, box, lo, hi, rc2, r, &rn)) {
            lj_derivs(sigma, eps, rn, d);
            v = -phi2(d, rn, r, I < J ? a : b, I < J ? b : a);
        }
    } else {
        double s = 0.0;
        for (int64_t k = 0; k < N; ++k) {
            if (k == I) continue;
            int64_t lo = I < k ? I : k, hi = I < k ? k : I;
            if (!pair_vector(pos, box, lo, hi, rc2, r, &rn)) continue;
            lj_derivs(sigma, eps, rn, d);
            s = dadd(s, -phi2(d, rn, r, I < k ? a : b, I < k ? b : a));
        }
        v = dmul(-1.0, s);
    }
    if (fabs(v) < tol) v = 0.0;
    if (masses != nullptr) v = v / __dsqrt_rn(dmul(masses[I], masses[J]));
    out[t] = v;
}


// ---------------------------------------------------------------------------
// Block-sparse first mode product support (snapshot path).
//
// For column (j,k) of Ψ with atoms J = j/3, K = k/3 the non-zero rows i lie in
// atoms {J, K} when J ≠ K (and only when J, K are neighbours), and in the
// neighbours of K (itself included) when J = K (the ASR column).  So with
// nbr(K) = {K} ∪ {J : flag(J,K)} every non-zero of the columns k ∈ K lies in
// rows and columns of nbr(K).

// Ascending neighbour list of every atom (itself included), stride N; the
// list's length, the self slot, and the largest length over all atoms.
__global__ void lj_neighbour_list_kernel(const uint8_t* __restrict__ flag, int N, int* __restrict__ nb,
                                         int* __restrict__ count, int* __restrict__ self_slot,
                                         int* __restrict__ max_count) {
    const int lane = threadIdx.x & 31;
    const int K = (int)(((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (K >= N) return;
    int c = 0;
    for (int J0 = 0; J0 < N; J0 += 32) {
        const int J = J0 + lane;
        const bool in = J < N && (J == K || flag[(int64_t)J * N + K]);
        const unsigned m = __ballot_sync(0xffffffffu, in);
        if (in) {
            const int slot = c + __popc(m & ((1u << lane) - 1u));
            nb[(int64_t)K * N + slot] = J;
            if (J == K) self_slot[K] = slot;
        }
        c += __popc(m);
    }
    if (lane == 0) {
        count[K] = c;
        atomicMax(max_count, c);
    }
}

// Coefficient tables of atom K (FP32, from the final mass-weighted FP64 Ψ):
//   pair part [kc][t][jl], jl = 3·slot + jc over L = 3·cap entries:
//       t < 3:  Ψ_mw[3J+t,     3J+jc, 3K+kc]   (J = nbr(K)[slot] ≠ K)
//       t ≥ 3:  Ψ_mw[3K+t-3,   3J+jc, 3K+kc]
//   self part [kc][jc][il], il = 3·slot + a:  Ψ_mw[3·nbr(K)[slot]+a, 3K+jc, 3K+kc]
// Entries past the list (and the pair part of the self slot) are zero.
__global__ void lj_sparse_coef_kernel(DenseArgs g, const int* __restrict__ nb, const int* __restrict__ count,
                                      const int* __restrict__ self_slot, int cap, float* __restrict__ coef,
                                      int* __restrict__ status) {
    const int K = blockIdx.x;
    const int N = (int)g.N, L = 3 * cap;
    const int cnt = count[K], ss = self_slot[K];
    if (cnt > cap) {  // a capacity fixed in advance was too small: report, write nothing
        if (threadIdx.x == 0) atomicCAS(status, 0, DEV_SPARSE_OVERFLOW);
        return;
    }
    const int* nbK = nb + (int64_t)K * N;
    float* out = coef + (int64_t)K * 27 * L;
    const double mK = g.masses ? g.masses[K] : 0.0;
    for (int e = threadIdx.x; e < 27 * L; e += blockDim.x) {
        double raw = 0.0, w = 0.0;
        if (e < 18 * L) {
            const int jl = e % L, kt = e / L, kc = kt / 6, t = kt % 6;
            const int sl = jl / 3, jc = jl % 3;
            if (sl < cnt && sl != ss) {
                const int J = nbK[sl];
                const int I = t < 3 ? J : K, a = t < 3 ? t : t - 3;
                const double mJ = g.masses ? g.masses[J] : 0.0;
                finish(g, element_value(g, I, a, J, jc, K, kc), mJ, mK, I, &raw, &w);
            }
        } else {
            const int f = e - 18 * L;
            const int il = f % L, kj = f / L, kc = kj / 3, jc = kj % 3;
            const int sl = il / 3, a = il % 3;
            if (sl < cnt) finish(g, element_value(g, nbK[sl], a, K, jc, K, kc), mK, mK, nbK[sl], &raw, &w);
        }
        out[e] = (float)w;
    }
}
}  // namespace

int lj_pair_tables(fcb200_context* h, const double* d_pos, int64_t N, const double* d_box, double sigma,
                   double eps, double r_cut, cudaStream_t s) {
    const int64_t pairs = N * N;
    FCB_TRY(h->pair_t.ensure(sizeof(double) * 27 * pairs));
    FCB_TRY(h->pair_flag.ensure(pairs));
    FCB_TRY(h->self_t.ensure(sizeof(double) * 27 * N));
    const double rc2 = r_cut * r_cut;
    lj_pair_kernel<<<(unsigned)((pairs + 127) / 128), 128, 0, s>>>(d_pos, d_box, N, sigma, eps, rc2,
                                                                     h->pair_t.as<double>(),
                                                                     h->pair_flag.as<uint8_t>());
    FCB_CUDA(cudaGetLastError());
    lj_self_kernel<<<(unsigned)((N * 27 + 127) / 128), 128, 0, s>>>(N, h->pair_t.as<double>(),
                                                                      h->pair_flag.as<uint8_t>(),
                                                                      h->self_t.as<double>());
    FCB_CUDA(cudaGetLastError());
    return FCB_OK;
}

int ifc3_dense_write(fcb200_context* h, int64_t N, double tol, const double* d_masses,
                     const AssemblyOut& out, cudaStream_t s, int blocks_per_sm) {
    DenseArgs g;
    g.N = N;
    g.n = 3 * N;
    g.n_pad = out.n_pad ? out.n_pad : g.n;
    g.tol = tol;
    g.T = h->pair_t.as<double>();
    g.flag = h->pair_flag.as<uint8_t>();
    g.S = h->self_t.as<double>();
    g.masses = d_masses;
    g.psi64 = out.psi64;
    g.psi64_weighted = out.psi64_weighted;
    g.psi32 = out.psi32;
    g.split_hi = out.split_hi;
    g.split_lo = out.split_lo;
    g.split_kind = out.split_kind;
    // The writer asks for the largest shared-memory carveout although it uses
    // none: an SM whose split was set for a block of the writer must still
    // take a CTA of the tensor-core mode product (211 KB) running beside it.
    static bool carveout_set[64] = {};
    if (h->device >= 0 && h->device < 64 && !carveout_set[h->device]) {
        FCB_CUDA(cudaFuncSetAttribute(ifc3_dense_kernel2, cudaFuncAttributePreferredSharedMemoryCarveout,
                                      cudaSharedmemCarveoutMaxShared));
        FCB_CUDA(cudaFuncSetAttribute(ifc3_dense_kernel<false>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                      cudaSharedmemCarveoutMaxShared));
        carveout_set[h->device] = true;
    }
    const int64_t cols = g.n * g.n;
    int64_t blocks = (cols + 7) / 8;
    const int64_t cap = (int64_t)h->sm_count * blocks_per_sm;
    if (blocks > cap) blocks = cap;
    if (g.n % 2 == 0 && g.n_pad % 2 == 0)
        ifc3_dense_kernel2<<<(unsigned)blocks, 256, 0, s>>>(g);
    else
        ifc3_dense_kernel<false><<<(unsigned)blocks, 256, 0, s>>>(g);
    FCB_CUDA(cudaGetLastError());
    return FCB_OK;
}

int mass_weight3_launch(double* d_psi, const double* d_masses, int64_t N, cudaStream_t s) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int64_t n = 3 * N;
    int64_t blocks = (n * n + 7) / 8;
    if (blocks > (int64_t)sms * 8) blocks = (int64_t)sms * 8;
    if (n % 2 == 0)
        mass_weight3_kernel<true><<<(unsigned)blocks, 256, 0, s>>>(d_psi, d_masses, n);
    else
        mass_weight3_kernel<false><<<(unsigned)blocks, 256, 0, s>>>(d_psi, d_masses, n);
    FCB_CUDA(cudaGetLastError());
    return FCB_OK;
}

int lj_second_order_launch(fcb200_context* h, const double* d_pos, int64_t N, const double* d_box,
                           double sigma, double eps, double r_cut, double tol, const double* d_masses,
                           double* d_ifc2, cudaStream_t s) {
    (void)h;
    const int64_t n = 3 * N;
    lj_ifc2_kernel<<<(unsigned)((n * n + 255) / 256), 256, 0, s>>>(d_pos, d_box, N, sigma, eps,
                                                                     r_cut * r_cut, tol, d_masses, d_ifc2);
    FCB_CUDA(cudaGetLastError());
    return FCB_OK;
}


// Launchers over caller-provided scratch (T: N*N*27 doubles, flag: N*N bytes,
// S: N*27 doubles).  Same kernels as above; used by the entry point whose
// scratch is a fixed device array instead of handle-owned allocations.
int lj_pair_tables_raw(double* T, uint8_t* flag, double* S, const double* d_pos, int64_t N, const double* d_box,
                       double sigma, double eps, double r_cut, cudaStream_t s) {
    const int64_t pairs = N * N;
    const double rc2 = r_cut * r_cut;
    lj_pair_kernel<<<(unsigned)((pairs + 127) / 128), 128, 0, s>>>(d_pos, d_box, N, sigma, eps, rc2, T, flag);
    FCB_CUDA(cudaGetLastError());
    lj_self_kernel<<<(unsigned)((N * 27 + 127) / 128), 128, 0, s>>>(N, T, flag, S);
    FCB_CUDA(cudaGetLastError());
    return FCB_OK;
}

int ifc3_dense_write_raw(const double* T, const uint8_t* flag, const double* S, int sm_count, int64_t N, double tol,
                         const double* d_masses, const AssemblyOut& out, cudaStream_t s) {
    DenseArgs g;
    g.N = N;
    g.n = 3 * N;
    g.n_pad = out.n_pad ? out.n_pad : g.n;
    g.tol = tol;
    g.T = T;
    g.flag = flag;
    g.S = S;
    g.masses = d_masses;
    g.psi64 = out.psi64;
    g.psi64_weighted = out.psi64_weighted;
    g.psi32 = out.psi32;
    g.split_hi = out.split_hi;
    g.split_lo = out.split_lo;
    g.split_kind = out.split_kind;
    const int64_t cols = g.n * g.n;
    int64_t blocks = (cols + 7) / 8;
    const int64_t cap = (int64_t)sm_count * 8;
    if (blocks > cap) blocks = cap;
    if (g.n % 2 == 0 && g.n_pad % 2 == 0)
        ifc3_dense_kernel2<<<(unsigned)blocks, 256, 0, s>>>(g);
    else
        ifc3_dense_kernel<false><<<(unsigned)blocks, 256, 0, s>>>(g);
    FCB_CUDA(cudaGetLastError());
    return FCB_OK;
}


int lj_neighbour_lists(fcb200_context* h, int64_t N, int* d_nb, int* d_count, int* d_self, int* d_max,
                       cudaStream_t s) {
    FCB_CUDA(cudaMemsetAsync(d_max, 0, sizeof(int), s));
    const int64_t threads = 32 * N;
    lj_neighbour_list_kernel<<<(unsigned)((threads + 255) / 256), 256, 0, s>>>(h->pair_flag.as<uint8_t>(), (int)N,
                                                                                 d_nb, d_count, d_self, d_max);
    FCB_CUDA(cudaGetLastError());
    return FCB_OK;
}

int lj_sparse_coefs(fcb200_context* h, int64_t N, double tol, const double* d_masses, const int* d_nb,
                    const int* d_count, const int* d_self, int cap, float* d_coef, cudaStream_t s) {
    DenseArgs g = {};
    g.N = N;
    g.n = 3 * N;
    g.n_pad = g.n;
    g.tol = tol;
    g.T = h->pair_t.as<double>();
    g.flag = h->pair_flag.as<uint8_t>();
    g.S = h->self_t.as<double>();
    g.masses = d_masses;
    lj_sparse_coef_kernel<<<(unsigned)N, 256, 0, s>>>(g, d_nb, d_count, d_self, cap, d_coef, h->d_status);
    FCB_CUDA(cudaGetLastError());
    return FCB_OK;
}

}  // namespace fcb
