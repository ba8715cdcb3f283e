// Adjoint of the LJ snapshot: gradient of a scalar of K3 with respect to the
// atomic positions and the LJ parameters σ, ε, with φ frozen.
//
// L = Σ_{abc} W[a,b,c] K3[a,b,c], K3 over modes [0,M) on every axis.  With
// Ψ_mw[i,j,k] = Ψ[i,j,k]/sqrt(m_i m_j m_k) and K3 = Ψ_mw ×₁ φ ×₂ φ ×₃ φ,
//     L = Σ_ijk G[i,j,k] Ψ_mw[i,j,k],   G = W ×₁ φᵀ ×₂ φᵀ ×₃ φᵀ,
// i.e. the three transposed mode products of mcc3 (src/mcc.jl:29-51) applied
// to W.  G runs on the same mode-product kernels (tensor cores or FP32), or in
// FP64 on the FP64 tensor-core mode product (FCB_ADJOINT_FP64).
//
// For the analytical LJ calculator every non-zero Ψ block belongs to one
// ordered pair (A,B) inside the cutoff: the blocks with two A's and one B hold
// −ϕ₃(d_AB) (third_order_analytical.jl:4-69) and the ASR block (A,A,A) holds
// Σ_B ϕ₃(d_AB) (asr.jl:19-40).  Hence
//     L = Σ_(A,B) Σ_abc ϕ₃(d_AB)_abc C_AB[abc],
//     C_AB = G'[AAA] − G'[AAB] − G'[ABA] − G'[BAA]   (G' = G / sqrt(m m m)),
// and with d_AB = r_A − r_B (single minimum image):
//     ∂L/∂r_A = Σ_B v_AB − Σ_B v_BA,   v_AB[d] = Σ_abc ϕ₄(d_AB)_abcd C_AB[abc],
//     ∂L/∂ε = L/ε,   ∂L/∂σ = Σ_(A,B) Σ_abc (∂ϕ₃/∂σ)(d_AB)_abc C_AB[abc],
// with ϕ₄ the fourth pair derivative (src/analytical/fourth_order_analytical.jl:184-198,
// LennardJones.jl:54-56).  Neither Ψ nor the fourth-order tensor is ever
// stored: each pair's blocks are recomputed where they are contracted.  The
// tolerance cutoff of Ψ (apply_tols!) is not differentiated.
#include "fcb200_internal.cuh"

namespace fcb {
namespace {

__device__ __forceinline__ void nearest_mirror(double r[3], const double* box) {
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const double L = box[d];
        if (r[d] > L / 2.0) r[d] = r[d] - L;
        else if (r[d] < -L / 2.0) r[d] = r[d] + L;
    }
}

__global__ void transpose_kernel(const float* __restrict__ phi, int64_t n, int64_t M, float* __restrict__ phiT) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n * M) return;
    const int64_t a = t % M, p = t / M;  // phiT[a + M p] = φ[p, a]
    phiT[t] = phi[p + n * a];
}

// Radial derivatives of the LJ pair potential (LennardJones.jl:38-56) and their σ-derivatives.
struct LJRad {
    double d1, d2, d3, d4;      // Φ′..Φ⁗
    double s1, s2, s3;          // ∂Φ′/∂σ, ∂Φ″/∂σ, ∂Φ‴/∂σ
};

__device__ LJRad lj_rad(double sigma, double eps, double r) {
    const double s6 = pow(sigma, 6.0), s12 = s6 * s6, s5 = s6 / sigma, s11 = s12 / sigma;
    const double r2 = r * r, r6 = r2 * r2 * r2, r7 = r6 * r, r8 = r7 * r, r9 = r8 * r, r10 = r9 * r;
    const double r13 = r6 * r7, r14 = r13 * r, r15 = r14 * r, r16 = r15 * r;
    LJRad o;
    o.d1 = -eps * (48.0 * s12 / r13 - 24.0 * s6 / r7);
    o.d2 = 4.0 * eps * (156.0 * s12 / r14 - 42.0 * s6 / r8);
    o.d3 = -4.0 * eps * (2184.0 * s12 / r15 - 336.0 * s6 / r9);
    o.d4 = 4.0 * eps * (32760.0 * s12 / r16 - 3024.0 * s6 / r10);
    o.s1 = -eps * (48.0 * 12.0 * s11 / r13 - 24.0 * 6.0 * s5 / r7);
    o.s2 = 4.0 * eps * (156.0 * 12.0 * s11 / r14 - 42.0 * 6.0 * s5 / r8);
    o.s3 = -4.0 * eps * (2184.0 * 12.0 * s11 / r15 - 336.0 * 6.0 * s5 / r9);
    return o;
}

// ϕ₃ (third_order_analytical.jl:216-224) with radial derivatives (f1,f2,f3)
__device__ __forceinline__ double phi3_of(double f1, double f2, double f3, const double nh[3], double r, int a, int b,
                                          int c) {
    const double A = f3 - 3.0 * f2 / r + 3.0 * f1 / (r * r);
    const double B = (f2 - f1 / r) / r;
    const double s = (b == c ? nh[a] : 0.0) + (c == a ? nh[b] : 0.0) + (a == b ? nh[c] : 0.0);
    return nh[a] * nh[b] * nh[c] * A + s * B;
}

// ϕ₄ (fourth_order_analytical.jl:184-198)
__device__ __forceinline__ double phi4_of(const LJRad& f, const double nh[3], double r, int a, int b, int c, int d) {
    const double E4 = f.d4 - 6.0 * f.d3 / r + 15.0 * f.d2 / (r * r) - 15.0 * f.d1 / (r * r * r);
    const double E3 = (f.d3 - 3.0 * f.d2 / r + 3.0 * f.d1 / (r * r)) / r;
    const double E2 = (f.d2 - f.d1 / r) / (r * r);
    auto dl = [](int x, int y) { return x == y ? 1.0 : 0.0; };
    const double v = nh[a] * nh[b] * dl(c, d) + nh[a] * nh[c] * dl(b, d) + nh[a] * nh[d] * dl(b, c) +
                     nh[b] * nh[c] * dl(a, d) + nh[b] * nh[d] * dl(a, c) + nh[c] * nh[d] * dl(a, b);
    return nh[a] * nh[b] * nh[c] * nh[d] * E4 + v * E3 +
           (dl(a, b) * dl(c, d) + dl(a, c) * dl(b, d) + dl(a, d) * dl(b, c)) * E2;
}

// one thread per ordered pair (A,B): v_AB, (∂ϕ₃/∂σ)·C, ϕ₃·C; G in FP32 or FP64
template <class GT>
__global__ void lj_adjoint_pair_kernel(const double* __restrict__ pos, const double* __restrict__ box, int64_t N,
                                       double sigma, double eps, double rc2, const double* __restrict__ masses,
                                       const GT* __restrict__ G, double* __restrict__ V, double* __restrict__ Sg,
                                       double* __restrict__ Lp) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= N * N) return;
    const int64_t A = p / N, B = p - A * N;
    double r[3] = {0, 0, 0};
    bool in = A != B;
    double d2 = 0.0;
    if (in) {
#pragma unroll
        for (int d = 0; d < 3; ++d) r[d] = pos[3 * A + d] - pos[3 * B + d];
        nearest_mirror(r, box);
        d2 = (r[0] * r[0] + r[1] * r[1]) + r[2] * r[2];
        in = d2 < rc2;
    }
    if (!in) {
        V[3 * p] = V[3 * p + 1] = V[3 * p + 2] = 0.0;
        Sg[p] = 0.0;
        Lp[p] = 0.0;
        return;
    }
    const int64_t n = 3 * N;
    const double rn = sqrt(d2), nh[3] = {r[0] / rn, r[1] / rn, r[2] / rn};
    const LJRad f = lj_rad(sigma, eps, rn);
    const double mA = masses[A], mB = masses[B];
    const double wAAA = 1.0 / sqrt(mA * mA * mA), wAAB = 1.0 / sqrt(mA * mA * mB);
    auto g = [&](int64_t i, int64_t j, int64_t k) { return (double)G[i + n * (j + n * k)]; };
    double v[3] = {0, 0, 0}, sg = 0.0, l = 0.0;
    for (int c = 0; c < 3; ++c)
        for (int b = 0; b < 3; ++b)
            for (int a = 0; a < 3; ++a) {
                const int64_t Aa = 3 * A + a, Ab = 3 * A + b, Ac = 3 * A + c, Ba = 3 * B + a, Bb = 3 * B + b,
                              Bc = 3 * B + c;
                const double C = wAAA * g(Aa, Ab, Ac) - wAAB * (g(Aa, Ab, Bc) + g(Aa, Bb, Ac) + g(Ba, Ab, Ac));
                l += phi3_of(f.d1, f.d2, f.d3, nh, rn, a, b, c) * C;
                sg += phi3_of(f.s1, f.s2, f.s3, nh, rn, a, b, c) * C;
#pragma unroll
                for (int d = 0; d < 3; ++d) v[d] += phi4_of(f, nh, rn, a, b, c, d) * C;
            }
    V[3 * p] = v[0];
    V[3 * p + 1] = v[1];
    V[3 * p + 2] = v[2];
    Sg[p] = sg;
    Lp[p] = l;
}

// ∂L/∂r_A = Σ_B v_AB − Σ_B v_BA (fixed order: deterministic)
__global__ void lj_adjoint_atom_kernel(int64_t N, const double* __restrict__ V, double* __restrict__ dpos) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 3 * N) return;
    const int64_t A = t / 3;
    const int d = (int)(t - 3 * A);
    double s = 0.0;
    for (int64_t B = 0; B < N; ++B) s += V[3 * (A * N + B) + d] - V[3 * (B * N + A) + d];
    dpos[t] = s;
}

// single-CTA fixed-order sums of Sg and Lp
__global__ void lj_adjoint_sum_kernel(int64_t NN, const double* __restrict__ Sg, const double* __restrict__ Lp,
                                      double eps, double* __restrict__ out) {
    __shared__ double s1[256], s2[256];
    double a = 0.0, b = 0.0;
    for (int64_t i = threadIdx.x; i < NN; i += blockDim.x) {
        a += Sg[i];
        b += Lp[i];
    }
    s1[threadIdx.x] = a;
    s2[threadIdx.x] = b;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) {
            s1[threadIdx.x] += s1[threadIdx.x + w];
            s2[threadIdx.x] += s2[threadIdx.x + w];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out[0] = s1[0];        // ∂L/∂σ
        out[1] = s2[0] / eps;  // ∂L/∂ε
        out[2] = s2[0];        // L
    }
}

}  // namespace

// G = W ×₁ φᵀ ×₂ φᵀ ×₃ φᵀ with W (M×M×M) and φ (n×n, modes [0,M)): output n³
// (doubles for FCB_ADJOINT_FP64, floats otherwise).
int adjoint_g(fcb200_context* h, int precision, const float* d_W, int64_t M, const float* d_phi, int64_t n,
              void* d_Gv, cudaStream_t s) {
    FCB_TRY(h->adj_phiT.ensure(sizeof(float) * (size_t)(n * M)));
    float* phiT = h->adj_phiT.as<float>();
    transpose_kernel<<<(unsigned)((n * M + 255) / 256), 256, 0, s>>>(d_phi, n, M, phiT);
    FCB_CUDA(cudaGetLastError());
    if (precision == FCB_ADJOINT_FP64) {
        // W and φᵀ widened exactly to FP64; intermediates and G in FP64.
        FCB_TRY(h->adj_w64.ensure(sizeof(double) * (size_t)(M * M * M)));
        FCB_TRY(h->adj_phiT64.ensure(sizeof(double) * (size_t)(n * M)));
        FCB_TRY(h->u1_f32.ensure(sizeof(double) * (size_t)(M * M * n)));
        FCB_TRY(h->u2_f32.ensure(sizeof(double) * (size_t)(M * n * n)));
        double* w64 = h->adj_w64.as<double>();
        double* pt64 = h->adj_phiT64.as<double>();
        double* u1 = h->u1_f32.as<double>();
        double* u2 = h->u2_f32.as<double>();
        FCB_TRY(widen_f32_to_f64(d_W, w64, M * M * M, s));
        FCB_TRY(widen_f32_to_f64(phiT, pt64, n * M, s));
        ModeProduct p1{M * M, M, n, M, M, M, M, M * M};
        FCB_TRY(mode_product_f64(w64, pt64, u1, p1, s));
        ModeProduct p2{M * n, M, n, M, M, M, M, M * n};
        FCB_TRY(mode_product_f64(u1, pt64, u2, p2, s));
        ModeProduct p3{n * n, M, n, M, M, n * n, n * n, n * n};
        return mode_product_f64(u2, pt64, static_cast<double*>(d_Gv), p3, s);
    }
    float* d_G = static_cast<float*>(d_Gv);
    if (precision == FCB_MCC3_FP32) {
        FCB_TRY(h->u1_f32.ensure(sizeof(float) * (size_t)(M * M * n)));
        FCB_TRY(h->u2_f32.ensure(sizeof(float) * (size_t)(M * n * n)));
        ModeProduct p1{M * M, M, n, M, M, M, M, M * M};
        FCB_TRY(mode_product_f32(d_W, phiT, h->u1_f32.as<float>(), p1, s));
        ModeProduct p2{M * n, M, n, M, M, M, M, M * n};
        FCB_TRY(mode_product_f32(h->u1_f32.as<float>(), phiT, h->u2_f32.as<float>(), p2, s));
        ModeProduct p3{n * n, M, n, M, M, n * n, n * n, n * n};
        FCB_TRY(mode_product_f32(h->u2_f32.as<float>(), phiT, d_G, p3, s));
        return FCB_OK;
    }
    const int kind = precision == FCB_MCC3_BF16X3 ? 1 : 2;
    const int64_t mp = pad_for(kind, M);
    const size_t esz = kind == 1 ? 2 : 4;
    FCB_TRY(h->adj_w_hi.ensure(esz * (size_t)(mp * M * M)));
    FCB_TRY(h->adj_w_lo.ensure(esz * (size_t)(mp * M * M)));
    FCB_TRY(h->phi_hi.ensure(esz * (size_t)(mp * n)));
    FCB_TRY(h->phi_lo.ensure(esz * (size_t)(mp * n)));
    FCB_TRY(split_operand(d_W, M * M, M, M, h->adj_w_hi.p, h->adj_w_lo.p, mp, kind, s));
    FCB_TRY(split_operand(phiT, n, M, M, h->phi_hi.p, h->phi_lo.p, mp, kind, s));
    FCB_TRY(h->u1_hi.ensure(esz * (size_t)(mp * M * n)));
    FCB_TRY(h->u1_lo.ensure(esz * (size_t)(mp * M * n)));
    FCB_TRY(h->u2_hi.ensure(esz * (size_t)(mp * n * n)));
    FCB_TRY(h->u2_lo.ensure(esz * (size_t)(mp * n * n)));
    ModeProduct p1{M * M, M, n, mp, mp, M, mp, mp * M};
    FCB_TRY(mode_product_tc(h, kind, h->adj_w_hi.p, h->adj_w_lo.p, h->phi_hi.p, h->phi_lo.p, h->u1_hi.p, h->u1_lo.p,
                            kind, p1, s));
    ModeProduct p2{M * n, M, n, mp, mp, M, mp, mp * n};
    FCB_TRY(mode_product_tc(h, kind, h->u1_hi.p, h->u1_lo.p, h->phi_hi.p, h->phi_lo.p, h->u2_hi.p, h->u2_lo.p, kind,
                            p2, s));
    ModeProduct p3{n * n, M, n, mp, mp, n * n, n * n, n * n};
    FCB_TRY(mode_product_tc(h, kind, h->u2_hi.p, h->u2_lo.p, h->phi_hi.p, h->phi_lo.p, d_G, nullptr, 0, p3, s));
    return FCB_OK;
}

int lj_adjoint_pairs(fcb200_context* h, const double* d_pos, int64_t N, const double* d_box, double sigma,
                     double eps, double r_cut, const double* d_masses, const void* d_G, bool g64, double* d_dpos,
                     double* d_scal, cudaStream_t s) {
    const int64_t NN = N * N;
    FCB_TRY(h->adj_pairs.ensure(sizeof(double) * (size_t)(5 * NN)));
    double* V = h->adj_pairs.as<double>();
    double* Sg = V + 3 * NN;
    double* Lp = Sg + NN;
    const unsigned blocks = (unsigned)((NN + 127) / 128);
    if (g64)
        lj_adjoint_pair_kernel<double><<<blocks, 128, 0, s>>>(d_pos, d_box, N, sigma, eps, r_cut * r_cut, d_masses,
                                                              static_cast<const double*>(d_G), V, Sg, Lp);
    else
        lj_adjoint_pair_kernel<float><<<blocks, 128, 0, s>>>(d_pos, d_box, N, sigma, eps, r_cut * r_cut, d_masses,
                                                             static_cast<const float*>(d_G), V, Sg, Lp);
    lj_adjoint_atom_kernel<<<(unsigned)((3 * N + 127) / 128), 128, 0, s>>>(N, V, d_dpos);
    lj_adjoint_sum_kernel<<<1, 256, 0, s>>>(NN, Sg, Lp, eps, d_scal);
    FCB_CUDA(cudaGetLastError());
    return FCB_OK;
}

}  // namespace fcb
