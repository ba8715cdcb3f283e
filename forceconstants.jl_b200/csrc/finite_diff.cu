// Finite-difference force constants on the GPU: an independent check of the
// analytical (LJ) and automatically differentiated (SW) assemblies.
//
// Reference semantics (ForceConstants.jl):
//   third_order_finite_diff_eng      src/finitediff/third_order_FD.jl:43-113
//   second_order! (FiniteDiffCalculator), second_order_finite_diff_single
//                                    src/finitediff/second_order_FD.jl:3-79
//   energy_loop (LJ, SW)             src/finitediff/finitediff_helper.jl:3-64
//   ASR!(ifc2)                       src/asr.jl:3-17
//
// The reference evaluates whole-cell energies at the stencil points.  Every
// stencil's weights sum to zero, so the terms of the energy that do not
// involve a displaced atom cancel exactly; here each stencil point sums only
// the terms that involve one of the element's atoms (LJ: pairs; SW: pairs and
// three-body terms centred anywhere), evaluated at that point's positions.
// The combination is the reference's formula with far less cancellation and
// O(neighbourhood) instead of O(N²) work per point.  One warp per element;
// lanes split the atom scans, and the warp reduction order is fixed, so
// results are deterministic.
//
// The reference's stencils are reproduced as written, including what they
// leave out: the two-same pattern (i,α,j,β,i,γ) displaces only (i,α) and
// (j,β), the all-same pattern only (i,α); elements with i = j ≠ k or
// j = k ≠ i have no stencil there and come back NaN.
#include "fcb200_internal.cuh"

namespace fcb {
namespace {

constexpr int FD_WARPS = 4;    // warps per block
constexpr int FD_CAP = 128;    // SW: centres and neighbours listed per warp

struct FdArgs {
    const double* pos;
    const double* box;
    int N;
    int kind;  // 0 LJ, 1 SW
    double sigma, eps, rc;
    double h;
};

// SW parameters of the reference (SW.jl:32-33, LAMMPS Si.sw).
constexpr double SW_EPS = 2.1683, SW_SIGMA = 2.0951, SW_A = 1.80, SW_LAMBDA = 21.0, SW_GAMMA = 1.20;
constexpr double SW_ACOEF = 7.049556277, SW_BCOEF = 0.6022245584, SW_P = 4.0, SW_Q = 0.0;

struct Displaced {
    int n;          // distinct atoms displaced (≤ 3)
    int atom[3];
    double p[3][3]; // their positions at this stencil point
};

__device__ __forceinline__ void mirror(double r[3], const double* box) {
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        if (r[d] > box[d] / 2.0) r[d] -= box[d];
        else if (r[d] < -box[d] / 2.0) r[d] += box[d];
    }
}

__device__ __forceinline__ int slot_in(const Displaced& D, int x) {
    for (int t = 0; t < D.n; ++t)
        if (D.atom[t] == x) return t;
    return -1;
}

__device__ __forceinline__ void pos_of(const FdArgs& a, const Displaced& D, int x, double out[3]) {
    const int t = slot_in(D, x);
    if (t >= 0) {
        out[0] = D.p[t][0];
        out[1] = D.p[t][1];
        out[2] = D.p[t][2];
    } else {
        out[0] = a.pos[3 * x];
        out[1] = a.pos[3 * x + 1];
        out[2] = a.pos[3 * x + 2];
    }
}

__device__ __forceinline__ double lj_pot(const FdArgs& a, double dist) {
    const double k = pow(a.sigma / dist, 6.0);
    return 4.0 * a.eps * k * (k - 1.0);
}

__device__ __forceinline__ double sw_pair(double dist) {
    return SW_ACOEF * SW_EPS * (SW_BCOEF * pow(SW_SIGMA / dist, SW_P) - pow(SW_SIGMA / dist, SW_Q)) *
           exp(SW_SIGMA / (dist - SW_A * SW_SIGMA));
}

__device__ __forceinline__ double sw_three(const double rij[3], const double rik[3], double dij, double dik) {
    const double cos0 = -1.0 / 3.0;
    const double rc = SW_A * SW_SIGMA, gs = SW_SIGMA * SW_GAMMA, le = SW_EPS * SW_LAMBDA;
    const double c = (rij[0] * rik[0] + rij[1] * rik[1] + rij[2] * rik[2]) / (dij * dik);
    return le * ((c - cos0) * (c - cos0)) * exp(gs / (dij - rc)) * exp(gs / (dik - rc));
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Pair terms with at least one displaced atom (each unordered pair once).
__device__ double local_pairs(const FdArgs& a, const Displaced& D, int lane) {
    double s = 0.0;
    const double rc2 = a.kind == 0 ? a.rc * a.rc : (SW_A * SW_SIGMA) * (SW_A * SW_SIGMA);
    for (int t = 0; t < D.n; ++t) {
        const int x = D.atom[t];
        for (int b = lane; b < a.N; b += 32) {
            if (b == x) continue;
            const int tb = slot_in(D, b);
            if (tb >= 0 && b < x) continue;  // pair inside D counted from its lower atom
            double pb[3];
            pos_of(a, D, b, pb);
            double r[3] = {D.p[t][0] - pb[0], D.p[t][1] - pb[1], D.p[t][2] - pb[2]};
            mirror(r, a.box);
            const double d2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
            if (a.kind == 0) {
                const double dist = sqrt(d2);
                if (dist < a.rc) s += lj_pot(a, dist);
            } else if (d2 < rc2) {
                s += sw_pair(sqrt(d2));
            }
        }
    }
    return s;
}

// SW three-body terms (centre i; pair j < k of i's neighbours) with any of
// i, j, k displaced.  A centre outside D must be a neighbour of a displaced
// atom; centres and neighbour lists are compacted into this warp's shared
// lists.  Returns NaN through *overflow when a list exceeds FD_CAP.
__device__ double local_triplets(const FdArgs& a, const Displaced& D, int lane, int* centres, int* nbrs,
                                 bool* overflow) {
    const double rc = SW_A * SW_SIGMA, rc2 = rc * rc;
    int nc = 0;
    for (int t = 0; t < D.n; ++t) {
        if (lane == 0) centres[nc] = D.atom[t];
        ++nc;
    }
    for (int b0 = 0; b0 < a.N; b0 += 32) {
        const int b = b0 + lane;
        bool near = false;
        if (b < a.N && slot_in(D, b) < 0) {
            double pb[3] = {a.pos[3 * b], a.pos[3 * b + 1], a.pos[3 * b + 2]};
            for (int t = 0; t < D.n && !near; ++t) {
                double r[3] = {D.p[t][0] - pb[0], D.p[t][1] - pb[1], D.p[t][2] - pb[2]};
                mirror(r, a.box);
                near = r[0] * r[0] + r[1] * r[1] + r[2] * r[2] < rc2;
            }
        }
        const unsigned m = __ballot_sync(0xffffffffu, near);
        const int slot = nc + __popc(m & ((1u << lane) - 1u));
        if (near && slot < FD_CAP) centres[slot] = b;
        nc += __popc(m);
    }
    __syncwarp();
    if (nc > FD_CAP) {
        *overflow = true;
        return 0.0;
    }
    double s = 0.0;
    for (int ci = 0; ci < nc; ++ci) {
        const int i = centres[ci];
        double pi[3];
        pos_of(a, D, i, pi);
        const bool i_in = slot_in(D, i) >= 0;
        int nn = 0;
        for (int b0 = 0; b0 < a.N; b0 += 32) {
            const int b = b0 + lane;
            bool in = false;
            if (b < a.N && b != i) {
                double pb[3];
                pos_of(a, D, b, pb);
                double r[3] = {pi[0] - pb[0], pi[1] - pb[1], pi[2] - pb[2]};
                mirror(r, a.box);
                in = r[0] * r[0] + r[1] * r[1] + r[2] * r[2] < rc2;
            }
            const unsigned m = __ballot_sync(0xffffffffu, in);
            const int slot = nn + __popc(m & ((1u << lane) - 1u));
            if (in && slot < FD_CAP) nbrs[slot] = b;
            nn += __popc(m);
        }
        __syncwarp();
        if (nn > FD_CAP) {
            *overflow = true;
            return 0.0;
        }
        const int npairs = nn * (nn - 1) / 2;
        for (int q = lane; q < npairs; q += 32) {
            // q -> (u < v) over the ascending neighbour list
            int u = 0, rem = q;
            while (rem >= nn - 1 - u) {
                rem -= nn - 1 - u;
                ++u;
            }
            const int v = u + 1 + rem;
            const int j = nbrs[u], k = nbrs[v];
            if (!(i_in || slot_in(D, j) >= 0 || slot_in(D, k) >= 0)) continue;
            double pj[3], pk[3];
            pos_of(a, D, j, pj);
            pos_of(a, D, k, pk);
            double rij[3] = {pi[0] - pj[0], pi[1] - pj[1], pi[2] - pj[2]};
            double rik[3] = {pi[0] - pk[0], pi[1] - pk[1], pi[2] - pk[2]};
            mirror(rij, a.box);
            mirror(rik, a.box);
            const double dij = sqrt(rij[0] * rij[0] + rij[1] * rij[1] + rij[2] * rij[2]);
            const double dik = sqrt(rik[0] * rik[0] + rik[1] * rik[1] + rik[2] * rik[2]);
            s += sw_three(rij, rik, dij, dik);
        }
        __syncwarp();
    }
    return s;
}

// Sum of the terms involving D at one stencil point.
__device__ double local_energy(const FdArgs& a, const Displaced& D, int lane, int* centres, int* nbrs,
                               bool* overflow) {
    double s = local_pairs(a, D, lane);
    if (a.kind == 1) s += local_triplets(a, D, lane, centres, nbrs, overflow);
    return warp_sum(s);
}

// A stencil: nt displaced (atom, component) slots, nc points with weights.
struct Stencil {
    int nt, nc;
    int atom[3], comp[3];
    double step[8][3];
    double w[8];
    double scale;
};

__device__ double run_stencil(const FdArgs& a, const Stencil& S, int lane, int* centres, int* nbrs,
                              bool* overflow) {
    Displaced D;
    D.n = 0;
    for (int t = 0; t < S.nt; ++t)
        if (slot_in(D, S.atom[t]) < 0) D.atom[D.n++] = S.atom[t];
    double acc = 0.0;
    for (int c = 0; c < S.nc; ++c) {
        for (int t = 0; t < D.n; ++t)
            for (int d = 0; d < 3; ++d) D.p[t][d] = a.pos[3 * D.atom[t] + d];
        for (int t = 0; t < S.nt; ++t) D.p[slot_in(D, S.atom[t])][S.comp[t]] += S.step[c][t];
        acc += S.w[c] * local_energy(a, D, lane, centres, nbrs, overflow);
    }
    return S.scale * acc;
}

__device__ bool third_stencil(const int64_t* e, double h, Stencil& S) {
    const int a1 = (int)e[0], a2 = (int)e[2], a3 = (int)e[4];
    const int c1 = (int)e[1], c2 = (int)e[3], c3 = (int)e[5];
    if (a1 != a2 && a2 != a3 && a1 != a3) {
        const double cb[8][3] = {{h, h, h},    {h, -h, -h}, {-h, -h, h}, {-h, h, -h},
                                 {-h, -h, -h}, {-h, h, h},  {h, -h, h},  {h, h, -h}};
        const double w[8] = {1, 1, 1, 1, -1, -1, -1, -1};
        S.nt = 3;
        S.nc = 8;
        S.atom[0] = a1, S.atom[1] = a2, S.atom[2] = a3;
        S.comp[0] = c1, S.comp[1] = c2, S.comp[2] = c3;
        for (int c = 0; c < 8; ++c) {
            for (int t = 0; t < 3; ++t) S.step[c][t] = cb[c][t];
            S.w[c] = w[c];
        }
        S.scale = 1.0 / (8.0 * (h * h * h));
        return true;
    }
    if (a1 == a2 && a2 == a3) {
        const double cb[4] = {-2 * h, -h, h, 2 * h};
        const double w[4] = {-1, 2, -2, 1};
        S.nt = 1;
        S.nc = 4;
        S.atom[0] = a1;
        S.comp[0] = c1;
        for (int c = 0; c < 4; ++c) {
            S.step[c][0] = cb[c];
            S.w[c] = w[c];
        }
        S.scale = 1.0 / (2.0 * (h * h * h));
        return true;
    }
    if (a1 != a2 && a1 == a3) {
        const double cb[6][2] = {{h, h}, {-h, h}, {0, -h}, {-h, -h}, {h, -h}, {0, h}};
        const double w[6] = {1, 1, 2, -1, -1, -2};
        S.nt = 2;
        S.nc = 6;
        S.atom[0] = a1, S.atom[1] = a2;
        S.comp[0] = c1, S.comp[1] = c2;
        for (int c = 0; c < 6; ++c) {
            S.step[c][0] = cb[c][0];
            S.step[c][1] = cb[c][1];
            S.w[c] = w[c];
        }
        S.scale = 1.0 / (2.0 * (h * h * h));
        return true;
    }
    return false;
}

__global__ void __launch_bounds__(32 * FD_WARPS) fd_third_kernel(FdArgs a, const int64_t* __restrict__ elems,
                                                                 int64_t m, double* __restrict__ out) {
    __shared__ int lists[FD_WARPS][2][FD_CAP];
    const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t e = (int64_t)blockIdx.x * FD_WARPS + wib;
    if (e >= m) return;
    Stencil S;
    double v = nan("");
    if (third_stencil(elems + 6 * e, a.h, S)) {
        bool overflow = false;
        v = run_stencil(a, S, lane, lists[wib][0], lists[wib][1], &overflow);
        if (overflow) v = nan("");
    }
    if (lane == 0) out[e] = v;
}

// FD IFC2: one warp per ordered pair (i < j) within the calculator's cutoff at
// the base positions; the 9 (α, β) entries and their transposes.
__global__ void __launch_bounds__(32 * FD_WARPS) fd_second_kernel(FdArgs a, double calc_rc2, double* __restrict__ ifc2,
                                                                  int* __restrict__ status) {
    __shared__ int lists[FD_WARPS][2][FD_CAP];
    const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t w = (int64_t)blockIdx.x * FD_WARPS + wib;
    const int64_t N = a.N, n = 3 * N;
    if (w >= N * N) return;
    const int i = (int)(w / N), j = (int)(w % N);
    if (j <= i) return;
    double r[3] = {a.pos[3 * i] - a.pos[3 * j], a.pos[3 * i + 1] - a.pos[3 * j + 1], a.pos[3 * i + 2] - a.pos[3 * j + 2]};
    mirror(r, a.box);
    if (!(r[0] * r[0] + r[1] * r[1] + r[2] * r[2] < calc_rc2)) return;
    const double h = a.h;
    Stencil S;
    S.nt = 2;
    S.nc = 4;
    S.atom[0] = i, S.atom[1] = j;
    const double cb[4][2] = {{h, h}, {-h, -h}, {h, -h}, {-h, h}};
    const double wt[4] = {1, 1, -1, -1};
    for (int c = 0; c < 4; ++c) {
        S.step[c][0] = cb[c][0];
        S.step[c][1] = cb[c][1];
        S.w[c] = wt[c];
    }
    S.scale = 1.0 / (4.0 * h * h);
    bool overflow = false;
    for (int al = 0; al < 3; ++al)
        for (int be = 0; be < 3; ++be) {
            S.comp[0] = al, S.comp[1] = be;
            const double v = run_stencil(a, S, lane, lists[wib][0], lists[wib][1], &overflow);
            if (lane == 0) {
                ifc2[(3 * i + al) + n * (3 * j + be)] = v;
                ifc2[(3 * j + be) + n * (3 * i + al)] = v;
            }
        }
    if (overflow && lane == 0) atomicCAS(status, 0, DEV_FD_OVERFLOW);
}

// ASR!(ifc2) (asr.jl:3-17): diagonal blocks = minus the sums of the rows'
// off-diagonal blocks, in ascending atom order.
__global__ void fd_asr2_kernel(double* __restrict__ ifc2, int N) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 9 * N) return;
    const int i = t / 9, al = (t % 9) / 3, be = t % 3;
    const int64_t n = 3 * (int64_t)N;
    double s = 0.0;
    for (int j = 0; j < N; ++j)
        if (j != i) s += ifc2[(3 * i + al) + n * (3 * j + be)];
    ifc2[(3 * i + al) + n * (3 * i + be)] = -s;
}

// apply_tols! (helper_funcs.jl:20-27): |x| < tol -> 0.
__global__ void fd_tol_kernel(double* __restrict__ v, int64_t count, double tol) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < count; t += stride)
        if (fabs(v[t]) < tol) v[t] = 0.0;
}

}  // namespace

int fd_third_order_launch(const double* d_pos, const double* d_box, int64_t N, int kind, double sigma, double eps,
                          double r_cut, const int64_t* d_elems, int64_t m, double h, double* d_out, cudaStream_t s) {
    if (m == 0) return FCB_OK;
    FdArgs a{d_pos, d_box, (int)N, kind, sigma, eps, r_cut, h};
    const int64_t blocks = (m + FD_WARPS - 1) / FD_WARPS;
    fd_third_kernel<<<(unsigned)blocks, 32 * FD_WARPS, 0, s>>>(a, d_elems, m, d_out);
    FCB_CUDA(cudaGetLastError());
    return FCB_OK;
}

int fd_second_order_launch(const double* d_pos, const double* d_box, int64_t N, int kind, double sigma, double eps,
                           double r_cut, double calc_r_cut, double tol, double h, double* d_ifc2, int* d_status,
                           cudaStream_t s) {
    const int64_t n = 3 * N;
    FCB_CUDA(cudaMemsetAsync(d_ifc2, 0, sizeof(double) * n * n, s));
    FdArgs a{d_pos, d_box, (int)N, kind, sigma, eps, r_cut, h};
    const int64_t warps = N * N;
    fd_second_kernel<<<(unsigned)((warps + FD_WARPS - 1) / FD_WARPS), 32 * FD_WARPS, 0, s>>>(
        a, calc_r_cut * calc_r_cut, d_ifc2, d_status);
    FCB_CUDA(cudaGetLastError());
    fd_asr2_kernel<<<(unsigned)((9 * N + 127) / 128), 128, 0, s>>>(d_ifc2, (int)N);
    FCB_CUDA(cudaGetLastError());
    if (tol > 0.0) {
        int64_t blocks = (n * n + 255) / 256;
        if (blocks > 4096) blocks = 4096;
        fd_tol_kernel<<<(unsigned)blocks, 256, 0, s>>>(d_ifc2, n * n, tol);
        FCB_CUDA(cudaGetLastError());
    }
    return FCB_OK;
}

}  // namespace fcb
