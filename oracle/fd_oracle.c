/*
 * ORACLE (test infrastructure only): CPU restatement of ForceConstants.jl's
 * finite-difference path.  Not a product path; only tests/ use it.
 *
 *   energy_loop(::PairPotential, ...)           src/finitediff/finitediff_helper.jl:3-21
 *   energy_loop(::StillingerWeberSilicon, ...)  src/finitediff/finitediff_helper.jl:24-64
 *   third_order_finite_diff_eng                 src/finitediff/third_order_FD.jl:43-113
 *   second_order! (FiniteDiffCalculator) + second_order_finite_diff_single
 *                                               src/finitediff/second_order_FD.jl:3-79
 *   LJ potential 4ε k(k-1), k = (σ/r)^6         src/interactions/LennardJones.jl
 *   SW Φ₂, Φ₃_si, parameters (LAMMPS Si.sw)     src/interactions/SW.jl:29-83
 *
 * Energies are whole-cell totals in the reference's loop order, so the stencil
 * combinations carry the same cancellation as the reference.  Indices are
 * 0-based (atom, component).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

static void mirror(double r[3], const double* box) {
    for (int d = 0; d < 3; ++d) {
        if (r[d] > box[d] / 2.0) r[d] -= box[d];
        else if (r[d] < -box[d] / 2.0) r[d] += box[d];
    }
}

typedef struct {
    int kind;  /* 0 = LJ, 1 = SW */
    double sigma, eps, r_cut;
} FdPot;

/* SW parameters of the reference (SW.jl:32-33). */
static const double SW_EPS = 2.1683, SW_SIGMA = 2.0951, SW_A = 1.80, SW_LAMBDA = 21.0, SW_GAMMA = 1.20;
static const double SW_A_COEF = 7.049556277, SW_B_COEF = 0.6022245584, SW_P = 4.0, SW_Q = 0.0;

static double lj_energy(const double* pos, int64_t N, const double* box, double sigma, double eps, double rc) {
    double U = 0.0;
    for (int64_t i = 0; i < N; ++i)
        for (int64_t j = i + 1; j < N; ++j) {
            double r[3] = {pos[3 * i] - pos[3 * j], pos[3 * i + 1] - pos[3 * j + 1], pos[3 * i + 2] - pos[3 * j + 2]};
            mirror(r, box);
            const double dist = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
            if (dist < rc) {
                const double k = pow(sigma / dist, 6.0);
                U += 4.0 * eps * k * (k - 1.0);
            }
        }
    return U;
}

static double sw_energy(const double* pos, int64_t N, const double* box) {
    const double cos0 = -1.0 / 3.0;
    const double rc = SW_A * SW_SIGMA, gs = SW_SIGMA * SW_GAMMA, le = SW_EPS * SW_LAMBDA;
    const double rc2 = rc * rc;
    double U = 0.0;
    for (int64_t i = 0; i < N; ++i)
        for (int64_t j = 0; j < N; ++j) {
            if (i == j) continue;
            double rij[3] = {pos[3 * i] - pos[3 * j], pos[3 * i + 1] - pos[3 * j + 1], pos[3 * i + 2] - pos[3 * j + 2]};
            mirror(rij, box);
            const double dij2 = rij[0] * rij[0] + rij[1] * rij[1] + rij[2] * rij[2];
            if (!(dij2 < rc2)) continue;
            const double dij = sqrt(dij2);
            if (i < j)
                U += SW_A_COEF * SW_EPS * (SW_B_COEF * pow(SW_SIGMA / dij, SW_P) - pow(SW_SIGMA / dij, SW_Q)) *
                     exp(SW_SIGMA / (dij - SW_A * SW_SIGMA));
            for (int64_t k = j + 1; k < N; ++k) {
                if (k == i) continue;
                double rik[3] = {pos[3 * i] - pos[3 * k], pos[3 * i + 1] - pos[3 * k + 1],
                                 pos[3 * i + 2] - pos[3 * k + 2]};
                mirror(rik, box);
                const double dik2 = rik[0] * rik[0] + rik[1] * rik[1] + rik[2] * rik[2];
                if (dik2 < rc2) {
                    const double dik = sqrt(dik2);
                    const double c = (rij[0] * rik[0] + rij[1] * rik[1] + rij[2] * rik[2]) / (dij * dik);
                    U += le * ((c - cos0) * (c - cos0)) * exp(gs / (dij - rc)) * exp(gs / (dik - rc));
                }
            }
        }
    return U;
}

static double energy(const FdPot* p, const double* pos, int64_t N, const double* box) {
    return p->kind == 0 ? lj_energy(pos, N, box, p->sigma, p->eps, p->r_cut) : sw_energy(pos, N, box);
}

/* Energies of the stencil points: combos[c][t] displaces (atom[t], comp[t]). */
static double stencil(const FdPot* p, double* pos, int64_t N, const double* box, const int64_t* atom,
                      const int* comp, int nt, const double (*combos)[3], const double* w, int nc) {
    double acc = 0.0;
    for (int c = 0; c < nc; ++c) {
        for (int t = 0; t < nt; ++t) pos[3 * atom[t] + comp[t]] += combos[c][t];
        const double E = energy(p, pos, N, box);
        for (int t = 0; t < nt; ++t) pos[3 * atom[t] + comp[t]] -= combos[c][t];
        acc += w[c] * E;
    }
    return acc;
}

/* third_order_finite_diff_eng for m elements e = (i,α,j,β,k,γ); NaN where the
 * reference has no stencil (i == j != k or j == k != i). */
void oracle_fd_third_order(int kind, const double* pos0, int64_t N, const double* box, double sigma, double eps,
                           double r_cut, const int64_t* elems, int64_t m, double h, double* out) {
    FdPot p = {kind, sigma, eps, r_cut};
    double* pos = (double*)malloc(sizeof(double) * 3 * N);
    memcpy(pos, pos0, sizeof(double) * 3 * N);
    for (int64_t e = 0; e < m; ++e) {
        const int64_t* q = elems + 6 * e;
        const int64_t a1 = q[0], a2 = q[2], a3 = q[4];
        const int c1 = (int)q[1], c2 = (int)q[3], c3 = (int)q[5];
        if (a1 != a2 && a2 != a3 && a1 != a3) {
            const double cb[8][3] = {{h, h, h},   {h, -h, -h},  {-h, -h, h}, {-h, h, -h},
                                     {-h, -h, -h}, {-h, h, h}, {h, -h, h},  {h, h, -h}};
            const double w[8] = {1, 1, 1, 1, -1, -1, -1, -1};
            const int64_t at[3] = {a1, a2, a3};
            const int cp[3] = {c1, c2, c3};
            out[e] = (1.0 / (8.0 * (h * h * h))) * stencil(&p, pos, N, box, at, cp, 3, cb, w, 8);
        } else if (a1 == a2 && a2 == a3) {
            const double cb[4][3] = {{-2 * h, 0, 0}, {-h, 0, 0}, {h, 0, 0}, {2 * h, 0, 0}};
            const double w[4] = {-1, 2, -2, 1};
            const int64_t at[1] = {a1};
            const int cp[1] = {c1};
            out[e] = (1.0 / (2.0 * (h * h * h))) * stencil(&p, pos, N, box, at, cp, 1, cb, w, 4);
        } else if (a1 != a2 && a1 == a3) {
            const double cb[6][3] = {{h, h, 0}, {-h, h, 0}, {0, -h, 0}, {-h, -h, 0}, {h, -h, 0}, {0, h, 0}};
            const double w[6] = {1, 1, 2, -1, -1, -2};
            const int64_t at[2] = {a1, a2};
            const int cp[2] = {c1, c2};
            out[e] = (1.0 / (2.0 * (h * h * h))) * stencil(&p, pos, N, box, at, cp, 2, cb, w, 6);
        } else {
            out[e] = NAN;
        }
    }
    free(pos);
}

/* second_order! with the FiniteDiffCalculator: pairs i<j within calc_rcut
 * (base positions), 4-point energy stencil, symmetric fill, then ASR (the
 * diagonal 3×3 blocks are minus the sums of their rows' off-diagonal blocks). */
void oracle_fd_second_order(int kind, const double* pos0, int64_t N, const double* box, double sigma, double eps,
                            double r_cut, double calc_rcut, double h, double* ifc2) {
    FdPot p = {kind, sigma, eps, r_cut};
    const int64_t n = 3 * N;
    double* pos = (double*)malloc(sizeof(double) * 3 * N);
    memcpy(pos, pos0, sizeof(double) * 3 * N);
    memset(ifc2, 0, sizeof(double) * n * n);
    const double rc2 = calc_rcut * calc_rcut;
    for (int64_t i = 0; i < N; ++i)
        for (int64_t j = i + 1; j < N; ++j) {
            double r[3] = {pos0[3 * i] - pos0[3 * j], pos0[3 * i + 1] - pos0[3 * j + 1],
                           pos0[3 * i + 2] - pos0[3 * j + 2]};
            mirror(r, box);
            if (!(r[0] * r[0] + r[1] * r[1] + r[2] * r[2] < rc2)) continue;
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) {
                    const double cb[4][3] = {{h, h, 0}, {-h, -h, 0}, {h, -h, 0}, {-h, h, 0}};
                    const double w[4] = {1, 1, -1, -1};
                    const int64_t at[2] = {i, j};
                    const int cp[2] = {a, b};
                    const double v = (1.0 / (4.0 * h * h)) * stencil(&p, pos, N, box, at, cp, 2, cb, w, 4);
                    ifc2[(3 * i + a) + n * (3 * j + b)] = v;
                    ifc2[(3 * j + b) + n * (3 * i + a)] = v;
                }
        }
    for (int64_t i = 0; i < N; ++i)
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) {
                double s = 0.0;
                for (int64_t j = 0; j < N; ++j)
                    if (j != i) s += ifc2[(3 * i + a) + n * (3 * j + b)];
                ifc2[(3 * i + a) + n * (3 * i + b)] = -s;
            }
    free(pos);
}

double oracle_fd_energy(int kind, const double* pos, int64_t N, const double* box, double sigma, double eps,
                        double r_cut) {
    FdPot p = {kind, sigma, eps, r_cut};
    return energy(&p, pos, N, box);
}
