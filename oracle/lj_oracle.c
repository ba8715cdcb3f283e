/*
 * ORACLE — test infrastructure only.  Nothing in the product imports, links or
 * calls this file; only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg use it, and only as the checker.
 *
 * CPU restatement of the ForceConstants.jl Lennard-Jones force-constant path
 * (reference paths are relative to the ForceConstants.jl repository root):
 *
 *   nearest_mirror!            src/helper_funcs.jl:7-17
 *   apply_tols!                src/helper_funcs.jl:20-27
 *   LJ Φ′ Φ″ Φ‴ Φ⁗             src/interactions/LennardJones.jl:38-56
 *   ϕ₂                         src/analytical/second_order_analytical.jl:44-51
 *   second_order!  (pairs)     src/analytical/second_order_analytical.jl:3-42
 *   ASR!(ifc2)                 src/asr.jl:3-17
 *   ϕ₃                         src/analytical/third_order_analytical.jl:216-224
 *   third_order!   (pairs)     src/analytical/third_order_analytical.jl:4-69
 *   ASR!(ifc3)                 src/asr.jl:19-40
 *   mass_weight_third_order!   src/analytical/third_order_analytical.jl:185-214
 *   third_order  (front)       src/ifc.jl:20-35 (zeros → third_order! → apply_tols!)
 *
 * Loop order and memory order follow the reference (pair loop i<j with the
 * 6-way permutation scatter, the strided ASR sum over the slowest index, the
 * serial 6-deep mass-weight loop), because bench.py times this file as the
 * reference's CPU path.  OpenMP over the outer atom loop stands in for the
 * reference's OhMyThreads `@tasks` over i.
 *
 * Floating-point evaluation order: every expression is evaluated left to
 * right exactly as the reference writes it, and compiled with
 * -ffp-contract=off so that no multiply-add is fused.  Integer powers use the
 * sequential product chain fc_ipow() below (the product kernel uses the same
 * chain), so the device result can be compared bit for bit.
 *
 * Layouts: positions pos[3*a + x] (column-major 3×N, Julia's Vector{SVector});
 * dense tensors are column-major (Julia) with DoF index 3*a + α, so
 * Ψ[ii,jj,kk] lives at ii + n*(jj + n*kk), n = 3N.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

static double fc_ipow(double x, int n) {
    double p = x;
    for (int i = 1; i < n; ++i) p = p * x;
    return p;
}

/* helper_funcs.jl:7-17 — single minimum image, strict comparisons. */
void oracle_nearest_mirror(double r[3], const double box[3]) {
    for (int d = 0; d < 3; ++d) {
        if (r[d] > box[d] / 2.0) r[d] -= box[d];
        else if (r[d] < -box[d] / 2.0) r[d] += box[d];
    }
}

/* LennardJones.jl:38-56.  d[0..3] = Φ′, Φ″, Φ‴, Φ⁗ at distance r. */
void oracle_lj_derivs(double sigma, double eps, double r, double d[4]) {
    double s6 = fc_ipow(sigma, 6), s12 = fc_ipow(sigma, 12);
    d[0] = (-1.0 * eps) * (48.0 * (s12 / fc_ipow(r, 13)) - 24.0 * (s6 / fc_ipow(r, 7)));
    d[1] = (4.0 * eps) * ((156.0 * (s12 / fc_ipow(r, 14))) - (42.0 * (s6 / fc_ipow(r, 8))));
    d[2] = (-4.0 * eps) * ((2184.0 * (s12 / fc_ipow(r, 15))) - (336.0 * (s6 / fc_ipow(r, 9))));
    d[3] = (4.0 * eps) * ((32760.0 * (s12 / fc_ipow(r, 16))) - (3024.0 * (s6 / fc_ipow(r, 10))));
}

/* third_order_analytical.jl:216-224 */
double oracle_phi3(const double d[4], double rn, const double r[3], int a, int b, int c) {
    double t1 = ((r[a] * r[b]) * r[c]) / fc_ipow(rn, 3);
    double t2 = ((d[2] - ((3.0 * d[1]) / rn)) + ((3.0 * d[0]) / fc_ipow(rn, 2)));
    double s = 0.0;
    if (b == c) s = s + r[a];
    if (c == a) s = s + r[b];
    if (a == b) s = s + r[c];
    double t3 = s / fc_ipow(rn, 2);
    double t4 = d[1] - (d[0] / rn);
    return (t1 * t2) + (t3 * t4);
}

/* second_order_analytical.jl:44-51 */
double oracle_phi2(const double d[4], double rn, const double r[3], int a, int b) {
    double t = ((r[a] * r[b]) / fc_ipow(rn, 2)) * (d[1] - (d[0] / rn));
    return (a == b) ? t + (d[0] / rn) : t;
}

/* helper_funcs.jl:20-27 */
void oracle_apply_tols(double* arr, int64_t len, double tol) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < len; ++i)
        if (fabs(arr[i]) < tol) arr[i] = 0.0;
}

/* asr.jl:3-17 */
void oracle_asr2(double* ifc2, int64_t N) {
    const int64_t n = 3 * N;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < N; ++i)
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) {
                int64_t ii = 3 * i + a, jj = 3 * i + b;
                double s = 0.0;
                for (int64_t c = b; c < n; c += 3) s += ifc2[ii + n * c];
                ifc2[ii + n * jj] = -1.0 * s;
            }
}

/* second_order_analytical.jl:3-42 — pair loop, then ASR.  ifc2 must be zero. */
void oracle_second_order_lj(const double* pos, int64_t N, const double box[3], double sigma,
                            double eps, double r_cut, double* ifc2) {
    const int64_t n = 3 * N;
    const double rc2 = r_cut * r_cut;
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t i = 0; i < N; ++i) {
        for (int64_t j = i + 1; j < N; ++j) {
            double r[3];
            for (int x = 0; x < 3; ++x) r[x] = pos[3 * i + x] - pos[3 * j + x];
            oracle_nearest_mirror(r, box);
            double d2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
            if (d2 < rc2) {
                double rn = sqrt(d2), d[4];
                oracle_lj_derivs(sigma, eps, rn, d);
                for (int a = 0; a < 3; ++a)
                    for (int b = 0; b < 3; ++b) {
                        int64_t ii = 3 * i + a, jj = 3 * j + b;
                        ifc2[ii + n * jj] = -oracle_phi2(d, rn, r, a, b);
                        ifc2[jj + n * ii] = ifc2[ii + n * jj];
                    }
            }
        }
    }
    oracle_asr2(ifc2, N);
}

/* asr.jl:19-40 — zero the (i,j,i) entry, then overwrite it with minus the
 * strided sum over the third index (γ:3:end), in ascending order. */
void oracle_asr3(double* psi, int64_t N) {
    const int64_t n = 3 * N, n2 = n * n;
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t i = 0; i < N; ++i)
        for (int64_t j = 0; j < N; ++j)
            for (int a = 0; a < 3; ++a) {
                int64_t ii = 3 * i + a;
                for (int b = 0; b < 3; ++b) {
                    int64_t jj = 3 * j + b;
                    for (int c = 0; c < 3; ++c) {
                        int64_t kk = 3 * i + c;
                        double* col = psi + ii + n * jj;
                        col[n2 * kk] = 0.0;
                        double s = 0.0;
                        for (int64_t k = c; k < n; k += 3) s += col[n2 * k];
                        col[n2 * kk] = -s;
                    }
                }
            }
}

/* third_order_analytical.jl:4-69 — pair loop with the 6-way permutation
 * scatter for both pair directions, then ASR!.  psi (n³) must be zero. */
void oracle_third_order_lj_pairs(const double* pos, int64_t N, const double box[3], double sigma,
                                 double eps, double r_cut, double* psi) {
    const int64_t n = 3 * N;
    const double rc2 = r_cut * r_cut;
#define PSI(x, y, z) psi[(x) + n * ((y) + n * (int64_t)(z))]
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t i = 0; i < N; ++i) {
        for (int64_t j = i + 1; j < N; ++j) {
            for (int dir = 0; dir < 2; ++dir) {
                double r[3];
                for (int x = 0; x < 3; ++x)
                    r[x] = dir == 0 ? pos[3 * i + x] - pos[3 * j + x] : pos[3 * j + x] - pos[3 * i + x];
                oracle_nearest_mirror(r, box);
                double d2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
                if (!(d2 < rc2)) continue;
                double rn = sqrt(d2), d[4];
                oracle_lj_derivs(sigma, eps, rn, d);
                for (int a = 0; a < 3; ++a)
                    for (int b = 0; b < 3; ++b)
                        for (int c = 0; c < 3; ++c) {
                            double val = -oracle_phi3(d, rn, r, a, b, c);
                            int64_t ii, jj, kk;
                            if (dir == 0) { ii = 3 * i + a; jj = 3 * i + b; kk = 3 * j + c; }
                            else          { ii = 3 * i + a; jj = 3 * j + b; kk = 3 * j + c; }
                            PSI(ii, jj, kk) = val; PSI(ii, kk, jj) = val;
                            PSI(jj, kk, ii) = val; PSI(jj, ii, kk) = val;
                            PSI(kk, ii, jj) = val; PSI(kk, jj, ii) = val;
                        }
            }
        }
    }
#undef PSI
    oracle_asr3(psi, N);
}

/* ifc.jl:20-35: zeros → third_order! → apply_tols!  (returns 0, or -1 when
 * the reference's `r_cut < L` assertion would fire). */
int oracle_third_order_lj(const double* pos, int64_t N, const double box[3], double sigma,
                          double eps, double r_cut, double tol, double* psi) {
    for (int d = 0; d < 3; ++d)
        if (!(r_cut < box[d])) return -1;
    const int64_t n = 3 * N;
    memset(psi, 0, sizeof(double) * (size_t)(n * n * n));
    oracle_third_order_lj_pairs(pos, N, box, sigma, eps, r_cut, psi);
    oracle_apply_tols(psi, n * n * n, tol);
    return 0;
}

/* The same third_order (ifc.jl:20-35) restricted to the middle-index columns
 * jj in [j0, j1): out[ii + n*((jj - j0) + w*kk)], w = j1 - j0 (an n × w × n
 * column-major slab).  The pair loop and its 6-way scatter run as in
 * oracle_third_order_lj_pairs, dropping only the writes whose middle index
 * falls outside the slab (every entry is written by exactly one pair
 * iteration, in the same order as there).  ASR! (asr.jl:19-40) at fixed
 * (ii, jj) sums along the third index only, so it stays inside the slab;
 * then apply_tols!.  Equal, entry for entry, to the slab's columns of the
 * full tensor; it lets large cells (400 atoms: 13.8 GB dense) be checked
 * slab by slab.  Returns -1 when the r_cut < L assertion would fire. */
int oracle_third_order_lj_slab(const double* pos, int64_t N, const double box[3], double sigma, double eps,
                               double r_cut, double tol, int64_t j0, int64_t j1, double* out) {
    for (int d = 0; d < 3; ++d)
        if (!(r_cut < box[d])) return -1;
    const int64_t n = 3 * N, w = j1 - j0;
    if (j0 < 0 || j1 > n || w <= 0) return -2;
    memset(out, 0, sizeof(double) * (size_t)(n * w * n));
    const double rc2 = r_cut * r_cut;
#define SLAB_SET(x, y, z, v)                                            \
    do {                                                                \
        if ((y) >= j0 && (y) < j1) out[(x) + n * (((y) - j0) + w * (int64_t)(z))] = (v); \
    } while (0)
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t i = 0; i < N; ++i) {
        for (int64_t j = i + 1; j < N; ++j) {
            for (int dir = 0; dir < 2; ++dir) {
                double r[3];
                for (int x = 0; x < 3; ++x)
                    r[x] = dir == 0 ? pos[3 * i + x] - pos[3 * j + x] : pos[3 * j + x] - pos[3 * i + x];
                oracle_nearest_mirror(r, box);
                double d2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
                if (!(d2 < rc2)) continue;
                double rn = sqrt(d2), d[4];
                oracle_lj_derivs(sigma, eps, rn, d);
                for (int a = 0; a < 3; ++a)
                    for (int b = 0; b < 3; ++b)
                        for (int c = 0; c < 3; ++c) {
                            double val = -oracle_phi3(d, rn, r, a, b, c);
                            int64_t ii, jj, kk;
                            if (dir == 0) { ii = 3 * i + a; jj = 3 * i + b; kk = 3 * j + c; }
                            else          { ii = 3 * i + a; jj = 3 * j + b; kk = 3 * j + c; }
                            SLAB_SET(ii, jj, kk, val); SLAB_SET(ii, kk, jj, val);
                            SLAB_SET(jj, kk, ii, val); SLAB_SET(jj, ii, kk, val);
                            SLAB_SET(kk, ii, jj, val); SLAB_SET(kk, jj, ii, val);
                        }
            }
        }
    }
#undef SLAB_SET
    /* asr.jl:19-40 on the slab's columns (ascending strided sum over kk). */
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t i = 0; i < N; ++i)
        for (int64_t jj = j0; jj < j1; ++jj)
            for (int a = 0; a < 3; ++a) {
                int64_t ii = 3 * i + a;
                double* col = out + ii + n * (jj - j0);
                for (int c = 0; c < 3; ++c) {
                    int64_t kk = 3 * i + c;
                    col[n * w * kk] = 0.0;
                    double s = 0.0;
                    for (int64_t k = c; k < n; k += 3) s += col[n * w * k];
                    col[n * w * kk] = -s;
                }
            }
    oracle_apply_tols(out, n * w * n, tol);
    return 0;
}

int oracle_second_order_lj_full(const double* pos, int64_t N, const double box[3], double sigma,
                                double eps, double r_cut, double tol, double* ifc2) {
    const int64_t n = 3 * N;
    memset(ifc2, 0, sizeof(double) * (size_t)(n * n));
    oracle_second_order_lj(pos, N, box, sigma, eps, r_cut, ifc2);
    oracle_apply_tols(ifc2, n * n, tol);
    return 0;
}

/* third_order_analytical.jl:185-214 — serial, reference loop order (the
 * innermost γ walks the slowest dimension). */
void oracle_mass_weight3(double* psi, const double* masses, int64_t N) {
    const int64_t n = 3 * N;
    for (int64_t i = 0; i < N; ++i)
        for (int64_t j = 0; j < N; ++j)
            for (int64_t k = 0; k < N; ++k)
                for (int a = 0; a < 3; ++a)
                    for (int b = 0; b < 3; ++b)
                        for (int c = 0; c < 3; ++c) {
                            int64_t ii = 3 * i + a, jj = 3 * j + b, kk = 3 * k + c;
                            double* p = psi + ii + n * (jj + n * kk);
                            if (*p != 0.0) *p = *p / sqrt((masses[i] * masses[j]) * masses[k]);
                        }
}

/* The user-side cast `CuArray{Float32}(ifc3.values)` (README.md:73-75). */
void oracle_cast_f32(const double* src, float* dst, int64_t len) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < len; ++i) dst[i] = (float)src[i];
}

int oracle_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void oracle_set_num_threads(int t) {
#ifdef _OPENMP
    if (t > 0) omp_set_num_threads(t);
#else
    (void)t;
#endif
}
